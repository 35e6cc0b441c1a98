"""GPU parity: the CUDA step (through the C ABI, libch4b200.so) against the oracle.

FP64 storage/arithmetic must be bit-identical to the oracle restatement and to the
compiled reference (both FP64, contraction off).  The FP32 and FP16-deviation forms
are checked against the FP64 oracle with the tolerances written below.
"""
import numpy as np
import pytest

import oracle as O
from lbcases import make_case, pop_items, run_restatement

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402


def run_gpu(cfg, state, nsteps, phi=None):
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        if "part" in state:
            sim.set_particles(state["part"])
        if phi is not None:
            sim.set_hit_phases(phi)
        sim.initialize()
        sim.step(nsteps)
        out = {k: sim.get_pop(k) for k, _ in pop_items(state)}
        if "part" in state:
            out["part"] = O.particles_as_dict(sim.get_particles(len(state["part"])))
        out.update(sim.fields())
        out["force"] = sim.force()
        out["avg"] = sim.averages()
        out["itime"] = sim.itime
        out["phi"] = sim.get_hit_phases()
    return out


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("name,nsteps", [("kolmogorov", 25), ("rb", 25), ("hit", 20), ("walls2", 25),
                                          ("scalar", 25), ("les", 25), ("particles", 12),
                                          ("particles_t", 12), ("particles_g", 12), ("particles_1w", 12),
                                          ("particles_or", 12),
                                          ("trt", 25), ("trt_les", 25), ("les_vd", 25), ("les_ls", 25),
                                          ("les_ts", 25), ("particles_tc", 12), ("duct", 25), ("duct_les", 25),
                                          ("box", 25), ("slipx", 25), ("slipz", 25), ("particles_tt", 12),
                                          ("particles_ttc", 12), ("particles_rb", 12), ("particles_duct", 12),
                                          ("particles_slip", 12), ("particles_reinj", 12), ("particles_bc", 12),
                                          ("particles_or2", 12), ("particles_swimt", 12), ("particles_swimb", 12),
                                          ("particles_swims", 12), ("particles_swimn", 12), ("particles_rdiff", 12),
                                          ("particles_rand", 12), ("les_sism", 25), ("les_kalman", 25),
                                          ("particles_rjr", 12), ("particles_orbc", 12),
                                          ("particles_sed", 12), ("particles_rad", 12)])
def test_fp64_bit_identical_to_oracle(name, nsteps):
    _, cfg, state = make_case(name, seed=11)
    ref = run_restatement(cfg, state, nsteps)
    gpu = run_gpu(cfg, state, nsteps)
    assert gpu["itime"] == nsteps
    if "part" in state:
        for f in ref["part"]:
            assert np.array_equal(gpu["part"][f], ref["part"][f]), "particle %s: max |d| %g" % (
                f, np.abs(gpu["part"][f] - ref["part"][f]).max())
    for k, _ in pop_items(state):
        assert np.array_equal(gpu[k], ref[k]), "%s: max |d| %g" % (k, np.abs(gpu[k] - ref[k]).max())
    for k in ("u", "dens", "force"):
        assert np.array_equal(gpu[k], ref[k]), k
    if "g" in state:
        assert np.array_equal(gpu["t"], ref["t"])
    if "h" in state:
        assert np.array_equal(gpu["s"], ref["s"])
    if "phi" in ref:
        assert np.array_equal(gpu["phi"], ref["phi"])


@pytest.mark.parametrize("name", ["kolmogorov", "rb", "hit", "walls2", "scalar", "les", "particles",
                                  "particles_t", "particles_g", "trt", "trt_les", "les_vd", "les_ls", "les_ts",
                                  "particles_tc", "duct", "duct_les", "box", "slipx", "slipz", "particles_tt",
                                  "particles_ttc", "particles_rb", "particles_duct", "particles_slip",
                                  "particles_reinj", "particles_bc", "particles_or2", "particles_swimt",
                                  "particles_swimb", "particles_swims", "particles_swimn", "particles_rdiff",
                                  "particles_rand", "les_sism", "les_kalman", "particles_rjr", "particles_orbc",
                                  "particles_sed", "particles_rad"])
def test_fp64_matches_compiled_reference(name):
    flagset, cfg, state = make_case(name, seed=5)
    if not O.ref_available(flagset):
        pytest.skip("reference build missing")
    ref = O.run_reference(flagset, cfg, 30, dict(pop_items(state)), parts=state.get("part"))
    gpu = run_gpu(cfg, state, 30)
    if "part" in ref:
        for f, v in ref["part"].items():
            assert np.array_equal(gpu["part"][f], v), "particle " + f
    for k, _ in pop_items(state):
        assert np.array_equal(gpu[k], ref[k]), k
    assert np.array_equal(gpu["u"], ref["u"])


# reduced precision: FP32 arithmetic with FP32 / FP16-deviation storage
# FP32: relative L2 of u within 1e-3 (u ~ 1e-3..1e-5 here, so this is ~1e-8 absolute),
# of rho within 1e-5, of T within 1e-6 (40 steps).
# FP16 deviations (11-bit mantissa): u within 0.2, rho within 1e-3, T within 2e-2.
@pytest.mark.parametrize("storage,tol_u,tol_rho,tol_t", [(1, 1e-3, 1e-5, 1e-6), (2, 0.2, 1e-3, 2e-2)])
@pytest.mark.parametrize("name", ["kolmogorov", "rb", "scalar", "hit", "trt", "box"])
def test_reduced_precision_error_bounds(name, storage, tol_u, tol_rho, tol_t):
    _, cfg64, state = make_case(name, seed=2)
    _, cfg, _ = make_case(name, seed=2, storage=storage)
    ref = run_restatement(cfg64, state, 40)
    gpu = run_gpu(cfg, state, 40)
    eu = rel_l2(gpu["u"], ref["u"])
    assert eu < tol_u, "u rel L2 %g" % eu
    er = rel_l2(gpu["dens"], ref["dens"])
    assert er < tol_rho, "rho rel L2 %g" % er
    if "g" in state:
        et = rel_l2(gpu["t"], ref["t"])
        assert et < tol_t, "t rel L2 %g" % et


@pytest.mark.parametrize("name", ["les_sism", "les_kalman", "les_lilly", "particles_jump", "particles_rdiff",
                                  "particles_swims", "particles_rb", "duct"])
def test_fp32_newer_flag_sets_close_to_fp64(name):
    """The FP32 path of the flag sets added with the later features: the lattice in FP32
    arithmetic and storage (particles keep FP64 state) stays within 1e-2 relative L2 of u
    after 20 steps of the FP64 oracle (eddy-viscosity switches such as SISM's |S| > |S_mean|
    may flip on a rounding difference, hence the looser bound than the plain flows')."""
    _, cfg64, state = make_case(name, seed=31)
    _, cfg, _ = make_case(name, seed=31, storage=1)
    ref = run_restatement(cfg64, state, 20)
    gpu = run_gpu(cfg, state, 20)
    assert rel_l2(gpu["u"], ref["u"]) < 1e-2
    if "part" in state:
        for f in ("x", "y", "z"):
            assert np.abs(gpu["part"][f] - ref["part"][f]).max() < 1e-4, f


def test_larger_lattice_bit_identical():
    # 32x24x16 thermal convection, 120 steps: FP64 GPU == oracle
    _, cfg, state = make_case("rb", seed=9)
    import lbcases
    rng = np.random.default_rng(9)
    cfg.NX, cfg.NY, cfg.NZ = 32, 24, 16
    cfg.SX, cfg.SY, cfg.SZ = 32.0, 24.0, 16.0
    state = {"p": lbcases.pops(rng, 32, 24, 16, 1.0, 1e-2),
             "g": lbcases.rb_temperature_pops(rng, 32, 24, 16, 1.0, 0.0, 1e-2)}
    ref = run_restatement(cfg, state, 120)
    gpu = run_gpu(cfg, state, 120)
    assert np.array_equal(gpu["p"], ref["p"])
    assert np.array_equal(gpu["g"], ref["g"])


def test_particles_fp32_fluid_close_to_fp64():
    """FP32 lattice arithmetic (FP64 particle state): positions after 30 steps
    within 1e-6 relative L2 of the FP64 oracle."""
    _, cfg64, state = make_case("particles", seed=4)
    _, cfg, _ = make_case("particles", seed=4, storage=1)
    ref = run_restatement(cfg64, state, 30)
    gpu = run_gpu(cfg, state, 30)
    pos = lambda d: np.stack([d["part"][k] for k in ("x", "y", "z")])
    assert rel_l2(pos(gpu), pos(ref)) < 1e-6


@pytest.mark.parametrize("name", ["kolmogorov", "rb", "walls2", "scalar", "particles", "box", "duct"])
def test_fp64_averages_match_oracle(name):
    """Global sums of dump_averages: the device's double-double reduction against the
    oracle's sequential FP64 sum -- within 1e-12 relative, cancelling means within the
    rounding bound of the sequential sum."""
    _, cfg, state = make_case(name, seed=13)
    ref = run_restatement(cfg, state, 15)
    gpu = run_gpu(cfg, state, 15)
    # a mean whose terms cancel (u_x, dT/dx, u_x T over the box) is held to the bound of
    # a sequential sum, N eps max|term|, instead of 1e-12 of its small value
    n = cfg.NX * cfg.NY * cfg.NZ
    umax, tmax = np.abs(ref["u"]).max(), np.abs(ref["t"]).max()
    # the Nusselt numbers combine <u T> and kappa <dT> over kappa deltaT / S (src/output.c:577-579)
    nu_norm = cfg.kappa * abs(cfg.deltaT) / cfg.SY if cfg.deltaT else 1.0
    scale = {"u": umax, "d": 2 * tmax, "ut": umax * tmax,
             "nu": (umax * tmax + cfg.kappa * 2 * tmax) / max(nu_norm, 1e-300)}
    for k, v in ref["avg"].items():
        kind = "ut" if k in ("uxt", "uyt", "uzt") else "u" if k in ("ux", "uy", "uz") else \
            "d" if k in ("dxt", "dyt", "dzt") else "nu" if k in ("nux", "nuy", "nuz") else None
        tol = 1e-12 * abs(v) + 1e-18 + (n * 2.2e-16 * scale[kind] if kind else 0.0)
        assert abs(gpu["avg"][k] - v) <= tol, "%s: %r vs %r" % (k, gpu["avg"][k], v)


@pytest.mark.parametrize("name", ["nozero", "cpower"])
def test_fp64_global_force_corrections_close_to_oracle(name):
    """NOZEROMODE / CONSTANT_POWER: the device sums the force field in double-double
    instead of the reference's sequential order, so FP64 agrees with the oracle (and
    the compiled reference) to 1e-12 relative L2 rather than bit for bit; the
    corrected force has zero mean."""
    flagset, cfg, state = make_case(name, seed=17)
    ref = run_restatement(cfg, state, 25)
    gpu = run_gpu(cfg, state, 25)
    for k, _ in pop_items(state):
        assert rel_l2(gpu[k], ref[k]) < 1e-12, k
    for k in ("u", "force"):
        assert rel_l2(gpu[k], ref[k]) < 1e-12, k
    f = gpu["force"].reshape(-1, 3)
    assert np.all(np.abs(f.mean(axis=0)) <= 1e-14 * np.abs(f).max())
    if O.ref_available(flagset):
        r = O.run_reference(flagset, cfg, 25, dict(pop_items(state)))
        assert rel_l2(gpu["u"], r["u"]) < 1e-12


def test_fp64_wale_close_to_oracle_and_reference():
    """LB_FLUID_LES_WALE: the WALE operator takes pow(J, 1.5), pow(S, 2.5), pow(J, 1.25);
    the device pow and the reference's libm differ by an ulp or two, so FP64 agrees with
    the oracle (and the compiled reference) to 1e-12 relative L2 rather than bit for bit."""
    flagset, cfg, state = make_case("les_wale", seed=19)
    ref = run_restatement(cfg, state, 25)
    gpu = run_gpu(cfg, state, 25)
    for k in ("p", "u"):
        assert rel_l2(gpu[k], ref[k]) < 1e-12, k
    if O.ref_available(flagset):
        r = O.run_reference(flagset, cfg, 25, dict(pop_items(state)))
        assert rel_l2(gpu["u"], r["u"]) < 1e-12


def test_fp64_smagorinsky_lilly_close_to_oracle_and_reference():
    """LB_FLUID_LES_SMAGORINSKY_LILLY: the reference forms Ri with pow(|S|, 2.0) from the
    host libm, which differs from the correctly rounded |S|*|S| of the device by an ulp in
    about one cell in a thousand, so FP64 agrees with the oracle (and the compiled
    reference) to 1e-12 relative L2 rather than bit for bit.  The case is a stably
    stratified channel where about half the cells have Ri >= 1 (no eddy viscosity)."""
    flagset, cfg, state = make_case("les_lilly", seed=21)
    ref = run_restatement(cfg, state, 25)
    gpu = run_gpu(cfg, state, 25)
    for k in ("p", "g", "u", "t"):
        assert rel_l2(gpu[k], ref[k]) < 1e-12, k
    if O.ref_available(flagset):
        r = O.run_reference(flagset, cfg, 25, dict(pop_items(state)))
        assert rel_l2(gpu["u"], r["u"]) < 1e-12
    # the correction is on: without the stratification's gravity the flow differs
    _, cfg0, _ = make_case("les_lilly", seed=21, gravity_y=0.0)
    assert rel_l2(run_gpu(cfg0, state, 25)["u"], gpu["u"]) > 1e-9


@pytest.mark.parametrize("name", ["particles_jump", "particles_jumpt"])
def test_fp64_run_and_tumble_close_to_oracle_and_reference(name):
    """LAGRANGE_ORIENTATION_ACTIVE_JUMP: a jumping tracer swims with
    swim_velocity * exp(-time_from_jump / jump_time); the device's exp is within an ulp of the
    host libm's the reference calls, not always equal to it, so FP64 agrees with the oracle
    (and the compiled reference) to 1e-12 relative L2 rather than bit for bit.  The jump
    decisions (shear rate or temperature against the critical value) are identical."""
    flagset, cfg, state = make_case(name, seed=23)
    ref = run_restatement(cfg, state, 12)
    gpu = run_gpu(cfg, state, 12)
    for f in ("x", "y", "z", "vx", "vy", "vz", "time_from_jump", "px_jump"):
        assert rel_l2(gpu["part"][f], ref["part"][f]) < 1e-12, f
    assert np.array_equal(gpu["part"]["time_from_jump"] == 0, ref["part"]["time_from_jump"] == 0)
    for k, _ in pop_items(state):
        assert rel_l2(gpu[k], ref[k]) < 1e-12, k
    if O.ref_available(flagset):
        r = O.run_reference(flagset, cfg, 12, dict(pop_items(state)), parts=state.get("part"))
        for f in ("x", "y", "z"):
            assert rel_l2(gpu["part"][f], r["part"][f]) < 1e-12, f


def test_fp32_global_force_corrections_close_to_fp64():
    _, cfg64, state = make_case("nozero", seed=18)
    _, cfg, _ = make_case("nozero", seed=18, storage=1)
    ref = run_restatement(cfg64, state, 40)
    gpu = run_gpu(cfg, state, 40)
    assert rel_l2(gpu["u"], ref["u"]) < 1e-3
    # FP32 T (~0.5) after 40 steps: a few unit roundoffs (2^-24) per step accumulate
    assert rel_l2(gpu["t"], ref["t"]) < 3e-6
