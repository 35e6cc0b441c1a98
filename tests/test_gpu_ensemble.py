"""Batched ensemble (ch4_ensemble_*): many lattices of different sizes in one
work-queue launch per step.

* every lattice advances exactly as it does alone (same kernel, per-cell work
  independent of the tile schedule) -- bit-identical populations;
* the ensemble path agrees with the single-lattice FP32 path and, in FP32, with
  the FP64 oracle within the reduced-precision tolerance;
* the tuner leaves the state untouched; admission by device memory refuses a slot
  that does not fit and accepts it after another slot leaves.
"""
import numpy as np
import pytest

import oracle as O
from lbcases import W, pops, rb_temperature_pops, run_restatement

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import abi  # noqa: E402

RB_FLAGS = ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
            "LB_TEMPERATURE_BC_Y"]


def rb_case(NX, NY, NZ, ra, seed, storage=abi.STORE_F32):
    bg = 0.05 ** 2 / NY
    nu = (bg * NY ** 3 / ra) ** 0.5
    cfg = O.make_config(NX, NY, NZ, RB_FLAGS, storage=storage, tau_u=0.5 + 3 * nu, tau_t=0.5 + 3 * nu, beta_t=1.0,
                        gravity_y=bg, T_bot=1.0, T_top=0.0, T_ref=0.5)
    rng = np.random.default_rng(seed)
    state = {"p": pops(rng, NX, NY, NZ, 1.0, 1e-3), "g": rb_temperature_pops(rng, NX, NY, NZ, 1.0, 0.0, 1e-3)}
    return cfg, state


CASES = [(16, 12, 1, 1e4, 1), (40, 20, 1, 3e4, 2), (24, 16, 3, 1e5, 3), (64, 24, 1, 2e5, 4), (12, 30, 2, 5e4, 5),
         (33, 17, 1, 8e4, 6)]


def run_ensemble(cases, nsteps, shape=None, tune=False, storage=abi.STORE_F32):
    out = []
    with ch4b200.Ensemble(storage) as ens:
        slots = []
        for cfg, st in cases:
            s = ens.add(cfg)
            ens.set_pop(s, "p", st["p"])
            ens.set_pop(s, "g", st["g"])
            ens.initialize(s)
            slots.append(s)
        if shape:
            ens.set_shape(*shape)
        if tune:
            ens.tune()
        ens.step(nsteps)
        ens.synchronize()
        for s in slots:
            out.append({"p": ens.get_pop(s, "p"), "g": ens.get_pop(s, "g"), "itime": ens.itime(s),
                        "avg": ens.averages(s), **ens.fields(s)})
    return out


def test_each_case_same_alone_and_in_the_mix():
    cases = [rb_case(*c) for c in CASES]
    mix = run_ensemble(cases, 37, shape=(128, 2))
    for (cfg, st), m in zip(cases, mix):
        alone = run_ensemble([(cfg, st)], 37, shape=(256, 4))[0]
        assert m["itime"] == 37
        assert np.array_equal(m["p"], alone["p"]) and np.array_equal(m["g"], alone["g"])


def test_ensemble_matches_single_lattice_fp32():
    cases = [rb_case(*c) for c in CASES[:3]]
    mix = run_ensemble(cases, 25)
    for (cfg, st), m in zip(cases, mix):
        with ch4b200.Simulation(cfg) as sim:
            sim.set_pop("p", st["p"])
            sim.set_pop("g", st["g"])
            sim.initialize()
            sim.step(25)
            p, g = sim.get_pop("p"), sim.get_pop("g")
        assert np.abs(m["p"] - p).max() <= 1e-6 * np.abs(p).max()
        assert np.abs(m["g"] - g).max() <= 1e-6 * np.abs(g).max()


def test_ensemble_fp32_close_to_fp64_oracle():
    cases = [rb_case(*c) for c in CASES[:4]]
    mix = run_ensemble(cases, 60)
    for (cfg, st), m in zip(cases, mix):
        cfg64 = O.make_config(cfg.NX, cfg.NY, cfg.NZ, RB_FLAGS, tau_u=cfg.tau_u, tau_t=cfg.tau_t, beta_t=1.0,
                              gravity_y=cfg.gravity_y, T_bot=1.0, T_top=0.0, T_ref=0.5)
        ref = run_restatement(cfg64, st, 60)
        # FP32 arithmetic and storage: T within 1e-5 relative L2 after 60 steps
        assert np.linalg.norm(m["t"] - ref["t"]) / np.linalg.norm(ref["t"]) < 1e-5
        # Nusselt number (dump_averages nuy = <u_y T - kappa dT/dy> / (kappa dT / H)): the FP32
        # velocity carries about one unit roundoff (2^-24) of error, which the division by the
        # small conductive flux kappa*dT/H (1e-4 .. 5e-4 here) amplifies; allow 4 unit roundoffs
        flux = cfg64.kappa * (cfg64.T_bot - cfg64.T_top) / cfg64.SY
        assert abs(m["avg"]["nuy"] - ref["avg"]["nuy"]) <= 4 * 2.0 ** -24 / flux


def test_tuner_keeps_state():
    cases = [rb_case(*c) for c in CASES[:4]]
    a = run_ensemble(cases, 10, shape=(256, 2))
    b = run_ensemble(cases, 10, tune=True)
    for x, y in zip(a, b):
        assert np.array_equal(x["p"], y["p"]) and np.array_equal(x["g"], y["g"])


def test_admission_by_device_memory():
    cfg, st = rb_case(64, 32, 1, 1e5, 1)
    need = ch4b200.ensemble_slot_bytes(cfg, abi.STORE_F32)
    with ch4b200.Ensemble(abi.STORE_F32, budget_bytes=int(need * 1.5)) as ens:
        s0 = ens.add(cfg)
        with pytest.raises(ch4b200.CH4Error) as e:
            ens.add(cfg)
        assert e.value.status == abi.ERR_NOMEM
        ens.remove(s0)
        s1 = ens.add(cfg)
        assert ens.bytes_in_use() == need
        ens.set_pop(s1, "p", st["p"])
        ens.set_pop(s1, "g", st["g"])
        ens.initialize(s1)
        ens.step(3)
        ens.synchronize()
        assert ens.itime(s1) == 3


def test_ensemble_rejects_hit_and_mixed_sets():
    with ch4b200.Ensemble(abi.STORE_F32) as ens:
        hit = O.make_config(8, 8, 8, ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT"], tau_u=0.6)
        with pytest.raises(ch4b200.CH4Error) as e:
            ens.add(hit)
        assert e.value.status == abi.ERR_UNSUPPORTED
        ens.add(rb_case(8, 8, 1, 1e4, 1)[0])
        kol = O.make_config(8, 8, 8, ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_KOLMOGOROV"], tau_u=0.6)
        with pytest.raises(ch4b200.CH4Error):
            ens.add(kol)


def test_fp16_ensemble_matches_single_lattice_fp16_and_fp64_bounds():
    """FP16-deviation storage in the ensemble: the same per-cell arithmetic as the
    single-lattice FP16 path -- a last-place FP32 difference can flip the rounding of a
    stored half, so agreement is within two FP16 ulps (2^-9 relative) of the largest
    stored deviation f - w*shift -- and the FP16 error bound of the single-lattice
    parity tests against the FP64 oracle (T within 2e-2 relative L2)."""
    cases = [rb_case(*c, storage=abi.STORE_F16) for c in CASES[:3]]
    mix = run_ensemble(cases, 30, storage=abi.STORE_F16)
    for (cfg, st), m in zip(cases, mix):
        with ch4b200.Simulation(cfg) as sim:
            sim.set_pop("p", st["p"])
            sim.set_pop("g", st["g"])
            sim.initialize()
            sim.step(30)
            p, g = sim.get_pop("p"), sim.get_pop("g")
        dev_p = np.abs(p - W * 1.0).max()
        dev_g = np.abs(g - W * 0.5).max()
        assert np.abs(m["p"] - p).max() <= 2.0 ** -9 * dev_p
        assert np.abs(m["g"] - g).max() <= 2.0 ** -9 * dev_g
        cfg64 = O.make_config(cfg.NX, cfg.NY, cfg.NZ, RB_FLAGS, tau_u=cfg.tau_u, tau_t=cfg.tau_t, beta_t=1.0,
                              gravity_y=cfg.gravity_y, T_bot=1.0, T_top=0.0, T_ref=0.5)
        ref = run_restatement(cfg64, st, 30)
        assert np.linalg.norm(m["t"] - ref["t"]) / np.linalg.norm(ref["t"]) < 2e-2
