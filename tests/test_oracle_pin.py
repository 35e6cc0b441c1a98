"""Pin the oracle: the C restatement (oracle/ch4_oracle.c) against the reference
solver itself, compiled from its own sources (oracle/Makefile -> oracle/_ref), on
the same seeded inputs.  The reference has no golden vectors of its own (its src/tests
directory is empty), so the compiled reference is the pin; the committed fixtures in
tests/golden/ (made by tests/golden/make_golden.py from the same binaries) keep the pin
available where the reference build is absent."""
import os

import numpy as np
import pytest

import oracle as O
from lbcases import CASES, make_case, pop_items, run_restatement

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _assert_same(a, b, what):
    assert a.shape == b.shape, what
    # bit-identical (IEEE equality; +0 and -0 compare equal)
    assert np.array_equal(a, b), "%s differs: max |d| = %g" % (what, np.abs(a - b).max())


@pytest.mark.parametrize("name,nsteps", [("kolmogorov", 20), ("rb", 20), ("hit", 15), ("walls2", 20),
                                          ("scalar", 20), ("les", 20), ("particles", 8),
                                          ("particles_t", 8), ("particles_g", 8), ("particles_1w", 8),
                                          ("particles_or", 8),
                                          ("trt", 20), ("trt_les", 20), ("les_vd", 20), ("les_ls", 20),
                                          ("les_wale", 20), ("les_ts", 20), ("particles_tc", 8), ("nozero", 15),
                                          ("cpower", 15), ("duct", 20), ("duct_les", 20), ("box", 20),
                                          ("slipx", 20), ("slipz", 20), ("particles_tt", 8), ("particles_ttc", 8),
                                          ("particles_rb", 8), ("particles_duct", 8), ("particles_slip", 8),
                                          ("particles_reinj", 8), ("particles_bc", 8), ("les_lilly", 20),
                                          ("particles_or2", 8), ("particles_swimt", 8), ("particles_swimb", 8),
                                          ("particles_swims", 8), ("particles_swimn", 8), ("particles_rdiff", 8),
                                          ("particles_rand", 8), ("les_sism", 20), ("les_kalman", 20),
                                          ("particles_jump", 8), ("particles_jumpt", 8),
                                          ("particles_rjr", 8), ("particles_orbc", 8),
                                          ("particles_sed", 8), ("particles_rad", 8)])
def test_restatement_matches_compiled_reference(name, nsteps):
    flagset, cfg, state = make_case(name, seed=3)
    if not O.ref_available(flagset):
        pytest.skip("reference build oracle/_ref/%s missing" % flagset)
    ref = O.run_reference(flagset, cfg, nsteps, dict(pop_items(state)), parts=state.get("part"))
    mine = run_restatement(cfg, state, nsteps)
    if "phi" in ref:
        _assert_same(mine["phi"], ref["phi"], "HIT phases")
    for k, _ in pop_items(state):
        _assert_same(mine[k], ref[k], "%s populations" % k)
    if "part" in ref:
        for f, v in ref["part"].items():
            _assert_same(mine["part"][f], v, "particle field " + f)
    # global averages of dump_averages, same summation order -> identical
    for k, v in ref["avg"].items():
        assert mine["avg"][k] == v, "average %s: %r vs %r" % (k, mine["avg"][k], v)
    _assert_same(mine["u"], ref["u"], "u")
    _assert_same(mine["dens"], ref["dens"], "dens")
    if "t" in ref:
        _assert_same(mine["t"], ref["t"], "t")
    if "s" in ref:
        _assert_same(mine["s"], ref["s"], "s")
    _assert_same(mine["force"], ref["force"], "force")


@pytest.mark.parametrize("flagset", sorted(O.FLAGSETS))
def test_flagset_headers_match_product_flags(flagset):
    """oracle/configs/<flagset>.h, read by the product's define.h reader, gives the
    flag bits the tests use for that flag set."""
    import ch4b200
    from ch4b200 import abi
    cfg = ch4b200.default_config()
    ch4b200.read_define(cfg, os.path.join(os.path.dirname(O.__file__), "configs", flagset + ".h"))
    assert cfg.flags == abi.flags_of(O.FLAGSETS[flagset])
    assert cfg.flags2 == abi.flags2_of(O.FLAGSETS[flagset])
    assert cfg.t0_kind == O.FLAGSET_EXTRA.get(flagset, {}).get("t0_kind", abi.T0_MEAN)


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_golden_fixture(name):
    path = os.path.join(GOLDEN, "%s.npz" % name)
    if not os.path.exists(path):
        pytest.skip("fixture %s not generated" % path)
    g = np.load(path)
    flagset, cfg, state = make_case(name, seed=int(g["seed"]))
    import hashlib
    for k, v in pop_items(state):
        h = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
        assert h == str(g["in_sha256_" + k]), "case generator changed for %s" % k
    mine = run_restatement(cfg, state, int(g["nsteps"]))
    for k, _ in pop_items(state):
        _assert_same(mine[k], g["out_" + k], k)
    for f in ("x", "y", "z", "vx", "vy", "vz", "ux", "Dt_ux", "t", "dt_t", "Dt_t", "dx_t", "t_p", "px", "py", "pz",
              "dt_px", "nx", "ny", "nz", "dt_nx", "sediment"):
        if "out_part_" + f in g.files:
            _assert_same(mine["part"][f], g["out_part_" + f], "particle " + f)
    for k in ("u", "t", "s", "phi"):
        if "out_" + k in g.files:
            _assert_same(mine[k], g["out_" + k], k)


def test_two_way_deposit_is_active():
    """The particle case really feeds momentum back: its force field differs from
    the same flow without the deposit (HIT forcing only)."""
    _, cfg, state = make_case("particles", seed=3)
    with_dep = run_restatement(cfg, state, 4)
    from ch4b200 import abi
    cfg2 = make_case("particles", seed=3)[1]
    cfg2.flags &= ~(abi.FLAGS["LAGRANGE_TWOWAY"] | abi.FLAGS["LAGRANGE_TWOWAY_MOMENTUM"])
    no_dep = run_restatement(cfg2, state, 4)
    assert np.abs(with_dep["force"] - no_dep["force"]).max() > 1e-12


@pytest.mark.parametrize("name", sorted(__import__("scalecases").MULTIBLOCK))
def test_restatement_reproduces_the_config_digests(name):
    """The restatement on the wide lattices of tests/scalecases.py reproduces the
    compiled reference's output digests (tests/golden/config_digests.json) bit for bit.
    (The 64^3 x 2000-step case is checked on the GPU only: minutes on one core.)"""
    import json
    import scalecases as S
    with open(os.path.join(GOLDEN, "config_digests.json")) as f:
        want = json.load(f)[name]
    flagset, cfg, state, steps = S.case(name)
    for k, v in pop_items(state):
        assert S.digest(v) == want["inputs"][k], "case generator changed for %s" % k
    mine = run_restatement(cfg, state, steps)
    for k, d in want["outputs"].items():
        assert S.digest(mine[k]) == d, k
    if "particles" in want:
        for f, d in want["particles"].items():
            assert S.digest(mine["part"][f]) == d, "particle " + f
    assert S.kinetic_energy(mine["u"]) == want["kinetic_energy"]
