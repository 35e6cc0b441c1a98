"""Lagrangian averages per particle type (dump_particle_averages,
src/lagrange.c:2598-2931): the oracle's restatement (oracle.particle_averages) against
the particle_averages.dat that the reference, compiled from its own sources, writes
after the same run (the harness's final dump_particle_averages).  The file holds %e
values (6 significant digits), so the restatement must agree to print precision; with
a temperature set the file carries the t columns, with LAGRANGE_OUTPUT_FLUID_AVERAGES
the fluid-velocity columns.
"""
import numpy as np
import pytest

import oracle as O
from lbcases import make_case, pop_items


def expected_rows(avg, time_now, therm, fluid, orient=0, tp=False):
    """The reference's columns (src/lagrange.c:2880-2922): v and a blocks, dp/dt (orient
    >= 1) and dn/dt (orient 2) blocks, the temperature block (+ t_p), the fluid block."""
    rows = []
    for ty, a in enumerate(avg):
        r = [time_now, float(ty)] + a[1:19]
        if orient >= 1:
            r += a[33:42]
        if orient >= 2:
            r += a[42:51]
        if therm:
            r += a[19:24]
            if tp:
                r.append(a[51])
        if fluid:
            r += a[24:33]
        rows.append(r)
    return np.array(rows)


@pytest.mark.parametrize("case,flagset,types,therm,fluid,orient,tp",
                         [("particles", "particles_fa", 3, False, True, 0, False),
                          ("particles_t", "particles_t", 4, True, False, 0, False),
                          ("particles", "particles", 1, False, False, 0, False),
                          ("particles_or2", "particles_or2", 2, False, False, 2, False),
                          ("particles_or", "particles_or", 3, False, False, 1, False),
                          ("particles_tt", "particles_tt", 2, True, False, 0, True)])
def test_restatement_matches_reference_file(case, flagset, types, therm, fluid, orient, tp):
    if not O.ref_available(flagset):
        pytest.skip("reference build oracle/_ref/%s missing" % flagset)
    _, cfg, state = make_case(case, seed=21)
    cfg.particle_types = types
    nsteps = 7
    ref = O.run_reference(flagset, cfg, nsteps, dict(pop_items(state)), parts=state["part"])
    got = np.loadtxt(ref["dat"]["particle_averages.dat"].splitlines(), ndmin=2)
    exp = expected_rows(O.particle_averages(ref["part"], types), float(nsteps), therm, fluid, orient, tp)
    assert got.shape == exp.shape
    assert np.all(np.abs(got - exp) <= 5e-6 * np.abs(exp) + 1e-300)


def test_types_follow_name_modulo():
    part = {f: np.zeros(5) for f in ("name", "vx", "vy", "vz", "ax", "ay", "az")}
    part["name"] = np.array([0.0, 1.0, 2.0, 3.0, 4.0])
    part["vx"] = np.array([1.0, 10.0, 3.0, 100.0, 5.0])
    avg = O.particle_averages(part, 2)
    assert avg[0][0] == 3.0 and avg[1][0] == 2.0           # names 0, 2, 4 / 1, 3
    assert avg[0][1] == (1.0 + 3.0 + 5.0) * (1.0 / 3.0)     # sum times 1/count, as the reference
    assert avg[1][7] == (1e4 + 1e8) * 0.5                   # pow(v, 4)


def test_particle_types_from_param_in(tmp_path):
    import ch4b200
    _, cfg, _ = make_case("particles", seed=1)
    O.write_param_in(str(tmp_path / "param.in"), cfg, 1, {"tau_drag_types": 3, "beta_coeff_types": 2})
    back = ch4b200.default_config()
    back.flags = cfg.flags
    ch4b200.read_param(back, str(tmp_path / "param.in"))
    assert back.particle_types == 6  # tau_drag_types x beta_coeff_types (GRADIENT + ADDEDMASS)
