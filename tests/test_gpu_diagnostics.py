"""dump_averages in full (ch4_diagnostics, ch4_dump_averages) against the reference.

The compiled reference runs the same seeded case and, after the last step, its own
dump_averages; the harness records every field of the volume averages and of the
x / y / z rulers at full precision, and leaves the ASCII files dump_averages wrote.
The device sums in a fixed parallel order, the reference sequentially: the records
agree within 1e-12 relative (plus 1e-12 of the field's largest value, for means that
cancel to ~0), and every file the reference wrote exists here with the same rows and
columns, equal to print precision (%e: 6 significant digits).
"""
import numpy as np
import pytest

import oracle as O
from lbcases import make_case, pop_items

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402

OWN_FILES = {"define.dat", "numbers.dat", "param.dat"}  # the reference's parameter echoes


def close(a, b, rtol, atol):
    if np.isnan(a) and np.isnan(b):
        return True
    return abs(a - b) <= rtol * abs(b) + atol


@pytest.mark.parametrize("name", ["kolmogorov", "rb", "hit", "walls2", "scalar", "les"])
def test_dump_averages_matches_reference(name, tmp_path):
    flagset, cfg, state = make_case(name, seed=23)
    if not O.ref_available(flagset):
        pytest.skip("reference build missing")
    nsteps = 12
    ref = O.run_reference(flagset, cfg, nsteps, dict(pop_items(state)))
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.initialize()
        sim.step(nsteps)
        got = sim.diagnostics()
        # the harness's call: time_now = nsteps * time_dt, irun = itime / 1
        sim.dump_averages(tmp_path, float(nsteps), nsteps)
    scale = {}
    for (scope, i, field), v in ref["diag"].items():
        scale[field] = max(scale.get(field, 0.0), abs(v) if np.isfinite(v) else 0.0)
    for (scope, i, field), v in ref["diag"].items():
        if scope == "global" and field in ("x", "y", "z"):
            continue  # summed centre coordinates, never normalised or printed
        mine = got["global"][field] if scope == "global" else got[scope][field][i]
        assert close(mine, v, 1e-12, 1e-12 * scale[field]), (scope, i, field, mine, v)
    files = {n: t for n, t in ref["dat"].items() if n not in OWN_FILES}
    assert "velocity_averages.dat" in files
    for fname, text in files.items():
        path = tmp_path / fname
        assert path.exists(), fname
        a = np.loadtxt(path, ndmin=2)
        b = np.loadtxt(text.splitlines(), ndmin=2)
        assert a.shape == b.shape, fname
        colscale = np.nanmax(np.abs(np.where(np.isfinite(b), b, 0.0)), axis=0)
        for r in range(b.shape[0]):
            for q in range(b.shape[1]):
                assert close(a[r, q], b[r, q], 2e-6, 1e-12 * colscale[q]), (fname, r, q, a[r, q], b[r, q])


def test_running_rulers_average_over_calls(tmp_path):
    """Two dumps: the *_run files hold the mean of the two rulers (irun = 2)."""
    _, cfg, state = make_case("rb", seed=24)
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.initialize()
        sim.step(3)
        r1 = sim.diagnostics()["y"]
        sim.dump_averages(tmp_path, 3.0, 1)
        sim.step(3)
        r2 = sim.diagnostics()["y"]
        sim.dump_averages(tmp_path, 6.0, 2)
    run = np.loadtxt(tmp_path / "temperature_averages_y_run.dat")
    assert run.shape == (cfg.NY, 14)
    assert np.allclose(run[:, 1], 0.5 * (r1["t"] + r2["t"]), rtol=2e-6, atol=1e-12)
    assert len(np.loadtxt(tmp_path / "velocity_averages.dat", ndmin=2)) == 2


def test_ascii_field_dumps_identical_to_reference(tmp_path):
    """OUTPUT_ASCII (flag set "ascii" = "rb" + OUTPUT_ASCII, time_dump_field = time_dt): the
    FP64 fields are bit-identical to the reference, so vel.<itime> and temp.<itime> are the
    same text byte for byte."""
    _, cfg, state = make_case("rb", seed=25)
    if not O.ref_available("ascii"):
        pytest.skip("reference build missing")
    nsteps = 9
    ref = O.run_reference("ascii", cfg, nsteps, dict(pop_items(state)), params={"time_dump_field": 1.0})
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.initialize()
        sim.step(nsteps)
        sim.dump_fields_ascii(tmp_path, nsteps)
    assert sorted(ref["run"]) == ["temp.%d" % nsteps, "vel.%d" % nsteps]
    for name, text in ref["run"].items():
        assert (tmp_path / name).read_text() == text, name
