"""ch4_averages_noalloc -- the averages reduction for callers that cannot allocate
device memory (a per-step diagnostic inside a stream-ordered loop, where cudaMalloc
would synchronise the device, or a device-memory budget already reserved in full).

It is called through the C ABI on device fields the test owns, twice in a row (the
second call reuses the library's static scratch left over from the first), and its
sums, normalised as src/output.c:498-579, must match the allocating entry point
ch4_averages_get within the tolerance of the other averages tests (1e-12 relative).
This file is collected last so that a failure here cannot stop the other tests.
"""
import numpy as np
import pytest

from lbcases import make_case, pop_items

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import abi  # noqa: E402


def _normalise(raw, cfg, therm, scal):
    h = np.array(raw, dtype=np.float64)
    norm = 1.0 / (cfg.SX * cfg.SY * cfg.SZ)
    h[:9] *= norm
    if therm:
        h[9:18] *= norm
        h[18:21] *= norm / (cfg.kappa * cfg.deltaT / cfg.SY)
    if scal:
        h[21:23] *= norm
    return dict(zip(abi.AVERAGE_FIELDS, h))


@pytest.mark.parametrize("name", ["rb", "scalar", "kolmogorov"])
def test_noalloc_averages_match_allocating_entry_point(name):
    _, cfg, state = make_case(name, seed=21)
    therm = bool(cfg.flags & abi.FLAGS["LB_TEMPERATURE"])
    scal = bool(cfg.flags & abi.FLAGS["LB_SCALAR"])
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.initialize()
        sim.step(17)
        f = sim.fields()
        ref = sim.averages()
    dev = torch.device("cuda", torch.cuda.current_device())
    dens = torch.from_numpy(np.ascontiguousarray(f["dens"])).to(dev)
    u = torch.from_numpy(np.ascontiguousarray(np.moveaxis(f["u"], -1, 0))).to(dev)
    t = torch.from_numpy(np.ascontiguousarray(f["t"])).to(dev) if therm else None
    s = torch.from_numpy(np.ascontiguousarray(f["s"])).to(dev) if scal else None
    stream = torch.cuda.current_stream().cuda_stream
    fw = bool(cfg.flags & abi.FLAGS["LB_FLUID_BC_Y"])
    sw = bool(cfg.flags & (abi.FLAGS["LB_TEMPERATURE_BC_Y"] | abi.FLAGS["LB_SCALAR_BC_Y"]))
    for call in range(2):
        sums = torch.full((23,), float("nan"), dtype=torch.float64, device=dev)
        ch4b200.averages_noalloc(dens.data_ptr(), u.data_ptr(), t.data_ptr() if t is not None else None,
                                 s.data_ptr() if s is not None else None, cfg.NX, cfg.NY, cfg.NZ, fw, sw, cfg.nu,
                                 cfg.kappa, sums.data_ptr(), stream)
        torch.cuda.synchronize()
        got = _normalise(sums.cpu().numpy(), cfg, therm, scal)
        for k, v in ref.items():
            assert abs(got[k] - v) <= 1e-12 * abs(v) + 1e-18, "call %d, %s: %r vs %r" % (call, k, got[k], v)


def test_noalloc_refuses_lattices_above_its_scratch():
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(ch4b200.CH4Error) as e:
        ch4b200.averages_noalloc(x.data_ptr(), x.data_ptr(), None, None, 1024, 1024, 256, 0, 0, 0.01, 0.01,
                                 x.data_ptr(), 0)
    assert e.value.status == abi.ERR_ARG
