"""Continuous-batching server (ch4b200.serve): requests of different kinds and sizes
share the device; each result is the same alone and in the mix; admission by a
device-memory budget delays but does not lose requests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from ch4b200 import abi  # noqa: E402
from ch4b200.serve import Request, Server, request_config, ensemble_slot_bytes  # noqa: E402


def small_requests():
    return [
        Request(0, "kolmogorov", 16, 130, arrival=0.0),
        Request(1, "rb", 16, 90, arrival=0.0),
        Request(2, "kolmogorov", 24, 60, les=True, arrival=0.01),
        Request(3, "rb", 24, 110, les=True, arrival=0.02),
        Request(4, "kolmogorov", 16, 75, les=True, tracers=500, arrival=0.03),
        Request(5, "rb", 32, 40, arrival=0.04),
        Request(6, "kolmogorov", 32, 150, arrival=0.05),
    ]


@pytest.mark.parametrize("cells_in_flight", [None, 20000])
def test_each_request_same_alone_and_in_the_mix(cells_in_flight):
    mix = Server(abi.STORE_F32, budget_bytes=8 << 30, block=32, cells_in_flight=cells_in_flight).run(small_requests())
    for req in mix:
        assert req.finished is not None and req.latency >= 0
        alone = Server(abi.STORE_F32, budget_bytes=8 << 30, block=32).run(
            [Request(req.rid, req.kind, req.size, req.steps, req.les, req.tracers, 0.0)])[0]
        for k, v in alone.result.items():
            a, b = req.result[k], v
            assert a == b or (np.isnan(a) and np.isnan(b)), "request %d %s: %r vs %r" % (req.rid, k, a, b)


def test_admission_by_memory_budget_queues_requests():
    reqs = [Request(i, "rb", 32, 20 + 5 * i, arrival=0.0) for i in range(6)]
    one = ensemble_slot_bytes(request_config(reqs[0], abi.STORE_F32), abi.STORE_F32)
    srv = Server(abi.STORE_F32, budget_bytes=int(2.5 * one), block=16)
    done = srv.run(reqs)
    assert all(r.finished is not None for r in done)
    # at most two fit at a time: the third is admitted only after one of the first two finished
    order = sorted(done, key=lambda r: r.admitted)
    assert order[2].admitted >= min(order[0].finished, order[1].finished)


def test_cells_in_flight_limits_concurrency():
    reqs = [Request(i, "kolmogorov", 24, 40, arrival=0.0) for i in range(4)]  # 13,824 cells each
    done = Server(abi.STORE_F32, budget_bytes=8 << 30, block=16, cells_in_flight=30000).run(reqs)
    order = sorted(done, key=lambda r: r.admitted)
    # two fit under the cap: the third waits for one of the first two
    assert order[2].admitted >= min(order[0].finished, order[1].finished)
