"""The integration patch of the library's guide, compiled: the reference's own sources
built with -DCH4_B200 (oracle/harness/ref_harness.c follows src/main.c and carries the
patch's block), linked to ch4-project_b200/ch4b200/libch4b200.so, its time loop running
through include/ch4.h.  On the CPU: the patched build compiles and links against the
library.  On the GPU: it reproduces the unpatched reference run bit for bit (FP64)."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from lbcases import make_case, pop_items

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLAGSETS = ["kolmogorov", "rb", "hit", "scalar", "les"]
CASE = {"kolmogorov": "kolmogorov", "rb": "rb", "hit": "hit", "scalar": "scalar", "les": "les"}


def _ref_src():
    src = os.environ.get("CH4_REF_SRC") or os.path.join(os.path.dirname(REPO), "reference", "src")
    return src if os.path.isdir(src) else None


def test_patched_reference_builds_and_links_the_library():
    src = _ref_src()
    if src is None:
        pytest.skip("reference sources absent")
    r = subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref-b200", "CFG=rb", "REF_SRC=" + src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    exe = os.path.join(REPO, "oracle", "_ref", "rb", "ch4ref_b200")
    dyn = subprocess.run(["readelf", "-d", exe], capture_output=True, text=True).stdout
    assert "libch4b200.so" in dyn and "$ORIGIN" in dyn


@pytest.mark.gpu
@pytest.mark.parametrize("flagset", FLAGSETS)
def test_patched_reference_reproduces_the_reference(flagset):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not (O.ref_available(flagset) and os.path.exists(O.ref_binary(flagset) + "_b200")):
        pytest.skip("reference builds missing")
    _, cfg, state = make_case(CASE[flagset], seed=51)
    pops = dict(pop_items(state))
    plain = O.run_reference(flagset, cfg, 20, pops)
    patched = O.run_reference(flagset, cfg, 20, pops, patched=True)
    for k in ("p", "g", "h", "u", "dens", "t", "s", "force", "phi"):
        if k in plain:
            assert np.array_equal(patched[k], plain[k]), "%s differs (max %g)" % (
                k, np.abs(patched[k] - plain[k]).max())
