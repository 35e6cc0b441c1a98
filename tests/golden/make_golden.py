"""Generate tests/golden/<case>.npz from the reference solver compiled by oracle/Makefile.

Run here, where the reference sources exist:  python tests/golden/make_golden.py [case ...]
Each fixture holds the seeded inputs (in_*), the step count and the reference's
outputs (out_*) after that many steps; tests/test_oracle_pin.py checks the oracle
restatement against them.
"""
import os
import sys

import hashlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "ch4-project_b200"))
import oracle as O  # noqa: E402
from lbcases import CASES, make_case, pop_items  # noqa: E402

NSTEPS = 12
SEED = 7

for name in sys.argv[1:] or sorted(CASES):
    flagset, cfg, state = make_case(name, seed=SEED)
    ref = O.run_reference(flagset, cfg, NSTEPS, dict(pop_items(state)), parts=state.get("part"))
    out = {"seed": SEED, "nsteps": NSTEPS}
    if "part" in ref:
        temperature = ("t", "dt_t", "Dt_t", "dx_t") if "t" in ref["part"] else ()
        if "t_p" in ref["part"]:
            temperature += ("t_p",)
        orientation = tuple(f for f in ("px", "py", "pz", "dt_px", "nx", "ny", "nz", "dt_nx") if f in ref["part"])
        orientation += tuple(f for f in ("sediment",) if f in ref["part"])
        for f in ("x", "y", "z", "vx", "vy", "vz", "ux", "Dt_ux") + temperature + orientation:
            out["out_part_" + f] = ref["part"][f]
    for k, v in pop_items(state):
        out["in_sha256_" + k] = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
        out["out_" + k] = ref[k]
    for k in ("u", "t", "s", "phi"):
        if k in ref:
            out["out_" + k] = ref[k]
    np.savez_compressed(os.path.join(HERE, "%s.npz" % name), **out)
    print(name, "ok")
