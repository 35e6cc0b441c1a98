"""Generate tests/golden/config_digests.json from the reference solver compiled by
oracle/Makefile, for the configuration-size parity cases of tests/scalecases.py.

Run here, where the reference sources exist (the 64^3 x 2000-step case takes a few
minutes on one core):  python tests/golden/make_config_digests.py [case ...]

For every case the file keeps the SHA-256 of the seeded inputs, the step count, and
for every output array of the reference's run its SHA-256, its L2 norm and (for the
velocity) the total kinetic energy; the reference's dump_averages sums come along.
tests/test_gpu_config_parity.py runs the same inputs through the C ABI in FP64 and
requires every digest to match.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
REPO = os.path.dirname(TESTS)
for p in (TESTS, os.path.join(REPO, "oracle"), os.path.join(REPO, "ch4-project_b200")):
    sys.path.insert(0, p)
import oracle as O  # noqa: E402
import scalecases as S  # noqa: E402

OUT = os.path.join(HERE, "config_digests.json")


def main(names):
    try:
        with open(OUT) as f:
            book = json.load(f)
    except FileNotFoundError:
        book = {}
    for name in names:
        flagset, cfg, state, steps = S.case(name)
        pops = {k: v for k, v in state.items() if k in ("p", "g", "h")}
        ref = O.run_reference(flagset, cfg, steps, pops, parts=state.get("part"))
        entry = {"flagset": flagset, "lattice": [cfg.NX, cfg.NY, cfg.NZ], "steps": steps,
                 "inputs": {k: S.digest(v) for k, v in pops.items()}, "outputs": {}, "norms": {},
                 "reference_seconds": ref["timing"]["seconds"]}
        for k in S.OUTPUTS:
            if k in ref:
                entry["outputs"][k] = S.digest(ref[k])
                entry["norms"][k] = float(np.linalg.norm(ref[k].ravel()))
        if "part" in ref:
            entry["particles"] = {f: S.digest(ref["part"][f]) for f in S.PARTICLE_OUTPUTS}
        entry["kinetic_energy"] = S.kinetic_energy(ref["u"])
        if "avg" in ref:
            entry["averages"] = ref["avg"]
        book[name] = entry
        print(name, "ok", "%.1f s" % entry["reference_seconds"], flush=True)
    with open(OUT, "w") as f:
        json.dump(book, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or S.NAMES)
