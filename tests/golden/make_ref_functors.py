"""Generate tests/golden/ref_functors.json from the reference's own
host-callable functors (EvaluatorLJ::force, PairEvaluatorLJ.h:17-60;
EvaluatorLJFS::force/energy, PairEvaluatorLJFS.h:15-57;
EvaluatorE3B switching / pair energy / force, EvaluatorE3B.h:67-249),
compiled from the reference source by oracle/ref.mk into oracle/_ref.

Run in a checkout where the reference source is present:
    make -f oracle/ref.mk && python tests/golden/make_ref_functors.py
The committed JSON lets the CPU tests pin the oracle without the reference."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import refkernels as R  # noqa: E402


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/librefkernels.so is not built")
    rng = np.random.default_rng(20261203)
    lj = []
    for _ in range(40):
        dr = rng.uniform(-3, 3, 3)
        if np.linalg.norm(dr) < 2.0:
            continue
        lj.append({"sigma": 3.0, "eps": 6.0, "rcut": 10.0, "dr": [float(v) for v in dr.astype(np.float32)],
                   "force": [float(v) for v in R.lj_force_host(3.0, 6.0, 10.0, dr)]})
    ljfs = []
    for _ in range(40):
        dr = rng.uniform(-2.0, 2.0, 3)
        if not 0.9 < np.linalg.norm(dr) < 2.5:
            continue
        o = R.ljfs_host(1.1, 0.8, 2.5, dr)
        ljfs.append({"sigma": 1.1, "eps": 0.8, "rcut": 2.5, "dr": [float(v) for v in dr.astype(np.float32)],
                     "force": [float(v) for v in o[:3]], "energy": float(o[3])})
    e3b = []
    for r in np.linspace(0.8, 5.5, 48):
        e3b.append({"r": float(r), "out": [float(v) for v in R.e3b_single_host(float(r))]})
    out = {"source": "reference functors compiled from source by oracle/ref.mk (EvaluatorLJ::force; "
                     "EvaluatorLJFS::force/energy on the parameters EvaluatorLJFS::forcePy forms; "
                     "EvaluatorE3B E3B3 single O-H term: switching, energy, force)",
           "lj": lj, "ljfs": ljfs, "e3b3_single": e3b}
    with open(os.path.join(HERE, "ref_functors.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(lj)} LJ, {len(ljfs)} LJFS and {len(e3b)} E3B vectors")


if __name__ == "__main__":
    main()
