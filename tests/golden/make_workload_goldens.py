"""Writes tests/golden/lfr_seed1.json and tests/golden/rmat16_seed2.json: the
oracle's dendrogram facts on the LFR-style n=2^20 graph (seed 1) and the
R-MAT scale-16 graph (seed 2), with the inputs' fingerprint.  Floats are
stored as hex strings (bit-exact).  Regression fixtures for the oracle and
the GPU path.

    python tests/golden/make_workload_goldens.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from louvaingpu_b200 import graphgen  # noqa: E402
from oracle import oracle as O  # noqa: E402


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def facts(about, n, s, d, w):
    r = O.Run(n, s, d, w)
    return {
        "about": about,
        "n_vertices": int(n),
        "n_entries": int(len(s)),
        "input_sha256": sha(s, d, w),
        "levels": [{"n_vertices": lv.n_vertices, "nnz": lv.nnz, "passes": lv.passes, "n_comms": lv.n_comms,
                    "q_start": lv.q_start.hex(), "q_level": lv.q.hex()} for lv in r.levels],
        "final_partition_sha256": sha(r.final.astype(np.int32)),
        "final_modularity_fp64": O.modularity_fp64(n, s, d, w, r.final).hex(),
    }


def main():
    n, s, d, w = graphgen.lfr()
    out = facts("oracle run on the LFR-style graph (n=2^20, degree exponent 2.5 on [5, 5000], community exponent "
                "1.5 on [50, 50000], mu=0.3, unit weights, seed 1), gain thresholds 1e-7; written by "
                "make_workload_goldens.py", n, s, d, w)
    with open(os.path.join(HERE, "lfr_seed1.json"), "w") as f:
        json.dump(out, f, indent=1)
    n, s, d, w = graphgen.rmat(16)
    out = facts("oracle run on the R-MAT scale-16 graph (edge factor 16, (0.57, 0.19, 0.19, 0.05), integer weights "
                "1..16, seed 2), gain thresholds 1e-7; written by make_workload_goldens.py", n, s, d, w)
    with open(os.path.join(HERE, "rmat16_seed2.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
