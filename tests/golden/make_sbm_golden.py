"""Writes tests/golden/sbm10k_seed0.json: the oracle's per-level facts on the
SBM 10k benchmark graph (seed 0, level gain threshold 1e-6), a regression
fixture for the oracle and the GPU path.

    python tests/golden/make_sbm_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from louvaingpu_b200 import graphgen  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    n, s, d, w = graphgen.sbm_10k(seed=0)
    r = O.Run(n, s, d, w, level_min_gain=1e-6)
    out = {
        "about": "oracle run on the SBM 10k graph (n=10,000, 100 blocks, p_in=0.1, p_out=0.0006, seed 0), "
                 "level gain threshold 1e-6; written by make_sbm_golden.py",
        "n_entries": int(len(s)),
        "passes": [lv.passes for lv in r.levels],
        "n_comms": [lv.n_comms for lv in r.levels],
        "q_level": [lv.q for lv in r.levels],
        "largest_community": int(np.bincount(r.final).max()),
        "final_modularity_fp64": O.modularity_fp64(n, s, d, w, r.final),
        "final_partition_level0_head": r.levels[0].part[:64].tolist(),
    }
    with open(os.path.join(HERE, "sbm10k_seed0.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
