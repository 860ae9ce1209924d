"""Writes the workload fixtures of tests/golden/, from the oracle on the CPU:

  lfr_seed1.json, rmat16_seed2.json, rmat22_seed2.json -- dendrogram facts of
      the LFR-style n=2^20 graph (seed 1) and the R-MAT scale-16 and 22
      graphs (seed 2), with the inputs' fingerprint;
  rmat25_seed2_level0.json -- level 0 of the R-MAT scale-25 graph (seed 2):
      input and CSR fingerprints, the decision vectors of one pass from the
      singleton state and from the state after that pass, the one-level
      phase's passes, Q and labels, and the coarse level-1 list and CSR.

Floats are stored as hex strings (bit-exact), arrays as SHA-256 of their
bytes.  Regression fixtures for the oracle and the GPU path.

    python tests/golden/make_workload_goldens.py [lfr rmat16 rmat22 rmat25]

The R-MAT 25 fixture needs about 50 GB of host memory and a few minutes.
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


def pass_decisions(c):
    """Decisions of one pass from the singleton state and of one pass from
    the state that pass commits (both with the decision rule of
    OneLevelKernel.cu:248-422), as int32 arrays."""
    V = c.V
    first = c.decide(np.arange(V, dtype=np.int32), c.k, np.ones(V, np.int32))[0]
    tot = np.bincount(first, weights=c.k, minlength=V)   # integral weights: exact in any order
    second = c.decide(first, tot, np.bincount(first, minlength=V).astype(np.int32))[0]
    return first, second


def csr_sha(c):
    return sha(c.off, c.col, c.w, c.k, c.loopw, c.has_loop)


def facts(about, n, s, d, w, decisions=False):
    r = O.Run(n, s, d, w)
    extra = {}
    if decisions:
        c = O.Csr(n, s, d, w)
        first, second = pass_decisions(c)
        extra = {"csr_sha256": csr_sha(c), "pass1_decisions_sha256": sha(first),
                 "pass2_decisions_sha256": sha(second)}
    return {
        "about": about,
        "n_vertices": int(n),
        "n_entries": int(len(s)),
        "input_sha256": sha(s, d, w),
        "levels": [{"n_vertices": lv.n_vertices, "nnz": lv.nnz, "passes": lv.passes, "n_comms": lv.n_comms,
                    "q_start": lv.q_start.hex(), "q_level": lv.q.hex()} for lv in r.levels],
        "final_partition_sha256": sha(r.final.astype(np.int32)),
        "final_modularity_fp64": O.modularity_fp64(n, s, d, w, r.final).hex(),
        **extra,
    }


def level0_facts(about, n, s, d, w):
    """Level 0 only, for graphs too large for a whole oracle run here."""
    out = {"about": about, "n_vertices": int(n), "n_entries": int(len(s)), "input_sha256": sha(s, d, w)}
    c = O.Csr(n, s, d, w)
    out.update(nnz=int(c.nnz), m=float(c.m).hex(), csr_sha256=csr_sha(c))
    first, second = pass_decisions(c)
    out.update(pass1_decisions_sha256=sha(first), pass2_decisions_sha256=sha(second))
    del c, first, second
    r = O.Run(n, s, d, w, max_levels=1)
    lv = r.levels[0]
    out.update(passes=lv.passes, n_comms=lv.n_comms, q_start=lv.q_start.hex(), q_level=lv.q.hex(),
               labels_sha256=sha(lv.labels), partition_sha256=sha(lv.part))
    cs, cd, cw = O.induce(n, s, d, w, lv.part)
    out.update(coarse_entries=int(len(cs)), coarse_list_sha256=sha(cs, cd, cw))
    cc = O.Csr(lv.n_comms, cs, cd, cw)
    out.update(coarse_nnz=int(cc.nnz), coarse_csr_sha256=csr_sha(cc))
    return out


def write(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, indent=1)


RMAT = "edge factor 16, (0.57, 0.19, 0.19, 0.05), integer weights 1..16, seed 2"


def main(which):
    if "lfr" in which:
        n, s, d, w = graphgen.lfr()
        write("lfr_seed1.json", facts(
            "oracle run on the LFR-style graph (n=2^20, degree exponent 2.5 on [5, 5000], community exponent "
            "1.5 on [50, 50000], mu=0.3, unit weights, seed 1), gain thresholds 1e-7; written by "
            "make_workload_goldens.py", n, s, d, w))
    if "rmat16" in which:
        n, s, d, w = graphgen.rmat(16)
        write("rmat16_seed2.json", facts(
            f"oracle run on the R-MAT scale-16 graph ({RMAT}), gain thresholds 1e-7; written by "
            "make_workload_goldens.py", n, s, d, w))
    if "rmat22" in which:
        n, s, d, w = graphgen.rmat(22)
        write("rmat22_seed2.json", facts(
            f"oracle run on the R-MAT scale-22 graph ({RMAT}), gain thresholds 1e-7, with the level-0 CSR and "
            "the decision vectors of a pass from the singleton state and of the pass after it; written by "
            "make_workload_goldens.py", n, s, d, w, decisions=True))
    if "rmat25" in which:
        n, s, d, w = graphgen.rmat(25)
        write("rmat25_seed2_level0.json", level0_facts(
            f"oracle on level 0 of the R-MAT scale-25 graph ({RMAT}), gain threshold 1e-7: CSR, the decision "
            "vectors of a pass from the singleton state and of the pass after it, the one-level phase, the "
            "coarse level-1 list and its CSR; written by make_workload_goldens.py", n, s, d, w))


if __name__ == "__main__":
    main(sys.argv[1:] or ["lfr", "rmat16", "rmat22", "rmat25"])
