"""Run one phase of the Louvain hot path on a synthetic graph generated on the
device, for timing and profiling (e.g. under ncu):

    python -m louvaingpu_b200.workload --graph rmat25 --phase run
    python -m louvaingpu_b200.workload --graph rmat20 --phase coarsen
    python -m louvaingpu_b200.workload --graph rmat25 --phase passes --repeat 2

Phases:
  load     lvg_load_edges_device: validation and the level-0 CSR build
  passes   load, then the level-0 one-level phase (lvg_one_level)
  coarsen  load, one level, renumber, then one coarsening (lvg_induce) into
           level 1 with its CSR build
  run      a whole dendrogram (lvg_load_edges_device + lvg_run)

Graphs: rmatS (R-MAT scale S, edge factor 16, a,b,c = 0.57,0.19,0.19,
integer weights 1..16, seed 2; self loops dropped, duplicates merged, both
directions present) or lfr (the LFR-style n = 2^20 graph, generated on the
host and copied to the device).  Wall time of the phase (device synchronised
on both sides) is printed per repeat; only the last repeat's phase is
preceded by the setup steps it needs.
"""
import argparse
import os
import sys
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "louvaingpu_b200"

import numpy as np  # noqa: E402

from . import graphgen  # noqa: E402
from .louvain import Louvain  # noqa: E402


def _graph(name):
    import torch
    if name.startswith("rmat"):
        dg = graphgen.rmat_device(int(name[4:]))
        return dg, (dg.src, dg.dst, dg.w, dg.n_entries, dg.n_vertices)
    if name == "lfr":
        n, s, d, w = graphgen.lfr()
        t = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (s, d, w)]
        return t, (t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), len(s), n)
    raise SystemExit(f"unknown graph {name}")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--graph", default="rmat25")
    ap.add_argument("--phase", choices=["load", "passes", "coarsen", "run"], default="run")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--thresholds", default="256,4096", help="tile,block maximum degrees")
    ap.add_argument("--coarsen", type=int, default=0,
                    help="coarsening of sorted symmetric levels: 0 automatic, 1 segment chunks, 2 by transposition, "
                         "3 sort of all keys")
    ap.add_argument("--levels", action="store_true", help="print each level's sizes and phase times after a run")
    a = ap.parse_args(argv)
    import torch
    torch.cuda.set_device(0)
    keep, args = _graph(a.graph)
    tile, block = (int(x) for x in a.thresholds.split(","))
    lv = Louvain(tile_max_degree=tile, block_max_degree=block, coarsen_mode=a.coarsen)

    def sync_time():
        torch.cuda.synchronize()
        return time.perf_counter()

    for r in range(a.repeat):
        if a.phase in ("load", "run"):
            t0 = sync_time()
            lv.load_edges_device(*args)
            if a.phase == "run":
                res = lv.run()
            t1 = sync_time()
            extra = f" levels {res.n_levels} q {res.q_final:.6f}" if a.phase == "run" else ""
        else:
            lv.load_edges_device(*args)
            q0 = lv.modularity()
            if a.phase == "passes":
                t0 = sync_time()
                q, p = lv.one_level(q0)
                t1 = sync_time()
                extra = f" passes {p} q {q:.6f}"
            else:
                lv.one_level(q0)
                _, C = lv.renumber()
                t0 = sync_time()
                lv.induce()
                t1 = sync_time()
                extra = f" communities {C}"
        print(f"{a.graph} {a.phase} repeat {r}: {1e3 * (t1 - t0):.1f} ms{extra}", flush=True)
        if a.levels and a.phase == "run":
            for l in range(res.n_levels):
                x = lv.level_info(l)
                print(f"  level {l}: V {x.n_vertices} E {x.n_entries} C {x.n_comms} build {x.ms_build:.2f} "
                      f"passes {x.ms_passes:.2f} renumber {x.ms_renumber:.2f} induce {x.ms_induce:.2f} ms", flush=True)
    lv.close()
    del keep


if __name__ == "__main__":
    main()
