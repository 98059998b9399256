"""A small, fixed workload for profiling (ncu) and quick timing.

    python -m gtalign_alpha_b200.profile_case --queries 2 --refs 500

Aligns the first `--queries` queries of the seeded benchmark workload (seed 2)
with `--refs` references under the default options (--no-detailed-search,
-s 0.5) in gtb_process_block calls (one warm-up call, one timed call) and
prints the wall time and the stage timings of the timed call.

    python -m gtalign_alpha_b200.profile_case --long 5000,37860

times long-chain pairs (a multi-domain assembly against its per-domain
perturbed partner), one call per pair.
"""
from __future__ import annotations

import argparse

from . import synth
from .api import GTalignB200, Options


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--queries", type=int, default=2)
    ap.add_argument("--refs", type=int, default=500)
    ap.add_argument("--speed13", action="store_true")
    ap.add_argument("--long", default="",
                    help="comma-separated lengths: time the long-chain pairs (assembly vs "
                         "its perturbed partner, one call per pair) instead")
    a = ap.parse_args()
    if a.long:
        long_chains([int(x) for x in a.long.split(",")])
        return
    wl = synth.config1(seed=2, n_queries=max(a.queries, 1), n_refs=a.refs)
    q, r = synth.pack(wl.queries[:a.queries]), synth.pack(wl.refs)
    opts = Options.speed(13) if a.speed13 else Options()
    import time
    with GTalignB200(0, 0, opts) as g:
        res = g.process_block(q, r, scorethld=0.5, alignments=False)
        t0 = time.perf_counter()
        res = g.process_block(q, r, scorethld=0.5, alignments=False)
        wall = time.perf_counter() - t0
    print("pairs", q.n * r.n, "launches", res.launches, "wall ms %.1f" % (1000 * wall),
          "stage ms (summed over concurrent sub-batches)", [round(x, 1) for x in res.timings_ms.tolist()])


def long_chains(lengths):
    """One gtb_process_block call per long-chain pair (gtalign defaults,
    --no-detailed-search, -s 0.5): wall time, TM-scores and stage timings."""
    import time
    import numpy as np
    from .shard import subset
    wl = synth.config2(seed=3, lengths=tuple(lengths))
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    with GTalignB200(0, 0, Options()) as g:
        g.process_block(subset(q, np.array([0])), subset(r, np.array([0])), scorethld=0.5,
                        alignments=False)
        for i in range(q.n):
            qi, ri = subset(q, np.array([i])), subset(r, np.array([i]))
            t0 = time.perf_counter()
            res = g.process_block(qi, ri, scorethld=0.5, alignments=False)
            wall = time.perf_counter() - t0
            print("length", lengths[i], "wall ms %.1f" % (1000 * wall),
                  "tm %.4f %.4f rmsd %.3f aligned %d" % (res.alndata[0, 0, 9], res.alndata[0, 0, 10],
                                                        res.alndata[0, 0, 8], res.alndata[0, 0, 4]),
                  "stage ms", [round(x, 1) for x in res.timings_ms.tolist()], flush=True)


if __name__ == "__main__":
    main()
