"""A small, fixed workload for profiling (ncu) and quick timing.

    python -m gtalign_alpha_b200.profile_case --queries 2 --refs 500

Aligns the first `--queries` queries of the seeded benchmark workload (seed 2)
with `--refs` references under the default options (--no-detailed-search,
-s 0.5) in gtb_process_block calls (one warm-up call, one timed call) and
prints the wall time and the stage timings of the timed call.
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
    a = ap.parse_args()
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


if __name__ == "__main__":
    main()
