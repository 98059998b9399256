"""A clustering run end to end against the reference's GPU build.

The structures of a fixture (rebuilt from its seeded generator) are aligned
all against all the way the reference's clustering run does it: in query
blocks, each query against every structure, with the coverage prefilter
(Options.clsfilter: a pair is compared only when the reference structure was
read as a query by the end of the block and the lengths reach the coverage,
CuBatch.cu:452-495).  The records feed gtb_cluster (the clustering writer's
linkage); its clusters must be the ones the reference's GPU build listed in
its gtalignclusters.lst for the same structures and options
(tests/golden/make_cluster_golden.py).
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

pytestmark = pytest.mark.gpu

# The same mixed-noise set under complete linkage is not pinned: there some
# pairs straddle the threshold by ~0.03 TM-score between the reference's GPU
# build and its CPU build (this library matches the CPU build's scores there,
# e.g. 0.4645 / 0.4701 for clsf01m02 against clsf01m00), and complete linkage
# splits those families differently.
SETS = ["cls_complete", "cls_single", "cls_mixed_single"]


def _clusters_by_library(chains, linkage, threshold, coverage=0.7, qblock=8):
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options, cluster
    n = len(chains)
    allsoa = synth.pack(chains)
    types = np.arange(n, dtype=np.int32)
    rec = np.zeros((n, n, 16), np.float32)
    opts = Options.speed(13, clsfilter=1, clscoverage=coverage)
    with GTalignB200(0, 0, opts) as g:
        for q0 in range(0, n, qblock):
            q1 = min(n, q0 + qblock)
            q = synth.pack(chains[q0:q1])
            res = g.process_block(q, allsoa, scorethld=0.5, alignments=False,
                                  qtypes=types[q0:q1], rtypes=types)
            rec[q0:q1] = res.alndata
    cl = cluster(rec, allsoa.lens, ids=[c.name for c in chains], linkage=linkage,
                 threshold=threshold, coverage=coverage)
    return [[chains[k].name for k in c] for c in cl.clusters]


@pytest.mark.parametrize("name", SETS)
def test_clusters_match_the_reference_gpu_build(name):
    import make_cluster_golden as mcg
    path = os.path.join(HERE, "golden", name + ".json")
    if not os.path.exists(path):
        pytest.skip("fixture %s not generated" % name)
    fx = json.load(open(path))
    p = fx["params"]
    chains = sorted(mcg.structures(p), key=lambda c: c.name)
    ours = _clusters_by_library(chains, p["linkage"], p["threshold"])
    ref = fx["clusters"]
    assert sorted(sorted(c) for c in ours) == sorted(sorted(c) for c in ref)
    # The representative (the member with the smallest linkage distance) is
    # not compared: within a family of near-copies the distances differ in
    # the fourth decimal, where the reference's GPU build and this library
    # may order them differently; the count is reported.
    same_rep = len({c[0] for c in ours} & {c[0] for c in ref})
    print("%s: %d clusters, %d with the same representative" % (name, len(ref), same_rep))
