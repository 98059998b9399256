"""Batching does not change results.

A block large enough to be split into concurrent sub-batches (two waves over
the library's streams), and the same block under a memory budget small enough
to force several batches, must give the records and transforms of the same
pairs aligned in small blocks of one sub-batch each.  Every pair is aligned
independently, so the three ways must agree bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


_WL = None


def _block():
    global _WL
    from gtalign_alpha_b200 import synth
    rng = np.random.default_rng(11)
    wl = synth.config0(seed=5, n_refs=40, qlen=64, lmin=20, lmax=90)
    _WL = wl
    refs = synth.random_chains(rng, list(rng.integers(20, 90, 100_000 - 40)), "r") + wl.refs
    return synth.pack(wl.queries), synth.pack(refs)


def test_sub_batches_and_budget_batches_match_small_blocks():
    from gtalign_alpha_b200.api import GTalignB200, Options
    from gtalign_alpha_b200.shard import subset
    q, r = _block()
    opts = Options(prescore=0.3, convergence=4)
    with GTalignB200(0, 0, opts) as g:
        whole = g.process_block(q, r, scorethld=0.3, alignments=False)
        parts = []
        for c in range(0, r.n, 10_000):
            sub = subset(r, np.arange(c, min(r.n, c + 10_000)))
            parts.append(g.process_block(q, sub, scorethld=0.3, alignments=False))
    small = np.concatenate([p.alndata for p in parts], axis=1)
    small_tfm = np.concatenate([p.tfm for p in parts], axis=1)
    assert np.array_equal(whole.alndata.view(np.uint32), small.view(np.uint32))
    assert np.array_equal(whole.tfm.view(np.uint32), small_tfm.view(np.uint32))
    # a 256 MiB budget forces several budget batches
    with GTalignB200(0, 256 << 20, opts) as g:
        tight = g.process_block(q, r, scorethld=0.3, alignments=False)
    assert np.array_equal(whole.alndata.view(np.uint32), tight.alndata.view(np.uint32))
    assert np.array_equal(whole.tfm.view(np.uint32), tight.tfm.view(np.uint32))
    # the generated homologs of the query are found
    names = [c.name for c in _WL.refs]
    hom = np.array([n.startswith("hom") for n in names])
    tm = whole.alndata[0, -40:, 9]
    assert hom.sum() > 0 and (tm[hom] > 0.5).mean() > 0.5


def test_sharded_search_with_the_gpu_library():
    """shard.search_sharded with the CUDA library as the per-rank process
    (world = 1: the plan, the shard and the result placement; ranks > 1 are
    the gloo test's): records and transforms equal an unsharded call, and a
    reusable ShardPlan gives the same."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options
    from gtalign_alpha_b200.shard import ShardPlan, search_sharded
    wl = synth.config0(seed=51, n_refs=40, qlen=120)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    with GTalignB200(0, 0, Options(prescore=0.3)) as g:
        ref = g.process_block(q, r, scorethld=0.3, alignments=False)

        def fn(qs, rs):
            res = g.process_block(qs, rs, scorethld=0.3, alignments=False)
            return res.alndata, res.tfm
        aln, tfm = search_sharded(q, r, fn, 0, 1)
        plan = ShardPlan(r, q.lens, 0, 1)
        aln2, tfm2 = search_sharded(q, r, fn, 0, 1, plan=plan)
    for a, t in ((aln, tfm), (aln2, tfm2)):
        assert np.array_equal(a.view(np.uint32), ref.alndata.view(np.uint32))
        assert np.array_equal(t.view(np.uint32), ref.tfm.view(np.uint32))


def test_kernel_timing_and_work_counters():
    """Per-family device times (gtb_set_kernel_timing / gtb_last_kernel_ms)
    and the device-counted work of a call: every family that ran has time
    and work, timing off leaves the times at 0, and the results do not
    depend on the timing."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options
    wl = synth.config0(seed=41, n_refs=60, qlen=120)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    with GTalignB200(0, 0, Options.speed(9)) as g:
        a = g.process_block(q, r, scorethld=0.0)
        assert (g.last_kernel_ms() == 0).all()
        w = g.last_work()
        assert (w > 0).all(), w
        g.set_kernel_timing(True)
        b = g.process_block(q, r, scorethld=0.0)
        ms = g.last_kernel_ms()
        assert (ms > 0).all(), ms
        assert np.array_equal(g.last_work(), w)
        g.set_kernel_timing(False)
    assert np.array_equal(a.alndata.view(np.uint32), b.alndata.view(np.uint32))
    with GTalignB200(0, 0, Options.speed(13)) as g:
        g.set_kernel_timing(True)
        g.process_block(q, r, scorethld=0.0)
        ms, w = g.last_kernel_ms(), g.last_work()
        assert (ms[:3] > 0).all() and ms[3] == 0 and w[3] == 0
