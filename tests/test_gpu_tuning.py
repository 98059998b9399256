"""Launch shapes change no result, and the autotuner picks among them.

gtb_tuning spreads the same work differently: seed offsets per CTA of a split
pair, CTAs per long refinement pair, DP pairs run as a CTA wavefront, pairs
per concurrent sub-batch.  Every pair is still aligned by the same arithmetic
in the same order, so the records, transforms, numeric errors and alignment
rows must agree bit for bit under every tuning.  The block has long pairs
(1,600-2,300 residues) so that every path the tuning touches is taken: split
seeds, the long-pair refinement tier, the CTA-wavefront DP, and two
sub-batches at the smallest sub_pairs.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TUNINGS = [
    dict(seed_chunk=128, refine_long_ctas=1, dp_cta_pairs=0, sub_pairs=1024),
    dict(seed_chunk=2048, refine_long_ctas=7, dp_cta_pairs=4096, sub_pairs=1024),
    dict(seed_chunk=300, refine_long_ctas=16, dp_cta_pairs=37, sub_pairs=1 << 20),
]


def _block(seed, nshort):
    from gtalign_alpha_b200 import synth
    rng = np.random.default_rng(seed)
    tmpl = synth.random_chains(rng, [1800], "t")[0]
    qs = synth.random_chains(rng, [260], "q") + [synth.homolog(rng, tmpl, 1.0, 0.03, "q1")]
    refs = synth.random_chains(rng, list(rng.integers(50, 400, nshort)), "r")
    refs += [synth.homolog(rng, tmpl, s, 0.05, "h%d" % k) for k, s in enumerate((0.5, 1.5, 2.5))]
    refs += synth.random_chains(rng, [1600, 2300], "l")
    order = rng.permutation(len(refs))
    refs = [refs[k] for k in order]
    return synth.pack(qs), synth.pack(refs)


def _same(a, b):
    assert np.array_equal(a.alndata.view(np.uint32), b.alndata.view(np.uint32))
    assert np.array_equal(a.tfm.view(np.uint32), b.tfm.view(np.uint32))
    assert np.array_equal(a.numerr.view(np.uint32), b.numerr.view(np.uint32))
    assert np.array_equal(a.alns_raw, b.alns_raw)


@pytest.mark.parametrize("speed,nshort", [(13, 1100), (9, 200)])
def test_results_do_not_depend_on_the_tuning(speed, nshort):
    from gtalign_alpha_b200.api import GTalignB200, Options
    q, r = _block(21 + speed, nshort)
    with GTalignB200(0, 0, Options.speed(speed)) as g:
        t0 = g.get_tuning().as_dict()
        assert t0 == dict(seed_chunk=512, refine_long_ctas=16, dp_cta_pairs=592, sub_pairs=16384)
        ref = g.process_block(q, r, scorethld=0.0)
        for t in TUNINGS:
            g.set_tuning(**t)
            assert g.get_tuning().as_dict() == t
            _same(g.process_block(q, r, scorethld=0.0), ref)
    # the template's three homologs are found by its noisy copy (query 1)
    assert (ref.tm_query[1] > 0.5).sum() >= 3


def test_set_tuning_refuses_out_of_range_fields():
    from gtalign_alpha_b200.api import GTalignB200, GTBError, Options
    with GTalignB200(0, 0, Options.speed(13)) as g:
        before = g.get_tuning().as_dict()
        for bad in (dict(seed_chunk=64), dict(refine_long_ctas=0), dict(refine_long_ctas=17),
                    dict(dp_cta_pairs=-1), dict(sub_pairs=100)):
            with pytest.raises(GTBError):
                g.set_tuning(**bad)
            assert g.get_tuning().as_dict() == before


def test_autotune_leaves_its_pick_set_and_changes_no_result():
    from gtalign_alpha_b200.api import GTalignB200, Options, pack_fields
    q, r = _block(40, 1100)
    with GTalignB200(0, 0, Options.speed(13)) as g:
        ref = g.process_block(q, r, scorethld=0.0)
        with g.upload(pack_fields(q)) as hq, g.upload(pack_fields(r)) as hr:
            best, ms, log = g.autotune(hq, hr, scorethld=0.0, trials=1)
        assert g.get_tuning().as_dict() == best.as_dict()
        # the start, then every other candidate of the four fields
        assert len(log) == 1 + 3 + 2 + 3 + 2
        assert log[0][0] == dict(seed_chunk=512, refine_long_ctas=16, dp_cta_pairs=592,
                                 sub_pairs=16384)
        assert ms > 0 and ms == min(m for t, m in log if t == best.as_dict())
        print("autotune:", best.as_dict(), "%.2f ms" % ms)
        _same(g.process_block(q, r, scorethld=0.0), ref)
