"""The bounded waits of the multi-CTA DP end in a status code, not a hang.

A long pair's DP runs as a wavefront over several CTAs, each strip waiting
(with a bounded spin) until the previous strip has published the values it
reads.  With the wait limit set to 0 spins, a wait that does not find its
values at once gives up: the kernel sets an error flag and returns, the call
ends with GTB_ERR_CUDA and a message, and the same handle then aligns
blocks correctly again.  No kernel traps or faults on this path; the waits
all end (the flag makes every other waiting CTA return too).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wavefront_wait_that_gives_up_is_a_status_code(oracle):
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, GTBError, Options
    # 2,000-residue assembly pair: 16 strips of 128 rows, a wavefront pair
    wl = synth.config2(seed=3, lengths=(2000,))
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    # the library's rule: at least 12 strips of 32*4 query rows and 512 reference residues
    assert (int(q.lens[0]) + 127) // 128 >= 12 and int(r.lens[0]) >= 512
    small = synth.config0(seed=11, n_refs=6, qlen=90, lmin=40, lmax=160)
    sq, sr = synth.pack(small.queries), synth.pack(small.refs)
    opts = Options.speed(13, prescore=0.0)
    with GTalignB200(0, 0, opts) as g:
        g.set_wait_limit(0)
        with pytest.raises(GTBError) as e:
            g.process_block(q, r, scorethld=0.0, alignments=False)
        assert e.value.status == 2
        assert "wait exceeded" in str(e.value)
        # the handle stays usable: a normal block, then the long pair with the
        # default limit, both equal to the oracle
        g.set_wait_limit(1 << 24)
        res = g.process_block(sq, sr, scorethld=0.0)
        ora = oracle.process_block(sq, sr, oracle.opts_from(refinement=0, convergence=2))
        assert np.array_equal(res.alndata.view(np.uint32), ora.out.view(np.uint32))
        res = g.process_block(q, r, scorethld=0.0, alignments=False)
        ora = oracle.process_block(q, r, oracle.opts_from(refinement=0, convergence=2))
        assert np.array_equal(res.alndata.view(np.uint32), ora.out.view(np.uint32))
        assert res.alndata[0, 0, 9] > 0.5
