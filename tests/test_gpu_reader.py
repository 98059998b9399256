"""Structures read from files go through the search unchanged.

Chains of the benchmark generator are written as PDB files and read back by
the host reader (gtb_read_pdb).  The reader's fields as they are (its
per-residue chain/insertion values, molecule-type vote, offsets) and the
same structures repacked from its SoA must give bit-identical results, and
the TM-scores must match those of the in-memory chains to the rounding of
the files' coordinates (3 decimals).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_reader_fields_feed_the_search(tmp_path):
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options, read_pdb
    wl = synth.config0(seed=12, n_refs=40, qlen=120, lmin=40, lmax=300)
    qp, rp = [], []
    for k, c in enumerate(wl.queries):
        qp.append(str(tmp_path / ("q%d.pdb" % k)))
        synth.write_pdb(c, qp[-1])
    for k, c in enumerate(wl.refs):
        rp.append(str(tmp_path / ("r%03d.pdb" % k)))
        synth.write_pdb(c, rp[-1])
    q, r = read_pdb(qp, minlen=1), read_pdb(rp, minlen=1)
    assert q.soa.n == len(wl.queries) and r.soa.n == len(wl.refs)
    with GTalignB200(0, 0, Options.speed(13)) as g:
        a = g.process_packed(q.packed, r.packed, scorethld=0.0)
        b = g.process_block(q.soa, r.soa, scorethld=0.0)
        c = g.process_block(synth.pack(wl.queries), synth.pack(wl.refs), scorethld=0.0)
    assert np.array_equal(a.alndata.view(np.uint32), b.alndata.view(np.uint32))
    assert np.array_equal(a.tfm.view(np.uint32), b.tfm.view(np.uint32))
    # the files' coordinates differ from the chains' by at most 5e-4 A; the
    # homologs' alignments are stable under that (unrelated pairs may settle
    # in other local optima)
    hi = c.tm_query > 0.5
    assert hi.sum() >= 3
    assert np.abs(a.tm_query[hi] - c.tm_query[hi]).max() < 2e-3
    assert os.path.basename(q.descriptions[0]) == "q0.pdb Chn:A"
