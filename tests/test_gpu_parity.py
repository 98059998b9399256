"""CUDA path against the oracle, through the C ABI (bit for bit).

Every per-pair record (scores, RMSD, counts, coordinates), every transform
and every alignment row of the library must equal the oracle's exactly:
both follow the same arithmetic (explicit FMAs, IEEE division/sqrt,
block-compensated sums in position order, FP64 quaternion solve).
"""
import numpy as np
import pytest

import golden_util as gu

pytestmark = pytest.mark.gpu


def _lib_opts(d):
    from gtalign_alpha_b200.api import Options
    return Options(refinement=d["refinement"], depth=d.get("depth", 2), convergence=d["convergence"],
                   prescore=d["prescore"], symmetric=d["symmetric"], referenced=d["referenced"],
                   nodeletions=d["nodeletions"], twotmscore=d.get("twotmscore", 0),
                   addsearchbyss=d.get("addsearchbyss", 0), presimilarity=d.get("presimilarity", 0.0),
                   nodetailedsearch=d.get("nodetailedsearch", 1), trigger=d.get("trigger", 50),
                   nbranches=d.get("nbranches", 5), gapcost=d.get("gapcost", 1),
                   seedrule=d.get("seedrule", 1), window=d.get("window", 256))


def _ora_opts(oracle, d, cls=None):
    return gu.oracle_opts(oracle, dict(d, depth=d.get("depth", 2), twotmscore=d.get("twotmscore", 0),
                                       addsearchbyss=d.get("addsearchbyss", 0),
                                       presimilarity=d.get("presimilarity", 0.0)), cls=cls)


def assert_same(res, ora, nq, nr):
    a = res.alndata.view(np.uint32)
    b = ora.out.view(np.uint32)
    bad = np.argwhere((a != b).any(axis=2))
    assert len(bad) == 0, ("records differ", bad[:5], res.alndata[tuple(bad[0])], ora.out[tuple(bad[0])])
    assert np.array_equal(res.tfm.view(np.uint32), ora.tfm.view(np.uint32))
    assert np.array_equal(res.numerr.view(np.uint32), ora.err.view(np.uint32))
    for qi in range(nq):
        for ri in range(nr):
            assert res.alignment(qi, ri) == ora.alns[qi][ri], (qi, ri)


def run_both(oracle, q, r, d, secstr=False):
    """The library (gtb_process_block, which builds the index trees itself when
    the detailed search is on) and the oracle (given the same trees)."""
    from gtalign_alpha_b200.api import GTalignB200, build_index
    with GTalignB200(0, 0, _lib_opts(d)) as g:
        res = g.process_block(q, r, scorethld=d["scorethld"], secstr=secstr)
    qx = rx = None
    if not d.get("nodetailedsearch", 1):
        qx, rx = build_index(q), build_index(r)
    ora = oracle.process_block(q, r, _ora_opts(oracle, d), qndx=qx, rndx=rx)
    return res, ora


@pytest.mark.parametrize("name", gu.LIBRARY_SETS)
def test_golden_sets_bit_identical(oracle, name):
    q, r, qn, rn, meta = gu.load(name)
    d = gu.cli_options(meta["options"])
    res, ora = run_both(oracle, q, r, d, secstr=True)
    assert_same(res, ora, q.n, r.n)
    assert res.qss.tobytes() == ora.qss.tobytes()
    assert res.rss.tobytes() == ora.rss.tobytes()
    assert res.launches > 20


@pytest.mark.parametrize("name", gu.FULL_SETS)
def test_small_configuration_full_size(oracle, name):
    """The small configuration at its full size: one 150-residue query
    against 1,000 targets (lengths U(50,500), 20% homologs), default options
    without the detailed search (--pre-score 0.4, -s 0.5) and --speed=13:
    records, transforms, numeric errors and alignment rows bit for bit."""
    q, r, qn, rn, meta = gu.load(name)
    d = gu.cli_options(meta["options"])
    res, ora = run_both(oracle, q, r, d)
    assert_same(res, ora, q.n, r.n)
    assert (res.alndata[0, :, 9] > 0).sum() > 150         # the reported pairs
    assert float(res.numerr[..., :2].max()) <= 1e-4 and float(res.numerr[..., 2].max()) <= 1e-3


def test_benchmark_workload_sample(oracle):
    """A seeded sample of the benchmark workload (2 queries of the 16 x 3,000
    references of its generator: log-normal lengths up to 2,000, homolog
    families), with the benchmark's options (defaults without the detailed
    search, -s 0.5), GPU against the oracle bit for bit."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.shard import subset
    wl = synth.config1(seed=2, n_queries=16, n_refs=3000)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    q = subset(q, np.array([0, 1]))
    d = dict(refinement=1, convergence=18, prescore=0.4, scorethld=0.5, symmetric=0, referenced=0,
             nodeletions=0)
    res, ora = run_both(oracle, q, r, d)
    assert_same(res, ora, q.n, r.n)
    assert (res.alndata[..., 9] > 0).sum() > 20


OPTSETS = {
    "speed13": dict(refinement=0, convergence=2, prescore=0.0, scorethld=0.0, symmetric=0, referenced=0, nodeletions=0),
    "default": dict(refinement=1, convergence=18, prescore=0.0, scorethld=0.0, symmetric=0, referenced=0, nodeletions=0),
    "filters": dict(refinement=1, convergence=18, prescore=0.4, scorethld=0.5, symmetric=0, referenced=0, nodeletions=0),
    "shallow": dict(refinement=1, convergence=6, prescore=0.3, scorethld=0.3, symmetric=0, referenced=0, nodeletions=0, depth=3),
    "sym": dict(refinement=1, convergence=4, prescore=0.0, scorethld=0.0, symmetric=1, referenced=1, nodeletions=1),
    # the other final-stage forms: log search, full search, full search in both phases
    "log": dict(refinement=-1, convergence=6, prescore=0.2, scorethld=0.2, symmetric=0, referenced=0, nodeletions=0),
    "full": dict(refinement=2, convergence=6, prescore=0.0, scorethld=0.0, symmetric=1, referenced=0, nodeletions=0),
    "fulla": dict(refinement=3, convergence=4, prescore=0.0, scorethld=0.0, symmetric=0, referenced=1, nodeletions=0),
    "twotm": dict(refinement=1, convergence=6, prescore=0.3, scorethld=0.3, symmetric=1, referenced=1, nodeletions=0,
                  twotmscore=1),
    "ssrr": dict(refinement=1, convergence=6, prescore=0.3, scorethld=0.3, symmetric=0, referenced=0, nodeletions=0,
                 addsearchbyss=1),
    "presim": dict(refinement=1, convergence=6, prescore=0.0, scorethld=0.0, symmetric=0, referenced=0, nodeletions=0,
                   presimilarity=12.0),
    # the spatial-index detailed search: defaults (--speed 9), --speed 12, and
    # the fragment seeds with other options
    "frg3": dict(refinement=1, convergence=6, prescore=0.2, scorethld=0.2, symmetric=0, referenced=0, nodeletions=0,
                 nodetailedsearch=0),
    "frg3s12": dict(refinement=0, convergence=2, prescore=0.0, scorethld=0.0, symmetric=0, referenced=0, nodeletions=0,
                    nodetailedsearch=0, depth=3),
    "frg3opts": dict(refinement=1, convergence=4, prescore=0.0, scorethld=0.0, symmetric=1, referenced=0, nodeletions=0,
                     nodetailedsearch=0, trigger=0, seedrule=0, nbranches=3, gapcost=2, window=512),
    "frg3seed2": dict(refinement=1, convergence=4, prescore=0.0, scorethld=0.0, symmetric=0, referenced=0, nodeletions=0,
                      nodetailedsearch=0, trigger=20, seedrule=2, nbranches=8, gapcost=0),
    # --depth 1 and 0: the secondary configuration sections and the extra DP
    # of every branch (--speed 5, and --speed 0 with its 16 branches and
    # --add-search-by-ss)
    "frg3d1": dict(refinement=1, convergence=4, prescore=0.2, scorethld=0.2, symmetric=0, referenced=0, nodeletions=0,
                   nodetailedsearch=0, depth=1, trigger=20),
    "frg3d0": dict(refinement=1, convergence=4, prescore=0.0, scorethld=0.0, symmetric=0, referenced=0, nodeletions=0,
                   nodetailedsearch=0, depth=0, trigger=0, nbranches=16, addsearchbyss=1),
}


@pytest.mark.parametrize("opt", list(OPTSETS))
def test_multi_query_ragged_lengths(oracle, opt):
    """3 queries, references from 3 to 700 residues (including structures too
    short for any fragment), both homologs and unrelated chains."""
    from gtalign_alpha_b200 import synth
    rng = np.random.default_rng(7)
    wl = synth.config0(seed=31, n_refs=18, qlen=140, lmin=3, lmax=700)
    wl.queries += synth.random_chains(rng, [60, 25], "qx")
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    res, ora = run_both(oracle, q, r, OPTSETS[opt])
    assert_same(res, ora, q.n, r.n)


@pytest.mark.parametrize("opt", ["speed13", "presim", "frg3"])
def test_clustering_prefilter(oracle, opt):
    """A clustering run in two query blocks over 12 structures: each block
    compares a reference only when its global index precedes the end of the
    block's and the shorter length reaches 0.6 of the longer
    (CheckMaxCoverage), and the --pre-similarity screen sees only the pairs
    left filtered (and may release them: similarity.cu:56-65); records,
    transforms and rows bit for bit."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, build_index
    rng = np.random.default_rng(11)
    base = synth.random_chains(rng, [60, 80, 95, 120, 150, 40])
    chains = base + [synth.homolog(rng, base[k], 0.9, 0.05, "h%d" % k) for k in range(6)]
    d = dict(OPTSETS[opt])
    lo = _lib_opts(d)
    lo.clsfilter, lo.clscoverage = 1, 0.6
    r = synth.pack(chains)
    rx = build_index(r) if not d.get("nodetailedsearch", 1) else None
    released = 0
    for b in range(2):
        q = synth.pack(chains[6 * b:6 * b + 6])
        qt = np.arange(6 * b, 6 * b + 6, dtype=np.int32)
        rt = np.where(np.arange(12) < 6 * b + 6, np.arange(12), 2**31 - 1).astype(np.int32)
        with GTalignB200(0, 0, lo) as g:
            res = g.process_block(q, r, scorethld=d["scorethld"], qtypes=qt, rtypes=rt)
        qx = build_index(q) if rx is not None else None
        ora = oracle.process_block(q, r, _ora_opts(oracle, d, cls=(rt, 6 * b + 6, 0.6)),
                                   qndx=qx, rndx=rx)
        assert_same(res, ora, q.n, r.n)
        released += int((res.alndata[..., 9] > 0).sum())
        if opt != "presim":      # the screen also releases pairs the prefilter left
            assert (res.alndata[:, 6 * b + 6:, 9] == 0).all()
    assert released > 12


def test_molecule_type_mismatch_is_skipped(oracle):
    """A protein query and a nucleic-acid reference are not compared
    (MpStage1.cpp:143-152): the record keeps its initial values."""
    from gtalign_alpha_b200 import synth
    wl = synth.config0(seed=32, n_refs=4, qlen=80)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    r.mol[1] = 1
    res, ora = run_both(oracle, q, r, OPTSETS["speed13"])
    assert_same(res, ora, q.n, r.n)
    assert res.alndata[0, 1, 9] == 0.0 and res.alndata[0, 1, 8] == np.float32(9999.9)


def test_single_pair_and_long_chain(oracle):
    from gtalign_alpha_b200 import synth
    rng = np.random.default_rng(9)
    a = synth.random_chains(rng, [1500], "long")[0]
    b = synth.homolog(rng, a, 1.5, 0.05, "longhom")
    q, r = synth.pack([a]), synth.pack([b])
    res, ora = run_both(oracle, q, r, OPTSETS["speed13"])
    assert_same(res, ora, 1, 1)
    assert res.alndata[0, 0, 9] > 0.5


def test_resident_blocks_match_process_block(oracle):
    import ctypes
    import torch
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options, pack_fields
    wl = synth.config0(seed=33, n_refs=10, qlen=100)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    with GTalignB200(0, 0, Options(prescore=0.0)) as g:
        ref = g.process_block(q, r, scorethld=0.0, alignments=False)
        L = g.lib
        L.gtb_block_upload.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_void_p)]
        L.gtb_block_free.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.gtb_process_resident.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]
        qb, rb = pack_fields(q), pack_fields(r)
        hq, hr = ctypes.c_void_p(), ctypes.c_void_p()
        assert L.gtb_block_upload(g.handle, qb.beg, qb.end, ctypes.byref(hq)) == 0
        assert L.gtb_block_upload(g.handle, rb.beg, rb.end, ctypes.byref(hr)) == 0
        d_out = torch.zeros(q.n * r.n * 16, dtype=torch.float32, device="cuda")
        d_tfm = torch.zeros(q.n * r.n * 12, dtype=torch.float32, device="cuda")
        for _ in range(2):
            st = L.gtb_process_resident(g.handle, ctypes.c_float(0.0), hq, hr,
                                        ctypes.c_void_p(d_out.data_ptr()),
                                        ctypes.c_void_p(d_tfm.data_ptr()), None)
            assert st == 0
            torch.cuda.synchronize()
            assert np.array_equal(d_out.cpu().numpy().view(np.uint32),
                                  ref.alndata.ravel().view(np.uint32))
            assert np.array_equal(d_tfm.cpu().numpy().view(np.uint32), ref.tfm.ravel().view(np.uint32))
        L.gtb_block_free(g.handle, hq)
        L.gtb_block_free(g.handle, hr)


def test_status_codes():
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, GTBError, Options
    wl = synth.config0(seed=34, n_refs=2, qlen=50)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    for bad in (dict(trigger=101), dict(nbranches=0), dict(window=100), dict(gapcost=3),
                dict(clsfilter=1, clscoverage=0.0), dict(clsfilter=1, clscoverage=1.5)):
        with GTalignB200(0, 0, Options(nodetailedsearch=0, **bad)) as g:
            with pytest.raises(GTBError) as e:
                g.process_block(q, r)
            assert e.value.status == 1, bad
    with GTalignB200(0, 0, Options(refinement=4)) as g:
        with pytest.raises(GTBError) as e:
            g.process_block(q, r)
        assert e.value.status == 1
    # a pair of two nucleic-acid structures is refused (the library has no
    # nucleic-acid secondary structure or final d0); a protein query against
    # a nucleic-acid reference is accepted and the pair skipped
    qn, rn = synth.pack(wl.queries), synth.pack(wl.refs)
    qn.mol[0] = 1
    rn.mol[1] = 1
    with GTalignB200(0, 0, Options()) as g:
        with pytest.raises(GTBError) as e:
            g.process_block(qn, rn)
        assert e.value.status == 4
        qn.mol[0] = 0
        g.process_block(qn, rn)
    with GTalignB200(0, 0, Options()) as g:
        with pytest.raises(GTBError) as e:
            g.process_block(q, r, scorethld=1.5)
        assert e.value.status == 1
        big = synth.SoA(np.array([70000], np.int32), np.array([0], np.int32),
                        np.zeros(70000, np.float32), np.zeros(70000, np.float32),
                        np.zeros(70000, np.float32), np.full(70000, 65, np.uint8),
                        np.zeros(1, np.int32))
        with pytest.raises(GTBError) as e:
            g.process_block(big, r)
        assert e.value.status == 5
        # the handle stays usable after errors
        res = g.process_block(q, r, scorethld=0.0)
        assert res.alndata.shape == (1, 2, 16)


@pytest.mark.parametrize("refinement,addss", [(1, 0), (-1, 0), (3, 0), (1, 1)])
def test_long_chain_assemblies(oracle, refinement, addss):
    """Multi-domain assemblies and their per-domain-perturbed partners (the
    long-chain configuration's construction at 1,200 and 2,000 residues):
    large DP matrices, many strips and thousands of refinement variants; the
    2,000-residue pair takes the many-CTA refinement path in every final
    form (one search, log search, full search in both phases); with
    --add-search-by-ss its DP runs there as a wavefront too."""
    from gtalign_alpha_b200 import synth
    wl = synth.config2(seed=3, lengths=(1200, 2000))
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    d = dict(refinement=refinement, convergence=18 if refinement == 1 else 4, prescore=0.4,
             scorethld=0.5, symmetric=0, referenced=0, nodeletions=0, addsearchbyss=addss)
    res, ora = run_both(oracle, q, r, d)
    assert_same(res, ora, q.n, r.n)
    assert res.alndata[0, 0, 9] > 0.5 and res.alndata[1, 1, 9] > 0.5


def test_longest_chain_pair_properties():
    """The longest pair of the long-chain configuration (37,860 residues,
    an assembly against its per-domain perturbed partner), at full size,
    checked through size-independent properties: the partner is found
    (TM > 0.5 by both lengths), the reported TM-scores and RMSD agree with
    their FP64 recomputation within the 1e-4 / 1e-3 tolerances, and the
    alignment rows agree with the record and pair most residues."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options
    wl = synth.config2(seed=3, lengths=(37860,))
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    with GTalignB200(0, 0, Options()) as g:
        res = g.process_block(q, r, scorethld=0.5, alignments=True)
    rec = res.alndata[0, 0]
    assert rec[9] > 0.5 and rec[10] > 0.5
    assert float(np.max(res.numerr[0, 0, :2])) <= 1e-4
    assert float(res.numerr[0, 0, 2]) <= 1e-3
    rows = res.alignment(0, 0)
    qrow, trow = rows[0], rows[2]
    assert len(qrow) == len(trow) == int(rec[4])
    assert sum(c != '-' for c in qrow) <= 37860 and sum(c != '-' for c in trow) <= 37860
    matched = sum(a != '-' and b != '-' for a, b in zip(qrow, trow))
    assert matched > 0.8 * 37860
