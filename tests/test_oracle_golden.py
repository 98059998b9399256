"""The oracle against the reference's own outputs (golden fixtures).

The reference's GPU build, run on the same inputs, agrees with its CPU build
(TM-scores within 1e-4) on 91% of the reported pairs of the full-size small
configuration and on 42-90% of the other sets; the oracle agrees with the CPU
build at the same rates (recorded with the GPU build's outputs in
tests/golden/*_refgpu.json).

The fixtures hold what the reference CPU build printed for seeded synthetic
sets (tests/golden/make_golden.py).  Low-TM pairs have several near-equal
local optima, and the reference's own result for them moves when the query
is merely rotated (`self_agreement` in each fixture).  The bar for the oracle
is therefore: agree with the reference at least as often as the reference
agrees with itself (minus a small sampling margin), agree on nearly every
generated homolog of the query, and agree exactly on everything that follows
from an identical alignment.
"""
import numpy as np
import pytest

import golden_util as gu

MARGIN = 0.12
HOMOLOGS = []


def rmsd_svd(P, Q):
    pc, qc = P.mean(0), Q.mean(0)
    H = (P - pc).T @ (Q - qc)
    U, S, Vt = np.linalg.svd(H)
    d = np.sign(np.linalg.det(Vt.T @ U.T))
    S[2] *= d
    e = ((P - pc) ** 2).sum() + ((Q - qc) ** 2).sum() - 2 * S.sum()
    return float(np.sqrt(max(e, 0.0) / len(P)))


def pairs_of(row_q, row_r, q0, r0):
    out, qi, ri = [], q0, r0
    for a, b in zip(row_q, row_r):
        if a != "-" and b != "-":
            out.append((qi, ri))
        if a != "-":
            qi += 1
        if b != "-":
            ri += 1
    return out


def run_oracle(oracle, name):
    q, r, qn, rn, meta = gu.load(name)
    d = gu.cli_options(meta["options"])
    qx = rx = None
    if not d["nodetailedsearch"]:
        # the reader's index trees (the search's input)
        from gtalign_alpha_b200.api import build_index
        qx, rx = build_index(q), build_index(r)
    o = oracle.process_block(q, r, gu.oracle_opts(oracle, d), qndx=qx, rndx=rx)
    return q, r, qn, rn, meta, d, o


@pytest.mark.parametrize("name", [s for s in gu.SETS if s != "c0_na"])
def test_oracle_matches_reference(oracle, name):
    q, r, qn, rn, meta, d, o = run_oracle(oracle, name)
    ref = meta["results"]
    s = d["scorethld"]
    ours = set()
    for qi in range(q.n):
        for ri in range(r.n):
            out = o.out[qi, ri]
            if max(out[9], out[10]) >= s and out[4] >= 1:
                ours.add(qn[qi] + "|" + rn[ri])
    theirs = set(ref.keys())
    union = ours | theirs
    assert len(ours & theirs) >= (1.0 - MARGIN) * len(union), (len(ours), len(theirs))

    dtm, same, hom_same = [], [], []
    for key in sorted(ours & theirs):
        a, b = key.split("|")
        qi, ri = qn.index(a), rn.index(b)
        out = o.out[qi, ri]
        g = ref[key]
        dd = max(abs(out[9] - g["tmq"]), abs(out[10] - g["tmr"]))
        rows = o.alns[qi][ri]
        ident = rows[0] == g["query_aln"] and rows[2] == g["refrn_aln"]
        dtm.append(dd)
        same.append(ident)
        if b.startswith("hom"):      # a generated homolog of the query
            # the same alignment, and the TM-scores within 1e-4 or higher (a
            # better superposition of that alignment: the reference's FP32
            # rotation solve can stop short of the TM-score optimum)
            lower = max(g["tmq"] - out[9], g["tmr"] - out[10])
            hom_same.append(ident and (dd <= 1e-4 or lower <= 1e-4))
        if ident:
            # everything that follows from the alignment agrees exactly
            assert rows[3] == g["query_secstr"] and rows[4] == g["refrn_secstr"], key
            assert int(out[6]) == g["n_identities"] and int(out[7]) == g["n_gaps"], key
            assert int(out[4]) == g["n_aligned"], key
            bq, be = int(out[2:3].view(np.uint32)[0]), int(out[3:4].view(np.uint32)[0])
            assert (bq & 0xffff, bq >> 16) == (g["query_from"], g["refn_from"]), key
            # with --no-deletions the reference's writer counts displayed residues
            if not d["nodeletions"]:
                assert (be & 0xffff, be >> 16) == (g["query_to"], g["refn_to"]), key
            assert abs(out[11] - g["d0q"]) < 6e-3 and abs(out[12] - g["d0r"]) < 6e-3
    dtm = np.array(dtm)
    sa = meta["self_agreement"]
    # sampling margin: at least MARGIN, or two standard errors of a proportion
    # near 1/2 over the set's pairs
    margin = max(MARGIN, 2.0 * np.sqrt(0.25 / max(len(dtm), 1)))
    assert (dtm <= 1e-4).mean() >= sa["frac_tm_1e4"] - margin, ((dtm <= 1e-4).mean(), sa)
    assert np.mean(same) >= sa["frac_aln_identical"] - margin, (np.mean(same), sa)
    if hom_same:
        assert np.mean(hom_same) >= 0.7, hom_same
    HOMOLOGS.extend(hom_same)


@pytest.mark.parametrize("name", ["c0_speed13", "c0_default"])
def test_oracle_rmsd_is_exact(oracle, name):
    """The reported RMSD is the optimal-superposition RMSD of the reported
    alignment (FP64 SVD recomputation, 1e-3 A)."""
    q, r, qn, rn, meta, d, o = run_oracle(oracle, name)
    qxyz = np.stack([q.x, q.y, q.z], 1).astype(np.float64)
    rxyz = np.stack([r.x, r.y, r.z], 1).astype(np.float64)
    n = 0
    for qi in range(q.n):
        for ri in range(r.n):
            out = o.out[qi, ri]
            if out[4] < 3:
                continue
            rows = o.alns[qi][ri]
            b = int(out[2:3].view(np.uint32)[0])
            pr = pairs_of(rows[0], rows[2], (b & 0xffff) - 1, (b >> 16) - 1)
            P = qxyz[[q.offs[qi] + a for a, _ in pr]]
            Q = rxyz[[r.offs[ri] + c for _, c in pr]]
            assert abs(rmsd_svd(P, Q) - out[8]) < 1e-3
            n += 1
    assert n > 10


def test_oracle_tm_errors_small(oracle):
    """|FP32 path - FP64 recomputation| of reported TM-scores is < 1e-5."""
    q, r, qn, rn, meta, d, o = run_oracle(oracle, "c0_speed13")
    assert o.err[..., :2].max() < 1e-5
    assert o.err[..., 2].max() < 1e-3


def test_oracle_homologs_overall(oracle):
    """Across all fixture sets, the generated homologs of the query get the
    reference's alignment and TM-score (1e-4) in at least 85% of cases."""
    if len(HOMOLOGS) < 40:
        for name in gu.SETS:
            if name != "c0_na":
                test_oracle_matches_reference(oracle, name)
    assert len(HOMOLOGS) >= 40
    assert np.mean(HOMOLOGS) >= 0.85, (np.mean(HOMOLOGS), len(HOMOLOGS))


def test_refinement_levels_pinned(oracle):
    """One homolog-only input, run by the reference at each --refinement code
    (-1 log search, 0 coarse, 1 one search, 2 full, 3 full in both final
    phases).  The oracle at the same code reproduces every pair (TM-scores
    within 1e-4, identical alignment rows), and at any other code it
    reproduces fewer: the five final-stage forms are told apart."""
    n_match = {}
    for lref, name in gu.LEVEL_SETS.items():
        q, r, qn, rn, meta = gu.load(name)
        for lo in gu.LEVEL_SETS:
            o = oracle.process_block(q, r, oracle.opts_from(
                refinement=lo, convergence=18, prescore=0.0, scorethld=0.0))
            c = 0
            for key, g in meta["results"].items():
                a, b = key.split("|")
                qi, ri = qn.index(a), rn.index(b)
                out, rows = o.out[qi, ri], o.alns[qi][ri]
                dd = max(abs(out[9] - g["tmq"]), abs(out[10] - g["tmr"]))
                c += dd <= 1e-4 and rows[0] == g["query_aln"] and rows[2] == g["refrn_aln"]
            n_match[lref, lo] = c
        npairs = len(meta["results"])
        assert n_match[lref, lref] >= 0.95 * npairs, (lref, n_match)
        for lo in gu.LEVEL_SETS:
            if lo != lref:
                assert n_match[lref, lref] > n_match[lref, lo], (lref, lo, n_match)


def test_oracle_2tm_scores(oracle):
    """--2tm-score: the secondary TM-scores (helix aligned to non-helix left
    out, printed to 5 significant digits) agree within 1e-4 wherever the
    reference and the oracle report the same alignment and the same TM-scores
    to the printed precision (the same superposition), on at least 90% of the
    pairs whose TM-scores agree within 1e-4 (some of those end on a different
    transform of nearly the same score, which moves the 2TM-score more)."""
    q, r, qn, rn, meta, d, o = run_oracle(oracle, "c0_2tm")
    same_sup, close = [], []
    for key, g in meta["results"].items():
        a, b = key.split("|")
        qi, ri = qn.index(a), rn.index(b)
        out, rows = o.out[qi, ri], o.alns[qi][ri]
        dd = max(abs(out[9] - g["tmq"]), abs(out[10] - g["tmr"]))
        e2 = max(abs(out[13] - g["tm2q"]), abs(out[14] - g["tm2r"]))
        assert out[13] <= out[9] + 1e-6 and out[14] <= out[10] + 1e-6
        if dd <= 1e-4:
            close.append(e2 <= 1e-4)
            if dd <= 1e-5 and rows[0] == g["query_aln"] and rows[2] == g["refrn_aln"]:
                same_sup.append(e2)
    assert len(same_sup) >= 20 and max(same_sup) <= 1e-4, (len(same_sup), max(same_sup))
    assert np.mean(close) >= 0.9, np.mean(close)


def test_oracle_search_by_ss_pinned(oracle):
    """--add-search-by-ss: with the stage the oracle reproduces the
    reference's run (TM-scores within 1e-4) at least as often as the
    reference reproduces itself, and clearly more often than without it."""
    q, r, qn, rn, meta = gu.load("c0_ssrr")
    agree = {}
    for ss in (0, 1):
        o = oracle.process_block(q, r, oracle.opts_from(
            refinement=1, convergence=18, prescore=0.0, scorethld=0.0, addsearchbyss=ss))
        c = 0
        for key, g in meta["results"].items():
            a, b = key.split("|")
            out = o.out[qn.index(a), rn.index(b)]
            c += max(abs(out[9] - g["tmq"]), abs(out[10] - g["tmr"])) <= 1e-4
        agree[ss] = c / len(meta["results"])
    assert agree[1] >= meta["self_agreement"]["frac_tm_1e4"] - MARGIN, agree
    assert agree[1] >= agree[0] + 0.1, agree


def test_oracle_presimilarity_pinned(oracle):
    """--pre-similarity: the pairs that pass the ungapped sequence-similarity
    screen are exactly the ones the reference reports (it reports every pair
    that proceeds with -s 0 and --pre-score 0); without the screen every pair
    proceeds."""
    q, r, qn, rn, meta = gu.load("c0_presim")
    d = gu.cli_options(meta["options"])
    theirs = set(meta["results"])
    for thr, expect in ((d["presimilarity"], theirs), (0.0, None)):
        o = oracle.process_block(q, r, oracle.opts_from(
            refinement=1, convergence=18, prescore=0.0, scorethld=0.0, presimilarity=thr))
        ours = {qn[qi] + "|" + rn[ri] for qi in range(q.n) for ri in range(r.n)
                if o.out[qi, ri, 4] >= 1}
        if expect is not None:
            assert ours == expect, (sorted(ours ^ expect))
        else:
            assert len(ours) == q.n * r.n > len(theirs)


def test_oracle_nucleic_acids(oracle):
    """Nucleic-acid pairs: the final d0 is the reference's nucleic-acid d0
    on every pair (GetD0finNA), protein-NA pairs are skipped, TM-scores
    agree as often as the reference agrees with itself, and the base-pair
    secondary structure rows agree on most characters.  The oracle takes
    each residue's partner as the truly least-deviating one, as the
    reference's GPU form does (sskna.cu); its CPU build, which made these
    fixtures, picks the partner with a vectorised reduction whose winner is
    not always the least-deviating candidate."""
    q, r, qn, rn, meta, d, o = run_oracle(oracle, "c0_na")
    ref = meta["results"]
    # the reference's reader drops references shorter than --dev-min-length
    # (20, PMBatchStrData.h:439-454) before they reach the path
    ours = {qn[0] + "|" + rn[ri] for ri in range(r.n) if o.out[0, ri, 4] >= 1 and r.lens[ri] >= 20}
    assert ours == set(ref)
    assert all(not rn[ri].startswith("prt") for ri in range(r.n) if o.out[0, ri, 4] >= 1)
    tm, same, tot = [], 0, 0
    for key, g in ref.items():
        ri = rn.index(key.split("|")[1])
        out, rows = o.out[0, ri], o.alns[0][ri]
        assert abs(out[11] - g["d0q"]) < 6e-3 and abs(out[12] - g["d0r"]) < 6e-3, key
        tm.append(max(abs(out[9] - g["tmq"]), abs(out[10] - g["tmr"])) <= 1e-4)
        if rows[0] == g["query_aln"] and rows[2] == g["refrn_aln"]:
            for a, c in zip(rows[3] + rows[4], g["query_secstr"] + g["refrn_secstr"]):
                tot += 1
                same += a == c
    assert np.mean(tm) >= meta["self_agreement"]["frac_tm_1e4"] - MARGIN, np.mean(tm)
    assert tot > 1000 and same / tot >= 0.8, (same, tot)


def _d0fin(L):
    return max(0.5, 1.24 * np.cbrt(L - 15.0) - 1.8) if L > 21 else 0.5


def _tm64(P, Q, R, t, d0, L):
    X = P @ np.asarray(R, np.float64).reshape(3, 3).T + np.asarray(t, np.float64)
    d2 = ((X - Q) ** 2).sum(1)
    return float((d0 * d0 / (d0 * d0 + d2)).sum() / L)


def classify(oracle, name):
    """Every pair the reference reports, against the oracle: 'same' (identical
    alignment and both TM-scores within 1e-4), else the reference's printed
    alignment and transform rescored in FP64 (TM-score by the shorter length,
    the search's objective) against the oracle's TM-score by that length:
    'tie' within 1e-4, 'better' or 'worse' for the oracle.  A pair the oracle
    leaves below -s is run again without the threshold for its TM-score."""
    q, r, qn, rn, meta, d, o = run_oracle(oracle, name)
    ref = meta["results"]
    qxyz = np.stack([q.x, q.y, q.z], 1).astype(np.float64)
    rxyz = np.stack([r.x, r.y, r.z], 1).astype(np.float64)
    cls = {"same": 0, "tie": 0, "better": 0, "worse": 0}
    diffs = []
    rerun = None
    for key, g in ref.items():
        a, b = key.split("|")
        qi, ri = qn.index(a), rn.index(b)
        out = o.out[qi, ri]
        lq, lr = int(q.lens[qi]), int(r.lens[ri])
        rows = o.alns[qi][ri]
        if rows[0] == g["query_aln"] and rows[2] == g["refrn_aln"] and \
                max(abs(out[9] - g["tmq"]), abs(out[10] - g["tmr"])) <= 1e-4:
            cls["same"] += 1
            diffs.append(0.0)
            continue
        pr = pairs_of(g["query_aln"], g["refrn_aln"], g["query_from"] - 1, g["refn_from"] - 1)
        P = qxyz[[q.offs[qi] + x for x, _ in pr]]
        Q = rxyz[[r.offs[ri] + y for _, y in pr]]
        L = min(lq, lr)
        if d["referenced"]:
            reft = _tm64(Q, P, g["rotation"], g["translation"], _d0fin(L), L)
        else:
            reft = _tm64(P, Q, g["rotation"], g["translation"], _d0fin(L), L)
        col = 9 if lq <= lr else 10
        ours = float(out[col])
        if ours == 0.0 and d["scorethld"] > 0:
            if rerun is None:
                d2 = dict(d, scorethld=0.0)
                qx = rx = None
                if not d["nodetailedsearch"]:
                    from gtalign_alpha_b200.api import build_index
                    qx, rx = build_index(q), build_index(r)
                rerun = oracle.process_block(q, r, gu.oracle_opts(oracle, d2), qndx=qx, rndx=rx)
            ours = float(rerun.out[qi, ri, col])
        diff = ours - reft
        diffs.append(diff)
        cls["tie" if abs(diff) <= 1e-4 else ("better" if diff > 0 else "worse")] += 1
    return cls, np.array(diffs)


@pytest.mark.parametrize("name", [s for s in gu.SETS if s != "c0_na"])
def test_oracle_optima_not_worse_than_reference(oracle, name):
    """Where the oracle and the reference part, the oracle's optimum is no
    worse on balance: the reference's own result moves between near-equal
    local optima when the query is only rotated, so a disagreement is a
    different optimum, not an error, as long as the oracle does not lose
    score systematically.  Per set: the mean TM-score difference (oracle -
    reference, FP64 rescored) is at least -5e-3 and the pairs where the
    oracle is worse exceed those where it is better by at most 20% of the
    pairs."""
    cls, diffs = classify(oracle, name)
    n = len(diffs)
    assert n > 0
    assert float(diffs.mean()) >= -5e-3, (cls, float(diffs.mean()))
    assert cls["worse"] - cls["better"] <= 0.2 * n, cls
