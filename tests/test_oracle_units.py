"""Building blocks of the oracle: the FP64 rotation solve, secondary
structure, constants."""
import os

import numpy as np


def kabsch_svd(P, Q):
    pc, qc = P.mean(0), Q.mean(0)
    H = (P - pc).T @ (Q - qc)
    U, S, Vt = np.linalg.svd(H)
    d = np.sign(np.linalg.det(Vt.T @ U.T))
    R = Vt.T @ np.diag([1, 1, d]) @ U.T
    return R, qc - R @ pc


def sums(P, Q):
    s = np.zeros(15)
    for i in range(3):
        for j in range(3):
            s[3 * i + j] = (P[:, i].astype(np.float64) * Q[:, j]).sum()
    s[9:12] = P.sum(0)
    s[12:15] = Q.sum(0)
    return s.astype(np.float32)


def test_solve_matches_svd_kabsch(oracle):
    rng = np.random.default_rng(0)
    for _ in range(100):
        n = int(rng.integers(8, 300))
        P = (rng.normal(size=(n, 3)) * 10).astype(np.float32)
        A = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        if np.linalg.det(A) < 0:
            A[:, 0] *= -1
        Q = (P @ A.T + rng.normal(size=(n, 3)) * rng.uniform(0.1, 2.0)).astype(np.float32)
        t = oracle.solve(sums(P, Q), n)
        R, tt = kabsch_svd(P.astype(np.float64), Q.astype(np.float64))
        assert np.abs(t[:9].reshape(3, 3) - R).max() < 2e-6
        assert np.abs(t[9:] - tt).max() < 1e-4


def test_solve_is_proper_rotation_for_reflections(oracle):
    """A mirrored point set still gets a proper rotation (det = +1)."""
    rng = np.random.default_rng(1)
    P = (rng.normal(size=(50, 3)) * 5).astype(np.float32)
    Q = P.copy()
    Q[:, 0] *= -1
    t = oracle.solve(sums(P, Q), 50)
    R = t[:9].reshape(3, 3).astype(np.float64)
    assert abs(np.linalg.det(R) - 1.0) < 1e-5
    assert np.abs(R @ R.T - np.eye(3)).max() < 1e-5


def test_solve_degenerate_gives_identity(oracle):
    P = np.zeros((1, 3), np.float32) + 3
    Q = np.zeros((1, 3), np.float32) + 5
    t = oracle.solve(sums(P, Q), 1)
    assert np.allclose(t[:9], np.eye(3).ravel())
    assert np.allclose(t[9:], [2, 2, 2])


def test_secstr_helix_and_strand(oracle):
    from gtalign_alpha_b200 import synth
    th = np.full((1, 40), np.deg2rad(91.0)); to = np.full((1, 40), np.deg2rad(50.0))
    X = synth._nerf_flat(th.ravel(), to.ravel(), np.array([40]))
    ss = oracle.secstr(X[:, 0], X[:, 1], X[:, 2]).decode()
    assert ss[:2] == "  " and ss[-2:] == "  "
    assert set(ss[2:-2]) == {"h"}
    th[:] = np.deg2rad(120.0); to[:] = np.deg2rad(-170.0)
    X = synth._nerf_flat(th.ravel(), to.ravel(), np.array([40]))
    ss = oracle.secstr(X[:, 0], X[:, 1], X[:, 2]).decode()
    assert set(ss[2:-2]) == {"e"}
    assert oracle.secstr(X[:4, 0], X[:4, 1], X[:4, 2]).decode() == "    "


def test_constants_follow_reference_formulas(oracle):
    import ctypes
    L = oracle.lib()
    v = [ctypes.c_float() for _ in range(5)]
    L.gto_constants(150, 300, *[ctypes.byref(x) for x in v])
    d0 = 1.24 * np.cbrt(150 - 15) - 1.8 + 0.8
    assert abs(v[0].value - d0) < 1e-5
    assert abs(v[2].value - (1.5 * 150 ** 0.3 + 3.5) ** 2) < 1e-3
    assert abs(v[3].value - (1.24 * np.cbrt(135) - 1.8)) < 1e-5
    L.gto_constants(10, 300, *[ctypes.byref(x) for x in v])
    assert abs(v[0].value - (0.168 + 0.8)) < 1e-6 and abs(v[3].value - 0.5) < 1e-7


def test_gonnet_scores_table():
    """gtb_gonnet.h: log2 of the Gonnet (1992) frequency ratios, 10^(G/10)
    rounded to 6 decimals: symmetric, the published diagonal (A 2.4, W 14.2,
    C 11.5), 0 for letters outside the 20 amino acids, 26 x 26 over A..Z."""
    import ctypes
    import math
    import subprocess
    import tempfile
    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    d = tempfile.mkdtemp()
    src = os.path.join(d, "g.c")
    with open(src, "w") as f:
        f.write('#include "gtb_gonnet.h"\nvoid dump(float* o) { gtb_gonnet_scores(o); }\n')
    so = os.path.join(d, "g.so")
    subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-I",
                           os.path.join(root, "gtalign_alpha_b200", "csrc"), "-o", so, src, "-lm"])
    out = np.zeros(26 * 26, np.float32)
    ctypes.CDLL(so).dump(out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    s = out.reshape(26, 26)
    assert np.array_equal(s, s.T)
    ix = lambda c: ord(c) - 65
    for c, g in (("A", 24), ("W", 142), ("C", 115), ("G", 66)):
        ratio = np.float32(round(10 ** (g / 100.0) * 1e6) / 1e6)
        assert abs(float(s[ix(c), ix(c)]) - math.log2(float(ratio))) < 1e-6
    for c in "BJOUXZ":
        assert (s[ix(c)] == 0).all()
    assert s[ix("W"), ix("W")] == s.max() and s[ix("W"), ix("D")] < 0


def test_clustering_prefilter(oracle):
    """A clustering run's prefilter (CheckMaxCoverage, coverage.cu:28-52):
    a pair is compared only when the reference's global index precedes the
    end of the query block's and the shorter length is at least the coverage
    times the longer; the pairs it compares keep their records, the rest
    get the filtered pair's record (TM-scores 0)."""
    from gtalign_alpha_b200 import synth
    rng = np.random.default_rng(7)
    base = synth.random_chains(rng, [60, 70, 90, 120])
    chains = base + [synth.homolog(rng, base[1], 0.8, 0.05, "h1"), synth.homolog(rng, base[3], 0.8, 0.05, "h3")]
    q = synth.pack(chains[:3])
    r = synth.pack(chains)
    rtype = np.array([0, 1, 2, 2**31 - 1, 2**31 - 1, 2**31 - 1], np.int32)
    rtype[4] = 1          # read as a query in an earlier block
    plain = oracle.process_block(q, r, oracle.opts_from(refinement=0, convergence=2))
    cov = 0.7
    cls = oracle.process_block(q, r, oracle.opts_from(refinement=0, convergence=2,
                                                     cls=(rtype, 3, cov)))
    lq, lr = q.lens[:, None].astype(np.float32), r.lens[None, :].astype(np.float32)
    passes = (rtype[None, :] < 3) & (np.maximum(lq, lr) * np.float32(cov) <= np.minimum(lq, lr))
    assert passes.any() and (~passes).any()
    a, b = plain.out, cls.out
    np.testing.assert_array_equal(a[passes], b[passes])
    np.testing.assert_array_equal(plain.tfm[passes], cls.tfm[passes])
    tm = b[~passes][:, 9:11]                # TM-scores by query and reference length
    assert (tm == 0).all() and (a[~passes][:, 9:11] > 0).all()
