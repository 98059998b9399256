"""TM-score adjoint (FP32 kernel) against FP64 central finite differences
and the FP64 analytic gradient; polishing never lowers the TM-score."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs(seed=0, P=24, lo=60, hi=600):
    """Aligned pairs of homologous synthetic chains (fixed 1:1 alignment) and
    a perturbed starting transform."""
    from gtalign_alpha_b200 import synth
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi, size=P)
    ch = synth.random_chains(rng, lens, "a")
    q, r, off, n, tfm, d0 = [], [], [], [], [], []
    o = 0
    for c in ch:
        x = c.xyz.astype(np.float64)
        R = synth._rot_random(rng)
        y = x @ R.T + rng.normal(0, 1.5, size=x.shape) + rng.uniform(-5, 5, size=3)
        # start from a slightly wrong transform
        ang = rng.normal(0, 0.05, size=3)
        th = np.linalg.norm(ang)
        K = np.array([[0, -ang[2], ang[1]], [ang[2], 0, -ang[0]], [-ang[1], ang[0], 0]])
        E = np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K
        R0 = E @ R
        t0 = y.mean(0) - R0 @ x.mean(0) + rng.normal(0, 0.5, size=3)
        q.append(x); r.append(y); off.append(o); n.append(len(x)); o += len(x)
        tfm.append(np.concatenate([R0.ravel(), t0]))
        L = len(x)
        d0.append(max(0.5, 1.24 * np.cbrt(L - 15) - 1.8))
    return (np.concatenate(q).astype(np.float32), np.concatenate(r).astype(np.float32),
            np.array(off, np.int64), np.array(n, np.int32), np.array(tfm, np.float32),
            np.array(d0, np.float32))


def tm64(q, r, T, d0):
    R = T[:9].reshape(3, 3).astype(np.float64)
    e = q.astype(np.float64) @ R.T + T[9:].astype(np.float64) - r
    return float(np.sum(d0 ** 2 / (d0 ** 2 + (e ** 2).sum(1))))


def grad64(q, r, T, d0):
    R = T[:9].reshape(3, 3).astype(np.float64)
    p = q.astype(np.float64) @ R.T
    e = p + T[9:] - r
    u = d0 ** 2 + (e ** 2).sum(1)
    ge = -2 * d0 ** 2 * e / u[:, None] ** 2
    return np.concatenate([np.cross(p, ge).sum(0), ge.sum(0)]), ge @ R


def rot(w):
    th = np.linalg.norm(w)
    K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    if th < 1e-15:
        return np.eye(3) + K
    return np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K


def test_gradient_matches_fd_and_fp64():
    import torch
    from gtalign_alpha_b200.adjoint import tm_adjoint
    q, r, off, n, tfm, d0 = _pairs()
    dev = "cuda"
    T = lambda a: torch.from_numpy(a).to(dev)
    tm, g, gq = tm_adjoint(T(q), T(r), T(off), T(n), T(tfm), T(d0), want_gq=True)
    tm, g, gq = tm.cpu().numpy(), g.cpu().numpy(), gq.cpu().numpy()
    for p in range(len(n)):
        s = slice(off[p], off[p] + n[p])
        Q, Rr, Tp, d = q[s], r[s].astype(np.float64), tfm[p].astype(np.float64), float(d0[p])
        assert abs(tm[p] - tm64(Q, Rr, Tp, d)) <= 1e-5 * max(1.0, tm[p])
        ga, gqa = grad64(Q, Rr, Tp, d)
        # FP64 central differences: h = 1e-5 rad, 1e-4 A
        fd = np.zeros(6)
        for k in range(3):
            w = np.zeros(3); w[k] = 1e-5
            Tpp, Tpm = Tp.copy(), Tp.copy()
            Tpp[:9] = (rot(w) @ Tp[:9].reshape(3, 3)).ravel(); Tpp[9:] = rot(w) @ Tp[9:]
            Tpm[:9] = (rot(-w) @ Tp[:9].reshape(3, 3)).ravel(); Tpm[9:] = rot(-w) @ Tp[9:]
            fd[k] = (tm64(Q, Rr, Tpp, d) - tm64(Q, Rr, Tpm, d)) / 2e-5
            Tpp, Tpm = Tp.copy(), Tp.copy()
            Tpp[9 + k] += 1e-4; Tpm[9 + k] -= 1e-4
            fd[3 + k] = (tm64(Q, Rr, Tpp, d) - tm64(Q, Rr, Tpm, d)) / 2e-4
        # rotating the transformed point about the origin also moves t: the
        # kernel's omega acts on R only, so compare with the analytic form
        # and the FD for the translation part
        scale = np.linalg.norm(ga) + 1e-12
        assert np.linalg.norm(g[p] - ga) <= 1e-3 * scale, (g[p], ga)
        assert np.linalg.norm(fd[3:] - ga[3:]) <= 1e-3 * (np.linalg.norm(ga[3:]) + 1e-9)
        assert np.abs(gq[s] - gqa).max() <= 1e-3 * (np.abs(gqa).max() + 1e-9)


def test_rotation_gradient_fd():
    """dTM/domega for R <- exp([omega]x) R (translation fixed) by FP64
    central differences, relative error <= 1e-3."""
    import torch
    from gtalign_alpha_b200.adjoint import tm_adjoint
    q, r, off, n, tfm, d0 = _pairs(seed=1, P=12)
    T = lambda a: torch.from_numpy(a).to("cuda")
    _, g, _ = tm_adjoint(T(q), T(r), T(off), T(n), T(tfm), T(d0))
    g = g.cpu().numpy()
    for p in range(len(n)):
        s = slice(off[p], off[p] + n[p])
        Q, Rr, Tp, d = q[s], r[s].astype(np.float64), tfm[p].astype(np.float64), float(d0[p])
        fd = np.zeros(3)
        for k in range(3):
            w = np.zeros(3); w[k] = 1e-5
            Tpp, Tpm = Tp.copy(), Tp.copy()
            Tpp[:9] = (rot(w) @ Tp[:9].reshape(3, 3)).ravel()
            Tpm[:9] = (rot(-w) @ Tp[:9].reshape(3, 3)).ravel()
            fd[k] = (tm64(Q, Rr, Tpp, d) - tm64(Q, Rr, Tpm, d)) / 2e-5
        assert np.linalg.norm(g[p, :3] - fd) <= 1e-3 * np.linalg.norm(fd), (g[p, :3], fd)


def test_polish_never_decreases_and_improves():
    import torch
    from gtalign_alpha_b200.adjoint import polish
    q, r, off, n, tfm, d0 = _pairs(seed=2, P=64)
    T = lambda a: torch.from_numpy(a).to("cuda")
    tt = T(tfm.copy())
    tb, ta = polish(T(q), T(r), T(off), T(n), tt, T(d0), steps=20)
    tb, ta, tn = tb.cpu().numpy(), ta.cpu().numpy(), tt.cpu().numpy()
    for p in range(len(n)):
        s = slice(off[p], off[p] + n[p])
        before = tm64(q[s], r[s].astype(np.float64), tfm[p].astype(np.float64), float(d0[p]))
        after = tm64(q[s], r[s].astype(np.float64), tn[p].astype(np.float64), float(d0[p]))
        assert after >= before - 1e-6 * n[p], (p, before, after)
        R = tn[p, :9].reshape(3, 3).astype(np.float64)
        assert np.abs(R @ R.T - np.eye(3)).max() < 1e-5
    assert (ta >= tb).all()
    assert np.mean(ta - tb) > 0


def test_autograd_function_matches_fp64():
    import torch
    from gtalign_alpha_b200.adjoint import TMScore
    q, r, off, n, tfm, d0 = _pairs(seed=3, P=6)
    dev = "cuda"
    qt = torch.from_numpy(q).to(dev).requires_grad_(True)
    tt = torch.from_numpy(tfm).to(dev).requires_grad_(True)
    tm = TMScore.apply(qt, tt, torch.from_numpy(r).to(dev), torch.from_numpy(off).to(dev),
                       torch.from_numpy(n).to(dev), torch.from_numpy(d0).to(dev))
    tm.sum().backward()
    # FP64 autograd of the same expression as the oracle of the gradient
    q64 = torch.from_numpy(q).double().requires_grad_(True)
    t64 = torch.from_numpy(tfm).double().requires_grad_(True)
    tot = 0
    for p in range(len(n)):
        s = slice(int(off[p]), int(off[p] + n[p]))
        R = t64[p, :9].reshape(3, 3)
        e = q64[s] @ R.T + t64[p, 9:] - torch.from_numpy(r[s]).double()
        tot = tot + (float(d0[p]) ** 2 / (float(d0[p]) ** 2 + (e ** 2).sum(1))).sum()
    tot.backward()
    gq, g64 = qt.grad.cpu().double(), q64.grad
    assert (gq - g64).abs().max() <= 1e-3 * g64.abs().max()
    gt, gt64 = tt.grad.cpu().double(), t64.grad
    assert (gt - gt64).abs().max() <= 1e-3 * gt64.abs().max()


def test_polishing_in_the_search_never_lowers_the_score():
    """polish_steps > 0 polishes each pair's final transform with the adjoint
    before the FP64 recomputation: the score by the shorter structure's
    length never goes down, the alignments stay, and homologs gain."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options
    wl = synth.config0(seed=23, n_refs=60, qlen=150, lmin=50, lmax=400)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    res = {}
    for steps in (0, 10):
        with GTalignB200(0, 0, Options(prescore=0.0, polish_steps=steps)) as g:
            res[steps] = g.process_block(q, r, scorethld=0.0, alignments=False)
    a, b = res[0].alndata[0], res[10].alndata[0]
    lq = q.lens[0]
    short = np.where(lq <= r.lens, a[:, 9], a[:, 10]), np.where(lq <= r.lens, b[:, 9], b[:, 10])
    assert np.all(short[1] >= short[0] - 1e-6)
    assert np.array_equal(a[:, 2:8], b[:, 2:8])          # same alignments
    gain = short[1] - short[0]
    assert (gain > 1e-5).sum() > 5
    assert float(np.max(res[10].numerr[0][:, :2])) < 1e-5  # FP32 vs FP64 of the polished transform
