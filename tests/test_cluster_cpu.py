"""Clustering from all-against-all records (gtb_cluster: host code, no device).

Single linkage is checked against its definition (connected components of
the pairs within the threshold; lambda values = the minimum spanning tree's
edge weights), complete linkage against a transcription of the reference's
progressive CLINK (TdClustWriter.h:438-488), which keeps two relayed
lambdas in int variables.
"""
import numpy as np
import pytest

from gtalign_alpha_b200.api import NOUT, GTBError, cluster


def records(tm, L=100):
    """Records of n structures of length L with TM-scores tm[q, i] (the
    aligned length covers both structures, so coverage never excludes)."""
    n = tm.shape[0]
    rec = np.zeros((n, n, NOUT), np.float32)
    rec[:, :, 4] = L
    rec[:, :, 9] = tm
    rec[:, :, 10] = tm
    return rec, np.full(n, L, np.int32)


def planted(seed, n=60, groups=6):
    rng = np.random.default_rng(seed)
    tm = rng.uniform(0.05, 0.45, size=(n, n)).astype(np.float32)
    g = rng.integers(0, groups, size=n)
    same = g[:, None] == g[None, :]
    tm[same] = rng.uniform(0.3, 0.95, size=int(same.sum()))
    return tm


def dist(tm):
    return np.maximum(np.float32(0), np.float32(1) - tm).astype(np.float32)


def components(d, thr):
    n = d.shape[0]
    parent = list(range(n))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a
    for q in range(n):
        for i in range(q):
            if d[q, i] <= thr:
                parent[find(q)] = find(i)
    groups = {}
    for a in range(n):
        groups.setdefault(find(a), set()).add(a)
    return {frozenset(s) for s in groups.values()}


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_single_linkage_is_threshold_components(seed):
    tm = planted(seed)
    rec, lens = records(tm)
    for thr in (0.5, 0.7):
        c = cluster(rec, lens, linkage=1, threshold=thr)
        assert {frozenset(x) for x in c.clusters} == components(dist(tm), np.float32(1 - thr))
        assert sorted(sum(c.clusters, [])) == list(range(tm.shape[0]))


def test_single_linkage_heights_are_the_spanning_tree():
    tm = planted(4)
    rec, lens = records(tm)
    c = cluster(rec, lens, linkage=1)
    d = dist(tm)
    n = d.shape[0]
    full = np.where(np.tril(np.ones((n, n), bool), -1), d, d.T)   # d[q, i] for i < q, mirrored
    # Prim
    inside = np.zeros(n, bool)
    inside[0] = True
    best = full[0].copy()
    w = []
    for _ in range(n - 1):
        best[inside] = np.inf
        j = int(np.argmin(best))
        w.append(best[j])
        inside[j] = True
        best = np.minimum(best, full[j])
    finite = np.sort(c.lam[c.lam < 999.0])
    assert np.allclose(finite, np.sort(np.array(w, np.float32)))
    assert (c.pi[:-1] > np.arange(n - 1)).all() and c.pi[-1] == n - 1


def test_representatives_and_file_order():
    tm = planted(5)
    rec, lens = records(tm)
    ids = ["s%03d" % (59 - k) for k in range(60)]
    c = cluster(rec, lens, ids=ids, linkage=1)
    sizes = [len(x) for x in c.clusters]
    assert sizes == sorted(sizes, reverse=True)
    for a, b in zip(c.clusters, c.clusters[1:]):
        if len(a) == len(b):
            assert ids[a[0]] < ids[b[0]]
    for x in c.clusters:
        assert c.lam[x[0]] == min(c.lam[k] for k in x)


def clink_transcribed(d):
    """The reference's progressive CLINK step by step, with its int relays."""
    n = d.shape[0]
    BIG = np.float32(999.9)
    pi = np.zeros(n, np.int64)
    lam = np.zeros(n, np.float32)
    for q in range(n):
        mu = [np.float32(d[q, i]) for i in range(q)] + [BIG]
        pi[q] = q
        lam[q] = BIG
        for i in range(q):
            if lam[i] < mu[i]:
                mu[pi[i]] = max(mu[pi[i]], mu[i])
                mu[i] = BIG
        a = q - 1
        for k in range(q):
            i = q - 1 - k
            if lam[i] >= mu[pi[i]] and mu[i] < mu[a]:
                a = i
            if lam[i] < mu[pi[i]]:
                mu[i] = BIG
        b = c = a
        if 0 <= a:
            b = int(pi[a]); pi[a] = q
            c = int(lam[a]); lam[a] = mu[a]
        if a < q - 1:
            while b < q - 1:
                dd = int(pi[b]); pi[b] = q
                e = int(lam[b]); lam[b] = np.float32(c)
                b, c = dd, e
            if b == q - 1:
                pi[b] = q
                lam[b] = np.float32(c)
        for i in range(q):
            if pi[pi[i]] == q and lam[i] >= lam[pi[i]]:
                pi[i] = q
    return pi, lam


@pytest.mark.parametrize("seed", [6, 7])
def test_complete_linkage_follows_the_reference_steps(seed):
    tm = planted(seed, n=40)
    rec, lens = records(tm)
    c = cluster(rec, lens, linkage=0)
    pi, lam = clink_transcribed(dist(tm))
    assert np.array_equal(c.pi, pi.astype(np.int32))
    assert np.array_equal(c.lam, lam)
    assert sorted(sum(c.clusters, [])) == list(range(40))


def test_coverage_and_unaligned_pairs_are_far():
    tm = np.full((3, 3), 0.9, np.float32)
    rec, lens = records(tm)
    rec[1, 0, 4] = 50          # 50 of 100 residues aligned: below 0.7 coverage
    rec[2, 0, 4] = 0           # not aligned
    c = cluster(rec, lens, linkage=1)
    assert {frozenset(x) for x in c.clusters} == {frozenset({0}), frozenset({1, 2})}
    c = cluster(rec, lens, linkage=1, coverage=0.4)
    assert {frozenset(x) for x in c.clusters} == {frozenset({0, 1, 2})}


def test_invalid_options():
    rec, lens = records(np.zeros((2, 2), np.float32))
    for kw in (dict(linkage=2), dict(measure=9), dict(coverage=0.0), dict(threshold=-1.0)):
        with pytest.raises(GTBError) as e:
            cluster(rec, lens, **kw)
        assert e.value.status == 1


def test_streaming_equals_all_at_once():
    """gtb_cluster_create/add/finish, one structure's records at a time
    (only the entries before it), give the all-at-once result; rows must
    come in order."""
    import ctypes
    from gtalign_alpha_b200.api import _CClusterOptions, load_library
    L = load_library()
    tm = planted(8, n=30)
    rec, lens = records(tm)
    for linkage in (0, 1):
        ref = cluster(rec, lens, linkage=linkage)
        o = _CClusterOptions(linkage, 0, 0.5, 0.7, 0)
        vp, ip, fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)
        L.gtb_cluster_create.argtypes = [ctypes.c_int, ip, ctypes.POINTER(_CClusterOptions),
                                         ctypes.POINTER(vp)]
        L.gtb_cluster_add.argtypes = [vp, ctypes.c_int, fp]
        L.gtb_cluster_finish.argtypes = [vp, ip, fp, ip, ip, ip, ip]
        L.gtb_cluster_destroy.argtypes = [vp]
        h = vp()
        assert L.gtb_cluster_create(30, lens.ctypes.data_as(ip), ctypes.byref(o), ctypes.byref(h)) == 0
        assert L.gtb_cluster_add(h, 1, None) == 1           # out of order
        for q in range(30):
            row = np.ascontiguousarray(rec[q, :q]) if q else np.zeros((1, NOUT), np.float32)
            assert L.gtb_cluster_add(h, q, row.ctypes.data_as(fp)) == 0
        pi = np.zeros(30, np.int32)
        lam = np.zeros(30, np.float32)
        member = np.zeros(30, np.int32)
        offset = np.zeros(31, np.int32)
        rep = np.zeros(30, np.int32)
        ncl = ctypes.c_int()
        assert L.gtb_cluster_finish(h, pi.ctypes.data_as(ip), lam.ctypes.data_as(fp),
                                    member.ctypes.data_as(ip), offset.ctypes.data_as(ip),
                                    rep.ctypes.data_as(ip), ctypes.byref(ncl)) == 0
        L.gtb_cluster_destroy(h)
        assert np.array_equal(pi, ref.pi) and np.array_equal(lam, ref.lam)
        got = sorted((sorted(member[offset[c]:offset[c + 1]]) for c in range(ncl.value)))
        assert got == sorted(sorted(x) for x in ref.clusters)
