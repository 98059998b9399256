"""The allocation-free entry point gives the results of gtb_process_block.

gtb_process_block_noalloc is for callers that cannot allocate device memory
at the time they align structures (code inside another framework's memory
pool, a fixed device footprint after start-up).  They pass their own device
buffers; the library's working memory is a fixed 16 MiB static device array.
This test calls it through the C ABI twice in a row on the same block (the
second call reuses the scratch the first left behind) and compares both
results with the allocating entry point, bit for bit as the other parity
tests do.  It also checks that an oversized block is refused before anything
runs.  The file is collected last so that a failure here never hides another
test's result.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class DevSoA(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("lens", ctypes.c_void_p), ("d_lens", ctypes.c_void_p),
                ("d_offs", ctypes.c_void_p), ("d_mol", ctypes.c_void_p),
                ("d_x", ctypes.c_void_p), ("d_y", ctypes.c_void_p), ("d_z", ctypes.c_void_p),
                ("d_rsd", ctypes.c_void_p), ("d_ss", ctypes.c_void_p)]


def _dev_block(s, keep):
    """Caller-owned device copies of a SoA block (allocated by the caller)."""
    import torch
    t = {
        "lens": torch.from_numpy(s.lens.astype(np.int32)).cuda(),
        "offs": torch.from_numpy(s.offs.astype(np.int32)).cuda(),
        "mol": torch.from_numpy(s.mol.astype(np.int32)).cuda(),
        "x": torch.from_numpy(s.x).cuda(), "y": torch.from_numpy(s.y).cuda(),
        "z": torch.from_numpy(s.z).cuda(),
        "rsd": torch.from_numpy(s.rsd).cuda(),
        "ss": torch.zeros(s.total, dtype=torch.uint8, device="cuda"),
    }
    hl = np.ascontiguousarray(s.lens, np.int32)
    keep.extend(list(t.values()) + [hl])
    return DevSoA(s.n, hl.ctypes.data, t["lens"].data_ptr(), t["offs"].data_ptr(),
                  t["mol"].data_ptr(), t["x"].data_ptr(), t["y"].data_ptr(), t["z"].data_ptr(),
                  t["rsd"].data_ptr(), t["ss"].data_ptr()), t


def _lib():
    from gtalign_alpha_b200.api import _COptions, load_library
    L = load_library()
    vp = ctypes.c_void_p
    L.gtb_process_block_noalloc.argtypes = [ctypes.c_int, ctypes.POINTER(_COptions), ctypes.c_float,
                                            ctypes.POINTER(DevSoA), ctypes.POINTER(DevSoA),
                                            vp, vp, vp, vp, ctypes.c_char_p, ctypes.c_size_t]
    L.gtb_process_block_noalloc.restype = ctypes.c_int
    return L


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options
    L = _lib()
    wl = synth.config0(seed=41, n_refs=9, qlen=130, lmin=40, lmax=300)
    wl.queries += synth.random_chains(np.random.default_rng(3), [75], "qz")
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    opts = Options(prescore=0.2, convergence=6)
    with GTalignB200(0, 0, opts) as g:
        ref = g.process_block(q, r, scorethld=0.3, alignments=False, secstr=True)
    keep = []
    dq, tq = _dev_block(q, keep)
    dr, tr = _dev_block(r, keep)
    np_ = q.n * r.n
    out = torch.zeros(np_ * 16, dtype=torch.float32, device="cuda")
    tfm = torch.zeros(np_ * 12, dtype=torch.float32, device="cuda")
    err = torch.zeros(np_ * 4, dtype=torch.float32, device="cuda")
    msg = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    copt = opts._c()
    for _ in range(2):
        out.fill_(-1.0)
        tfm.fill_(-1.0)
        st = L.gtb_process_block_noalloc(0, ctypes.byref(copt), ctypes.c_float(0.3),
                                         ctypes.byref(dq), ctypes.byref(dr), out.data_ptr(),
                                         tfm.data_ptr(), err.data_ptr(), stream, msg, 256)
        assert st == 0, msg.value
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.alndata.ravel().view(np.uint32))
        assert np.array_equal(tfm.cpu().numpy().view(np.uint32), ref.tfm.ravel().view(np.uint32))
        assert np.array_equal(err.cpu().numpy().view(np.uint32), ref.numerr.ravel().view(np.uint32))
        assert tq["ss"].cpu().numpy().tobytes() == ref.qss.tobytes()
        assert tr["ss"].cpu().numpy().tobytes() == ref.rss.tobytes()


def test_noalloc_rejects_blocks_beyond_its_scratch():
    import torch
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import Options
    L = _lib()
    rng = np.random.default_rng(5)
    # two 3000-residue chains need ~2.3 MB of traceback words per pair: 8 pairs > 16 MiB
    big = synth.random_chains(rng, [3000, 3000], "big")
    refs = synth.random_chains(rng, [3000, 3000, 3000, 3000], "bigr")
    q, r = synth.pack(big), synth.pack(refs)
    keep = []
    dq, _ = _dev_block(q, keep)
    dr, _ = _dev_block(r, keep)
    out = torch.zeros(8 * 16, dtype=torch.float32, device="cuda")
    tfm = torch.zeros(8 * 12, dtype=torch.float32, device="cuda")
    msg = ctypes.create_string_buffer(256)
    copt = Options()._c()
    st = L.gtb_process_block_noalloc(0, ctypes.byref(copt), ctypes.c_float(0.5), ctypes.byref(dq),
                                     ctypes.byref(dr), out.data_ptr(), tfm.data_ptr(), None,
                                     torch.cuda.current_stream().cuda_stream, msg, 256)
    assert st == 3
    assert b"static scratch" in msg.value
    assert float(out.abs().sum().item()) == 0.0


def _call(L, opts, q, r, thr=0.5):
    import torch
    keep = []
    dq, tq = _dev_block(q, keep)
    dr, tr = _dev_block(r, keep)
    np_ = q.n * r.n
    out = torch.full((np_ * 16,), -1.0, dtype=torch.float32, device="cuda")
    tfm = torch.full((np_ * 12,), -1.0, dtype=torch.float32, device="cuda")
    err = torch.zeros(np_ * 4, dtype=torch.float32, device="cuda")
    msg = ctypes.create_string_buffer(256)
    copt = opts._c()
    st = L.gtb_process_block_noalloc(0, ctypes.byref(copt), ctypes.c_float(thr), ctypes.byref(dq),
                                     ctypes.byref(dr), out.data_ptr(), tfm.data_ptr(), err.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream, msg, 256)
    torch.cuda.synchronize()
    return st, msg.value, out.cpu().numpy(), tfm.cpu().numpy(), err.cpu().numpy()


def test_noalloc_long_pair_matches_allocating_entry_point():
    """A 2,000 x 2,000-residue assembly pair: gtb_process_block runs its DP
    as a multi-CTA wavefront and its refinement over many CTAs; the
    allocation-free call runs both on single warps.  The results must be the
    same bits, on two calls in a row."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options
    L = _lib()
    wl = synth.config2(seed=3, lengths=(2000,))
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    opts = Options(prescore=0.4, convergence=4)
    with GTalignB200(0, 0, opts) as g:
        ref = g.process_block(q, r, scorethld=0.5, alignments=False)
    assert ref.alndata[0, 0, 9] > 0.5
    for _ in range(2):
        st, msg, out, tfm, err = _call(L, opts, q, r)
        assert st == 0, msg
        assert np.array_equal(out.view(np.uint32), ref.alndata.ravel().view(np.uint32))
        assert np.array_equal(tfm.view(np.uint32), ref.tfm.ravel().view(np.uint32))
        assert np.array_equal(err.view(np.uint32), ref.numerr.ravel().view(np.uint32))


def test_noalloc_refuses_nucleic_acid_pairs():
    """A block pairing two nucleic-acid structures is refused before any work
    (the output buffers keep their contents), as gtb_process_block refuses it;
    a protein query against the same nucleic-acid reference is accepted."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import Options
    L = _lib()
    rng = np.random.default_rng(9)
    na = synth.na_hairpins(rng, 2, 8, 5, "na0")
    na2 = synth.na_moved_copy(rng, na, 0.5, "na1")
    prot = synth.random_chains(rng, [60], "p")
    st, msg, out, _, _ = _call(L, Options(), synth.pack([na]), synth.pack([na2]))
    assert st == 4, msg
    assert b"nucleic" in msg
    assert np.all(out == -1.0)
    st, msg, out, _, _ = _call(L, Options(), synth.pack(prot), synth.pack([na2]))
    assert st == 0, msg
