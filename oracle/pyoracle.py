"""ctypes bindings of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
NOUT = 16
NERR = 4


def build(force: bool = False) -> str:
    """Compile oracle/gtoracle.c into oracle/liboracle.so (gcc, OpenMP)."""
    src = os.path.join(HERE, "gtoracle.c")
    deps = [src, os.path.join(HERE, "gtoracle.h"),
            os.path.join(os.path.dirname(HERE), "gtalign_alpha_b200", "csrc", "gtb_gonnet.h")]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(d) for d in deps):
        subprocess.check_call([
            "gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp",
            "-o", LIB, src, "-lm"])
    return LIB


class _Opts(ctypes.Structure):
    _fields_ = [("stepinit", ctypes.c_int), ("refinement", ctypes.c_int),
                ("depth", ctypes.c_int), ("convergence", ctypes.c_int),
                ("prescore", ctypes.c_float), ("scorethld", ctypes.c_float),
                ("symmetric", ctypes.c_int), ("referenced", ctypes.c_int),
                ("nodeletions", ctypes.c_int), ("twotmscore", ctypes.c_int),
                ("addsearchbyss", ctypes.c_int), ("presimilarity", ctypes.c_float),
                ("nodetailedsearch", ctypes.c_int), ("trigger", ctypes.c_int),
                ("nbranches", ctypes.c_int), ("gapcost", ctypes.c_float),
                ("seedrule", ctypes.c_int), ("window", ctypes.c_int),
                ("clsfilter", ctypes.c_int), ("clsrtype", ctypes.POINTER(ctypes.c_int)),
                ("clsqend", ctypes.c_int), ("clscoverage", ctypes.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        up = ctypes.POINTER(ctypes.c_ubyte)
        cp = ctypes.c_char_p
        L.gto_process_block.argtypes = [
            ctypes.POINTER(_Opts),
            ctypes.c_int, ip, fp, fp, fp, up, ip,
            ctypes.c_int, ip, fp, fp, fp, up, ip,
            fp, fp, fp, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.gto_process_block.restype = ctypes.c_int
        L.gto_process_block_ndx.argtypes = [
            ctypes.POINTER(_Opts),
            ctypes.c_int, ip, fp, fp, fp, up, ip, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ip, fp, fp, fp, up, ip, ctypes.c_void_p, ctypes.c_void_p,
            fp, fp, fp, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.gto_process_block_ndx.restype = ctypes.c_int
        L.gto_solve.argtypes = [fp, ctypes.c_int, fp]
        L.gto_solve.restype = ctypes.c_int
        L.gto_secstr.argtypes = [ctypes.c_int, fp, fp, fp, ctypes.c_void_p]
        L.gto_constants.argtypes = [ctypes.c_int, ctypes.c_int, fp, fp, fp, fp, fp]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


@dataclass
class OracleResult:
    out: np.ndarray      # (nq, nr, 16)
    tfm: np.ndarray      # (nq, nr, 12)
    err: np.ndarray      # (nq, nr, 4)
    alns: list           # [nq][nr] -> tuple of 5 strings
    qss: np.ndarray
    rss: np.ndarray


def opts_from(refinement: int = 0, convergence: int = 2, prescore: float = 0.0,
              scorethld: float = 0.0, depth: int = 2, symmetric: int = 0,
              referenced: int = 0, nodeletions: int = 0, twotmscore: int = 0,
              addsearchbyss: int = 0, presimilarity: float = 0.0,
              nodetailedsearch: int = 1, trigger: int = 50, nbranches: int = 5,
              gapcost: int = 1, seedrule: int = 1, window: int = 256,
              cls=None) -> _Opts:
    """Options in the gtalign command line's encoding: --refinement -1 log
    search, 0 coarse, 1 one search (the default), 2 full, 3 full in both final
    phases (the oracle, like the reference, stores code + 1); --depth 0..3
    (3 = shallow); --2tm-score; --add-search-by-ss; --pre-similarity; the
    detailed search: --no-detailed-search, --trigger, --nbranches, --gapcost
    code (0: -0.8, 1: -1.2, 2: -3.0), --seedrule code (0: fragments, 1: 64-,
    2: 128-residue local alignment frames), --window.  cls: a clustering
    run's prefilter, (the references' global indices, the end of the query
    block's global indices, --cls-coverage), or None."""
    o = _Opts(5 if depth == 3 else 1, refinement + 1, depth, convergence,
              prescore, scorethld, symmetric, referenced, nodeletions, twotmscore,
              addsearchbyss, presimilarity, nodetailedsearch, trigger, nbranches,
              (-0.8, -1.2, -3.0)[gapcost], (0, 64, 128)[seedrule], window)
    if cls is not None:
        rtype, qend, coverage = cls
        arr = np.ascontiguousarray(rtype, dtype=np.int32)
        o.clsfilter = 1
        o.clsrtype = arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        o.clsqend = int(qend)
        o.clscoverage = float(coverage)
        o._cls_keep = arr          # the array outlives the options
    return o


def _ndx_ptrs(ndx):
    """(float* [3], int* [3]) arrays of an index (x, y, z, left, right, residue)."""
    fa = (ctypes.c_void_p * 3)(*[np.ascontiguousarray(a, np.float32).ctypes.data for a in ndx[:3]])
    ia = (ctypes.c_void_p * 3)(*[np.ascontiguousarray(a, np.int32).ctypes.data for a in ndx[3:]])
    return fa, ia


def process_block(qsoa, rsoa, opts: _Opts, nthreads: int = 0, qndx=None, rndx=None) -> OracleResult:
    """qndx/rndx: the blocks' index trees (six arrays each), needed when
    opts.nodetailedsearch is 0."""
    L = lib()
    nq, nr = qsoa.n, rsoa.n
    out = np.zeros((nq * nr, NOUT), np.float32)
    tfm = np.zeros((nq * nr, 12), np.float32)
    err = np.zeros((nq * nr, NERR), np.float32)
    widths = (qsoa.lens[:, None].astype(np.int64) + rsoa.lens[None, :] + 1).ravel() * 5
    off = np.zeros(nq * nr, np.int64)
    if nq * nr > 1:
        off[1:] = np.cumsum(widths[:-1])
    alnbuf = np.zeros(int(widths.sum()), np.uint8)
    qss = np.zeros(qsoa.total, np.uint8)
    rss = np.zeros(rsoa.total, np.uint8)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    keep = []
    qf = qi_ = rf = ri_ = None
    if qndx is not None and rndx is not None:
        keep = [np.ascontiguousarray(a) for a in list(qndx) + list(rndx)]
        qf, qi_ = _ndx_ptrs(keep[:6])
        rf, ri_ = _ndx_ptrs(keep[6:])
    rc = L.gto_process_block_ndx(
        ctypes.byref(opts),
        nq, _p(qsoa.lens, ctypes.c_int), _p(qsoa.x, ctypes.c_float), _p(qsoa.y, ctypes.c_float),
        _p(qsoa.z, ctypes.c_float), _p(qsoa.rsd, ctypes.c_ubyte), _p(qsoa.mol, ctypes.c_int),
        qf, qi_,
        nr, _p(rsoa.lens, ctypes.c_int), _p(rsoa.x, ctypes.c_float), _p(rsoa.y, ctypes.c_float),
        _p(rsoa.z, ctypes.c_float), _p(rsoa.rsd, ctypes.c_ubyte), _p(rsoa.mol, ctypes.c_int),
        rf, ri_,
        _p(out, ctypes.c_float), _p(tfm, ctypes.c_float), _p(err, ctypes.c_float),
        alnbuf.ctypes.data, _p(off, ctypes.c_longlong),
        qss.ctypes.data, rss.ctypes.data, nthreads)
    if rc != 0:
        raise RuntimeError("oracle failed: %d" % rc)
    alns = []
    for qi in range(nq):
        row = []
        for ri in range(nr):
            p = qi * nr + ri
            W = int(qsoa.lens[qi] + rsoa.lens[ri] + 1)
            seg = alnbuf[off[p]:off[p] + 5 * W]
            strs = []
            for k in range(5):
                s = seg[k * W:(k + 1) * W].tobytes()
                strs.append(s.split(b"\0", 1)[0].decode("latin-1"))
            row.append(tuple(strs))
        alns.append(row)
    return OracleResult(out.reshape(nq, nr, NOUT), tfm.reshape(nq, nr, 12),
                        err.reshape(nq, nr, NERR), alns, qss, rss)


def solve(sums15: np.ndarray, n: int) -> np.ndarray:
    L = lib()
    s = np.ascontiguousarray(sums15, np.float32)
    t = np.zeros(12, np.float32)
    L.gto_solve(_p(s, ctypes.c_float), int(n), _p(t, ctypes.c_float))
    return t


def secstr(x, y, z) -> bytes:
    L = lib()
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    z = np.ascontiguousarray(z, np.float32)
    ss = np.zeros(len(x), np.uint8)
    L.gto_secstr(len(x), _p(x, ctypes.c_float), _p(y, ctypes.c_float), _p(z, ctypes.c_float),
                 ss.ctypes.data)
    return ss.tobytes()
