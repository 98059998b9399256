"""Host-side mirror of the reference's batch interface over the C ABI.

``GTalignB200.process_block`` corresponds to the reference's
``CuBatch::ProcessBlock`` (src/libmycu/cubatch/CuBatch.cuh:74-85): a block of
query structures and a block of reference structures, packed structure-of-
arrays exactly as ``PMBatchStrData`` packs them (field pointer arrays
``pmbeg``/``pmend``, src/libgenp/gdats/PM2DVectorFields.h:220-239), go in;
per-pair result records (gproc.h:148-168), 12-float transformation matrices
and alignment rows come out.  Everything runs in the in-tree CUDA library
``libgtb200.so``; there is no CPU fallback: a missing library is an error.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .synth import SoA

PKG = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(PKG, "libgtb200.so")

NOUT = 16
NERR = 4
NFIELDS = 10
# result record fields (gproc.h:148-168)
OUT_BEGCOORDS, OUT_ENDCOORDS, OUT_ALNLENGTH, OUT_PSTVS, OUT_IDNTS, OUT_NGAPS = 2, 3, 4, 5, 6, 7
OUT_RMSD, OUT_SCOREQ, OUT_SCORER, OUT_D0Q, OUT_D0R = 8, 9, 10, 11, 12

STATUS = {0: "GTB_OK", 1: "GTB_ERR_ARG", 2: "GTB_ERR_CUDA", 3: "GTB_ERR_NOMEM",
          4: "GTB_ERR_UNSUPPORTED", 5: "GTB_ERR_TOO_LONG", 6: "GTB_ERR_NOT_BUILT"}


class GTBError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (STATUS.get(status, str(status)), msg))
        self.status = status


class _COptions(ctypes.Structure):
    _fields_ = [("refinement", ctypes.c_int), ("depth", ctypes.c_int),
                ("convergence", ctypes.c_int), ("prescore", ctypes.c_float),
                ("symmetric", ctypes.c_int), ("referenced", ctypes.c_int),
                ("nodeletions", ctypes.c_int), ("nodetailedsearch", ctypes.c_int),
                ("addsearchbyss", ctypes.c_int), ("twotmscore", ctypes.c_int),
                ("polish_steps", ctypes.c_int), ("presimilarity", ctypes.c_float),
                ("trigger", ctypes.c_int), ("nbranches", ctypes.c_int),
                ("gapcost", ctypes.c_int), ("seedrule", ctypes.c_int), ("window", ctypes.c_int),
                ("clsfilter", ctypes.c_int), ("clscoverage", ctypes.c_float)]


class _CResults(ctypes.Structure):
    _fields_ = [("alndata", ctypes.c_void_p), ("tfm", ctypes.c_void_p),
                ("alns", ctypes.c_void_p), ("numerr", ctypes.c_void_p),
                ("qss", ctypes.c_void_p), ("rss", ctypes.c_void_p)]


class Tuning(ctypes.Structure):
    """Launch shapes of a handle (gtb_tuning); none changes a result."""
    _fields_ = [("seed_chunk", ctypes.c_int), ("refine_long_ctas", ctypes.c_int),
                ("dp_cta_pairs", ctypes.c_int), ("sub_pairs", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class _CTuningTrial(ctypes.Structure):
    _fields_ = [("t", Tuning), ("ms", ctypes.c_float)]


@dataclass
class Options:
    """Per-pair computation options, with the gtalign command line's codes.

    Defaults are the command line's defaults except ``nodetailedsearch``,
    which is 1 here (the spatial-index detailed search off); the command
    line's default, --speed 9, is ``Options.speed(9)``.
    """
    refinement: int = 1        # -1 log, 0 coarse, 1 one (default), 2 full, 3 full in both phases
    depth: int = 2
    convergence: int = 18
    prescore: float = 0.4
    symmetric: int = 0
    referenced: int = 0
    nodeletions: int = 0
    nodetailedsearch: int = 1
    addsearchbyss: int = 0
    twotmscore: int = 0
    polish_steps: int = 0      # adjoint polishing of the final transforms (this library only)
    presimilarity: float = 0.0  # --pre-similarity (0: off)
    trigger: int = 50          # detailed search: --trigger (percent)
    nbranches: int = 5         # --nbranches
    gapcost: int = 1           # --gapcost code: -0.8, -1.2, -3.0
    seedrule: int = 1          # --seedrule code: fragments, 64-, 128-residue frames
    window: int = 256          # --window
    clsfilter: int = 0         # 1: a clustering run's prefilter (blocks carry global indices)
    clscoverage: float = 0.7   # --cls-coverage

    @classmethod
    def speed(cls, level: int, **kw) -> "Options":
        """The --speed presets (gtalign.cpp:833-867, gtalign.h:189-208):
        13 = --no-detailed-search --refinement=0 --convergence=2; 10..12 =
        --depth=3 with --trigger 0/20/50, --refinement=0 --convergence=2; 7..9
        = --depth=2 with --trigger 0/20/50 (9 is the command line's default);
        4..6 = --depth=1 and 1..3 = --depth=0 with --trigger 0/20/50; 0 =
        --depth=0 --trigger=0 --nbranches=16 --add-search-by-ss."""
        if level == 13:
            return cls(refinement=0, convergence=2, **kw)
        trig = {0: 0, 1: 20, 2: 50}
        if 10 <= level <= 12:
            return cls(nodetailedsearch=0, depth=3, trigger=trig[level - 10], refinement=0,
                       convergence=2, **kw)
        if 7 <= level <= 9:
            return cls(nodetailedsearch=0, depth=2, trigger=trig[level - 7], **kw)
        if 4 <= level <= 6:
            return cls(nodetailedsearch=0, depth=1, trigger=trig[level - 4], **kw)
        if 1 <= level <= 3:
            return cls(nodetailedsearch=0, depth=0, trigger=trig[level - 1], **kw)
        if level == 0:
            return cls(nodetailedsearch=0, depth=0, trigger=0, nbranches=16, addsearchbyss=1, **kw)
        raise GTBError(1, "--speed %d out of 0..13" % level)

    def _c(self) -> _COptions:
        return _COptions(self.refinement, self.depth, self.convergence, self.prescore,
                         self.symmetric, self.referenced, self.nodeletions,
                         self.nodetailedsearch, self.addsearchbyss, self.twotmscore,
                         self.polish_steps, self.presimilarity, self.trigger, self.nbranches,
                         self.gapcost, self.seedrule, self.window, self.clsfilter,
                         self.clscoverage)


_lib = None


def load_library():
    """Load the in-tree libgtb200.so; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise GTBError(6, "libgtb200.so not built (run gtalign_alpha_b200.build.build())")
    L = ctypes.CDLL(LIBPATH)
    vp, fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)
    L.gtb_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_COptions), ctypes.POINTER(vp)]
    L.gtb_create.restype = ctypes.c_int
    L.gtb_process_block.argtypes = [vp, ctypes.c_float, vp, vp, vp, vp, ctypes.POINTER(_CResults)]
    L.gtb_process_block.restype = ctypes.c_int
    L.gtb_alns_size.argtypes = [vp, vp, vp, vp]
    L.gtb_alns_size.restype = ctypes.c_size_t
    L.gtb_last_error.argtypes = [vp]
    L.gtb_last_error.restype = ctypes.c_char_p
    L.gtb_last_launch_count.argtypes = [vp]
    L.gtb_last_launch_count.restype = ctypes.c_longlong
    L.gtb_last_timings.argtypes = [vp, fp]
    L.gtb_last_timings.restype = ctypes.c_int
    L.gtb_process_block_ndx.argtypes = [vp, ctypes.c_float, vp, vp, vp, vp, vp, vp,
                                        ctypes.POINTER(_CResults)]
    L.gtb_process_block_ndx.restype = ctypes.c_int
    L.gtb_build_index.argtypes = [vp, vp, vp]
    L.gtb_build_index.restype = ctypes.c_int
    L.gtb_last_work.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    L.gtb_last_work.restype = ctypes.c_int
    L.gtb_set_kernel_timing.argtypes = [vp, ctypes.c_int]
    L.gtb_set_kernel_timing.restype = ctypes.c_int
    L.gtb_last_kernel_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.gtb_last_kernel_ms.restype = ctypes.c_int
    L.gtb_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
    L.gtb_set_wait_limit.restype = ctypes.c_int
    L.gtb_destroy.argtypes = [vp]
    L.gtb_destroy.restype = None
    L.gtb_block_upload.argtypes = [vp, vp, vp, ctypes.POINTER(vp)]
    L.gtb_block_upload.restype = ctypes.c_int
    L.gtb_block_free.argtypes = [vp, vp]
    L.gtb_block_free.restype = None
    L.gtb_process_resident.argtypes = [vp, ctypes.c_float, vp, vp, vp, vp, vp]
    L.gtb_process_resident.restype = ctypes.c_int
    L.gtb_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.gtb_get_tuning.restype = ctypes.c_int
    L.gtb_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.gtb_set_tuning.restype = ctypes.c_int
    L.gtb_autotune.argtypes = [vp, ctypes.c_float, vp, vp, ctypes.c_int, ctypes.POINTER(Tuning),
                               ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_CTuningTrial),
                               ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.gtb_autotune.restype = ctypes.c_int
    L.gtb_tm_adjoint.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.gtb_tm_adjoint.restype = ctypes.c_int
    L.gtb_polish.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp]
    L.gtb_polish.restype = ctypes.c_int
    _lib = L
    return L


@dataclass
class PackedBlock:
    """The 10 SoA field arrays of a block and their begin/end pointers."""
    arrays: list
    beg: ctypes.Array
    end: ctypes.Array
    n: int
    npos: int


def pack_fields(s: SoA, types=None) -> PackedBlock:
    """Lay out a block the way PMBatchStrData does (one array per field).
    types: the structures' global indices in a clustering run (pps2DType), or
    None (zeros)."""
    n, N = s.n, s.total
    insch = np.zeros(N, np.int32)
    first = s.offs[s.mol > 0]
    insch[first] = 1                      # sign of the first residue: > 0 = nucleic acid
    arrays = [
        np.ascontiguousarray(s.lens, np.int32),
        np.ascontiguousarray(s.offs, np.uint32),
        np.zeros(n, np.int32) if types is None else np.ascontiguousarray(types, np.int32),
        np.ascontiguousarray(s.x, np.float32),
        np.ascontiguousarray(s.y, np.float32),
        np.ascontiguousarray(s.z, np.float32),
        insch,
        np.arange(N, dtype=np.int32),
        np.ascontiguousarray(s.rsd, np.uint8),
        np.zeros(N, np.uint8),
    ]
    beg = (ctypes.c_void_p * NFIELDS)()
    end = (ctypes.c_void_p * NFIELDS)()
    for f, a in enumerate(arrays):
        beg[f] = a.ctypes.data
        end[f] = a.ctypes.data + a.nbytes
    return PackedBlock(arrays, beg, end, n, N)


def build_index(s: SoA) -> Tuple[np.ndarray, ...]:
    """The block's index trees as the reference's reader makes them
    (gtb_build_index): node x, y, z (float32), left and right child and
    residue (int32), one entry per residue."""
    L = load_library()
    pk = pack_fields(s)
    arrs = [np.zeros(s.total, np.float32) for _ in range(3)] + [np.zeros(s.total, np.int32) for _ in range(3)]
    ndx = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    st = L.gtb_build_index(pk.beg, pk.end, ndx)
    if st != 0:
        raise GTBError(st, "gtb_build_index failed")
    return tuple(arrs)


@dataclass
class BlockResult:
    alndata: np.ndarray            # (nq, nr, 16)
    tfm: np.ndarray                # (nq, nr, 12)
    numerr: Optional[np.ndarray]   # (nq, nr, 4)
    alns_raw: Optional[np.ndarray] # reference layout bytes
    qlens: np.ndarray
    rlens: np.ndarray
    roffs: np.ndarray
    qss: Optional[np.ndarray] = None
    rss: Optional[np.ndarray] = None
    launches: int = 0
    timings_ms: np.ndarray = field(default_factory=lambda: np.zeros(7, np.float32))
    # device-counted work: seed position visits, refinement position visits, DP cells
    work: np.ndarray = field(default_factory=lambda: np.zeros(3, np.uint64))

    @property
    def tm_query(self) -> np.ndarray:
        return self.alndata[..., OUT_SCOREQ]

    @property
    def tm_ref(self) -> np.ndarray:
        return self.alndata[..., OUT_SCORER]

    @property
    def rmsd(self) -> np.ndarray:
        return self.alndata[..., OUT_RMSD]

    def alignment(self, qi: int, ri: int) -> Tuple[str, str, str, str, str]:
        """(query row, middle row, target row, query SS, target SS)."""
        if self.alns_raw is None:
            raise ValueError("alignments were not requested")
        nr = len(self.rlens)
        Nr = int(self.rlens.sum())
        base = 0
        for k in range(qi):
            base += 5 * (Nr + nr * (int(self.qlens[k]) + 1))
        lq = int(self.qlens[qi])
        rowlen = Nr + nr * (lq + 1)
        col = int(self.roffs[ri]) + ri * (lq + 1)
        W = lq + int(self.rlens[ri]) + 1
        rows = []
        for f in range(5):
            seg = self.alns_raw[base + f * rowlen + col: base + f * rowlen + col + W].tobytes()
            rows.append(seg.split(b"\0", 1)[0].decode("latin-1"))
        return tuple(rows)


class GTalignB200:
    """One handle = one device area (the CuBatch analogue)."""

    def __init__(self, device: int = 0, mem_bytes: int = 0, options: Optional[Options] = None):
        self.lib = load_library()
        self.options = options or Options()
        self._h = ctypes.c_void_p()
        copt = self.options._c()
        st = self.lib.gtb_create(device, mem_bytes, ctypes.byref(copt), ctypes.byref(self._h))
        if st != 0:
            msg = self.lib.gtb_last_error(self._h).decode() if self._h else ""
            if self._h:
                self.lib.gtb_destroy(self._h)
                self._h = ctypes.c_void_p()
            raise GTBError(st, msg)

    def close(self) -> None:
        if self._h:
            self.lib.gtb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_wait_limit(self, spins: int) -> None:
        """Spins a bounded wait of the multi-CTA DP makes before it gives up."""
        st = self.lib.gtb_set_wait_limit(self._h, int(spins))
        if st != 0:
            raise GTBError(st, "wait limit must be >= 0")

    def last_work(self) -> np.ndarray:
        """Device-counted work of the last call (seed visits, refinement
        visits, DP cells, the detailed search's slot-score DP cells)."""
        w = np.zeros(4, np.uint64)
        self.lib.gtb_last_work(self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)))
        return w

    def set_kernel_timing(self, on: bool) -> None:
        """Per-family device timing of the following calls (gtb_set_kernel_timing)."""
        self.lib.gtb_set_kernel_timing(self._h, 1 if on else 0)

    def last_kernel_ms(self) -> np.ndarray:
        """Summed device time (ms) of the last call's seed, refinement, DP
        and detailed-search launches."""
        ms = np.zeros(4, np.float32)
        self.lib.gtb_last_kernel_ms(self._h, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        return ms

    def get_tuning(self) -> Tuning:
        t = Tuning()
        self.lib.gtb_get_tuning(self._h, ctypes.byref(t))
        return t

    def set_tuning(self, t: Optional[Tuning] = None, **fields) -> None:
        """Set the launch shapes: a Tuning, or fields changed from the
        current one (seed_chunk=..., refine_long_ctas=..., ...)."""
        t2 = self.get_tuning() if t is None else Tuning(**t.as_dict())
        for k, v in fields.items():
            if k not in t2.as_dict():
                raise GTBError(1, "no tuning field %r" % k)
            setattr(t2, k, int(v))
        st = self.lib.gtb_set_tuning(self._h, ctypes.byref(t2))
        if st != 0:
            raise GTBError(st, self.lib.gtb_last_error(self._h).decode())

    def upload(self, blk: PackedBlock) -> "ResidentBlock":
        """A block copied to the device once (gtb_block_upload)."""
        h = ctypes.c_void_p()
        st = self.lib.gtb_block_upload(self._h, blk.beg, blk.end, ctypes.byref(h))
        if st != 0:
            raise GTBError(st, self.lib.gtb_last_error(self._h).decode())
        return ResidentBlock(self, h, blk.n)

    def autotune(self, queries: "ResidentBlock", refs: "ResidentBlock", scorethld: float = 0.5,
                 trials: int = 1, nlog: int = 32):
        """Pick the launch shapes for this workload (gtb_autotune; the blocks
        are ResidentBlocks or gtb_block handles): returns
        (the tuning left set, its ms per call, [(tuning dict, ms) tried])."""
        best = Tuning()
        ms = ctypes.c_float()
        log = (_CTuningTrial * nlog)()
        nl = ctypes.c_int()
        qh, rh = getattr(queries, "h", queries), getattr(refs, "h", refs)
        st = self.lib.gtb_autotune(self._h, float(scorethld), qh, rh, int(trials),
                                   ctypes.byref(best), ctypes.byref(ms), log, nlog,
                                   ctypes.byref(nl))
        if st != 0:
            raise GTBError(st, self.lib.gtb_last_error(self._h).decode())
        return best, float(ms.value), [(log[k].t.as_dict(), float(log[k].ms)) for k in range(nl.value)]

    def process_block(self, queries: SoA, refs: SoA, scorethld: float = 0.5,
                      alignments: bool = True, numerr: bool = True,
                      secstr: bool = False, qndx=None, rndx=None, qtypes=None,
                      rtypes=None) -> BlockResult:
        """qndx/rndx (build_index): the blocks' index trees as a reader made
        them; without them the library builds the same when it needs them.
        qtypes/rtypes: the structures' global indices in a clustering run
        (Options.clsfilter)."""
        qb, rb = pack_fields(queries, qtypes), pack_fields(refs, rtypes)
        return self.process_packed(qb, rb, scorethld, alignments, numerr, secstr, qndx=qndx,
                                   rndx=rndx)

    def process_packed(self, qb: PackedBlock, rb: PackedBlock, scorethld: float = 0.5,
                       alignments: bool = True, numerr: bool = True,
                       secstr: bool = False, out: Optional[dict] = None,
                       qndx=None, rndx=None) -> BlockResult:
        nq, nr = qb.n, rb.n
        if out is None:
            out = {}
        aln = out.get("alndata")
        if aln is None or aln.shape != (nq * nr, NOUT):
            aln = np.zeros((nq * nr, NOUT), np.float32)
        tfm = out.get("tfm")
        if tfm is None or tfm.shape != (nq * nr, 12):
            tfm = np.zeros((nq * nr, 12), np.float32)
        err = np.zeros((nq * nr, NERR), np.float32) if numerr else None
        alns = None
        if alignments:
            sz = self.lib.gtb_alns_size(qb.beg, qb.end, rb.beg, rb.end)
            alns = np.zeros(sz, np.uint8)
        qss = np.zeros(qb.npos, np.uint8) if secstr else None
        rss = np.zeros(rb.npos, np.uint8) if secstr else None
        res = _CResults(aln.ctypes.data, tfm.ctypes.data,
                        alns.ctypes.data if alns is not None else None,
                        err.ctypes.data if err is not None else None,
                        qss.ctypes.data if qss is not None else None,
                        rss.ctypes.data if rss is not None else None)
        if qndx is not None and rndx is not None:
            qn = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in qndx])
            rn = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in rndx])
            st = self.lib.gtb_process_block_ndx(self._h, float(scorethld), qb.beg, qb.end, qn,
                                                rb.beg, rb.end, rn, ctypes.byref(res))
        else:
            st = self.lib.gtb_process_block(self._h, float(scorethld), qb.beg, qb.end, rb.beg,
                                            rb.end, ctypes.byref(res))
        if st != 0:
            raise GTBError(st, self.lib.gtb_last_error(self._h).decode())
        tms = np.zeros(7, np.float32)
        self.lib.gtb_last_timings(self._h, tms.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        return BlockResult(aln.reshape(nq, nr, NOUT), tfm.reshape(nq, nr, 12),
                           err.reshape(nq, nr, NERR) if err is not None else None,
                           alns, qb.arrays[0].copy(), rb.arrays[0].copy(), rb.arrays[1].copy(),
                           qss, rss, int(self.lib.gtb_last_launch_count(self._h)), tms,
                           self.last_work())


class ResidentBlock:
    """A block on the device (GTalignB200.upload); free it before the handle."""

    def __init__(self, g: GTalignB200, h: ctypes.c_void_p, n: int):
        self.g, self.h, self.n = g, h, n

    def free(self) -> None:
        if self.h:
            self.g.lib.gtb_block_free(self.g.handle, self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()


class _CReaderOptions(ctypes.Structure):
    _fields_ = [("ter", ctypes.c_int), ("split", ctypes.c_int), ("hetatm", ctypes.c_int),
                ("mol", ctypes.c_int), ("aatom", ctypes.c_char * 5), ("natom", ctypes.c_char * 5),
                ("minlen", ctypes.c_int), ("maxlen", ctypes.c_int), ("infmt", ctypes.c_int)]


@dataclass
class ReadBlock:
    """Structures read by read_pdb: the block as a SoA (for process_block),
    its reference-layout fields as read (PackedBlock, for process_packed and
    gtb_block_upload) and each structure's description."""
    soa: SoA
    packed: PackedBlock
    descriptions: list


def read_pdb(paths, ter: int = 3, split: int = 0, hetatm: bool = False, mol: int = 2,
             aatom: str = " CA ", natom: str = " C3'", minlen: int = 20, maxlen: int = 65535,
             infmt: int = 0, threads: int = 0) -> ReadBlock:
    """Read PDB and PDBx/mmCIF files (plain or gzip) into one block
    (gtb_read_pdb), with the reference's interpretation options (--ter,
    --split, --hetatm, --mol, --aatom, --natom, --dev-min-length,
    --dev-max-length, --infmt).  Host code."""
    L = load_library()
    L.gtb_read_pdb.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_CReaderOptions),
                               ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                               ctypes.c_size_t]
    L.gtb_read_pdb.restype = ctypes.c_int
    L.gtb_structs_size.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_longlong)]
    L.gtb_structs_fields.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.gtb_structs_description.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.gtb_structs_description.restype = ctypes.c_char_p
    L.gtb_structs_free.argtypes = [ctypes.c_void_p]
    L.gtb_structs_free.restype = None
    if len(aatom) != 4 or len(natom) != 4:
        raise GTBError(1, "atom names have 4 characters")
    o = _CReaderOptions(int(ter), int(split), int(bool(hetatm)), int(mol), aatom.encode(),
                        natom.encode(), int(minlen), int(maxlen), int(infmt))
    enc = [os.fsencode(p) for p in paths]
    arr = (ctypes.c_char_p * max(1, len(enc)))(*enc)
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(512)
    st = L.gtb_read_pdb(ctypes.cast(arr, ctypes.c_void_p), len(enc), ctypes.byref(o), int(threads),
                        ctypes.byref(h), err, 512)
    if st != 0:
        raise GTBError(st, err.value.decode())
    try:
        ns, npos = ctypes.c_int(), ctypes.c_longlong()
        L.gtb_structs_size(h, ctypes.byref(ns), ctypes.byref(npos))
        beg = (ctypes.c_void_p * NFIELDS)()
        end = (ctypes.c_void_p * NFIELDS)()
        L.gtb_structs_fields(h, beg, end)
        dtypes = [np.int32, np.uint32, np.int32, np.float32, np.float32, np.float32, np.int32,
                  np.int32, np.uint8, np.uint8]
        arrays = []
        for f, dt in enumerate(dtypes):
            nb = (end[f] or 0) - (beg[f] or 0)
            a = np.empty(nb // np.dtype(dt).itemsize, dt)
            if nb:
                ctypes.memmove(a.ctypes.data, beg[f], nb)
            arrays.append(a)
        desc = [L.gtb_structs_description(h, i).decode() for i in range(ns.value)]
    finally:
        L.gtb_structs_free(h)
    pb = (ctypes.c_void_p * NFIELDS)()
    pe = (ctypes.c_void_p * NFIELDS)()
    for f, a in enumerate(arrays):
        pb[f] = a.ctypes.data
        pe[f] = a.ctypes.data + a.nbytes
    packed = PackedBlock(arrays, pb, pe, ns.value, int(npos.value))
    lens, offs = arrays[0], arrays[1].astype(np.int32)
    first = arrays[6][offs] if ns.value else np.zeros(0, np.int32)
    soa = SoA(lens.copy(), offs, arrays[3].copy(), arrays[4].copy(), arrays[5].copy(),
              arrays[8].copy(), (first > 0).astype(np.int32))
    return ReadBlock(soa, packed, desc)


class _CClusterOptions(ctypes.Structure):
    _fields_ = [("linkage", ctypes.c_int), ("measure", ctypes.c_int),
                ("threshold", ctypes.c_float), ("coverage", ctypes.c_float),
                ("onesided", ctypes.c_int)]


@dataclass
class Clusters:
    """Clusters of n structures: each a list of structure indices with the
    representative first, listed as the reference's cluster file lists them
    (largest first, then by the representative's id); and the pointer
    representation (pi, lambda) of the linkage."""
    clusters: list
    pi: np.ndarray
    lam: np.ndarray


def cluster(alndata: np.ndarray, lens: np.ndarray, ids: Optional[list] = None,
            linkage: int = 0, measure: int = 0, threshold: float = 0.5,
            coverage: float = 0.7, onesided: bool = False) -> Clusters:
    """Cluster n structures from the (n, n, GTB_NOUT) records of their
    all-against-all block with gtb_cluster (the --cls options: linkage 0
    complete / 1 single, measure = --sort, threshold, coverage, one-sided).
    ``ids`` (default: the indices as strings) order clusters of equal size."""
    L = load_library()
    rec = np.ascontiguousarray(alndata, dtype=np.float32)
    n = int(rec.shape[0])
    if rec.shape != (n, n, NOUT):
        raise GTBError(1, "records must have shape (n, n, %d)" % NOUT)
    lens = np.ascontiguousarray(lens, dtype=np.int32)
    ids = [str(i) for i in range(n)] if ids is None else list(ids)
    o = _CClusterOptions(linkage, measure, threshold, coverage, 1 if onesided else 0)
    pi = np.zeros(n, np.int32)
    lam = np.zeros(n, np.float32)
    member = np.zeros(n, np.int32)
    offset = np.zeros(n + 1, np.int32)
    rep = np.zeros(n, np.int32)
    ncl = ctypes.c_int(0)
    ip = ctypes.POINTER(ctypes.c_int)
    fp = ctypes.POINTER(ctypes.c_float)
    L.gtb_cluster.argtypes = [ctypes.c_int, fp, ip, ctypes.POINTER(_CClusterOptions),
                              ip, fp, ip, ip, ip, ip]
    L.gtb_cluster.restype = ctypes.c_int
    st = L.gtb_cluster(n, rec.ctypes.data_as(fp), lens.ctypes.data_as(ip), ctypes.byref(o),
                       pi.ctypes.data_as(ip), lam.ctypes.data_as(fp), member.ctypes.data_as(ip),
                       offset.ctypes.data_as(ip), rep.ctypes.data_as(ip), ctypes.byref(ncl))
    if st != 0:
        raise GTBError(st, "gtb_cluster: invalid arguments")
    cl = [list(member[offset[c]:offset[c + 1]]) for c in range(ncl.value)]
    cl.sort(key=lambda c: (-len(c), ids[c[0]]))
    return Clusters(cl, pi, lam)
