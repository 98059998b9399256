"""TM-score adjoint and superposition polishing for fixed alignments.

Thin torch wrappers over the C ABI entry points gtb_tm_adjoint and
gtb_polish (CUDA kernels in csrc/gtb_adjoint.cu).  Layout: for P pairs,
pair p owns n[p] aligned residue pairs starting at row off[p] of the (N, 3)
float32 tensors q (query, moved by the transform) and r (reference);
tfm is (P, 12): row-major rotation then translation; d0 is (P,).
"""
from __future__ import annotations

import ctypes

import torch

from .api import GTBError, load_library


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _check(q, r, off, n, tfm, d0):
    for t in (q, r, tfm, d0):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise GTBError(1, "q, r, tfm, d0 must be contiguous float32 CUDA tensors")
    if not (off.is_cuda and off.dtype == torch.int64 and n.is_cuda and n.dtype == torch.int32):
        raise GTBError(1, "off must be int64 and n int32 CUDA tensors")


def tm_adjoint(q, r, off, n, tfm, d0, want_gq: bool = False):
    """TM (P,), gradient (P, 6) = (dTM/domega, dTM/dt), optional dTM/dq (N, 3).

    omega is a rotation vector applied on the left (R <- exp([omega]x) R),
    about the origin."""
    _check(q, r, off, n, tfm, d0)
    L = load_library()
    P = tfm.shape[0]
    tm = torch.empty(P, dtype=torch.float32, device=q.device)
    g = torch.empty(P, 6, dtype=torch.float32, device=q.device)
    gq = torch.zeros_like(q) if want_gq else None
    st = L.gtb_tm_adjoint(None, P, _ptr(off), _ptr(n), _ptr(q), _ptr(r), _ptr(tfm), _ptr(d0),
                          _ptr(tm), _ptr(g), _ptr(gq),
                          ctypes.c_void_p(torch.cuda.current_stream(q.device).cuda_stream))
    if st != 0:
        raise GTBError(st, "gtb_tm_adjoint failed")
    return tm, g, gq


def polish(q, r, off, n, tfm, d0, steps: int = 10):
    """Projected-gradient ascent on SO(3) x R^3; tfm is updated in place.
    Returns (tm_before, tm_after); a step is kept only if it raises TM."""
    _check(q, r, off, n, tfm, d0)
    L = load_library()
    P = tfm.shape[0]
    tb = torch.empty(P, dtype=torch.float32, device=q.device)
    ta = torch.empty(P, dtype=torch.float32, device=q.device)
    st = L.gtb_polish(None, P, _ptr(off), _ptr(n), _ptr(q), _ptr(r), _ptr(tfm), _ptr(d0),
                      int(steps), _ptr(tb), _ptr(ta),
                      ctypes.c_void_p(torch.cuda.current_stream(q.device).cuda_stream))
    if st != 0:
        raise GTBError(st, "gtb_polish failed")
    return tb, ta


class TMScore(torch.autograd.Function):
    """TM-score sums of P pairs as a differentiable function of the query
    coordinates q (N, 3) and the transforms tfm (P, 12).

    Backward: dTM/dq_i = R^T dTM/de_i (kernel), dTM/dt = sum_i dTM/de_i,
    dTM/dR = sum_i dTM/de_i q_i^T = R sum_i (dTM/dq_i) q_i^T.
    """

    @staticmethod
    def forward(ctx, q, tfm, r, off, n, d0):
        tm, g, gq = tm_adjoint(q.contiguous(), r, off, n, tfm.contiguous(), d0, want_gq=True)
        ctx.save_for_backward(q, tfm, off, n, g, gq)
        return tm

    @staticmethod
    def backward(ctx, gout):
        q, tfm, off, n, g, gq = ctx.saved_tensors
        P = tfm.shape[0]
        N = q.shape[0]
        # pair index and residue row of every aligned position, on the device:
        # row = off[pair] + (position - first position of the pair)
        nl = n.long()
        tot = int(nl.sum()) if P else 0
        pid = torch.repeat_interleave(torch.arange(P, device=q.device), nl, output_size=tot)
        start = torch.cumsum(nl, 0) - nl
        rows = off.long()[pid] + (torch.arange(tot, device=q.device) - start[pid])
        w = gout[pid]
        grad_q = torch.zeros_like(q)
        grad_q[rows] = gq[rows] * w[:, None]
        R = tfm[:, :9].reshape(P, 3, 3)
        outer = torch.zeros(P, 3, 3, device=q.device, dtype=q.dtype)
        outer.index_add_(0, pid, gq[rows][:, :, None] * q[rows][:, None, :])
        dR = torch.bmm(R, outer) * gout[:, None, None]
        dt = g[:, 3:] * gout[:, None]
        grad_tfm = torch.cat([dR.reshape(P, 9), dt], dim=1)
        return grad_q, grad_tfm, None, None, None, None
