"""A small, fixed workload for profiling (ncu) and quick timing.

    python -m gtalign_alpha_b200.profile_case --queries 2 --refs 500

Aligns the first `--queries` queries of the seeded benchmark workload (seed 2)
with `--refs` references under the default options (--no-detailed-search,
-s 0.5) in gtb_process_block calls (one warm-up call, one timed call) and
prints the wall time and the stage timings of the timed call.

    python -m gtalign_alpha_b200.profile_case --long 5000,37860

times long-chain pairs (a multi-domain assembly against its per-domain
perturbed partner), one call per pair;

    python -m gtalign_alpha_b200.profile_case --adjoint 1000000 --steps 10

times adjoint polishing of a million fixed-alignment pairs.
"""
from __future__ import annotations

import argparse

from . import synth
from .api import GTalignB200, Options


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--queries", type=int, default=2)
    ap.add_argument("--refs", type=int, default=500)
    ap.add_argument("--speed13", action="store_true")
    ap.add_argument("--long", default="",
                    help="comma-separated lengths: time the long-chain pairs (assembly vs "
                         "its perturbed partner, one call per pair) instead")
    ap.add_argument("--adjoint", type=int, default=0,
                    help="time adjoint polishing of this many fixed-alignment pairs instead")
    ap.add_argument("--steps", type=int, default=10, help="polishing steps (--adjoint)")
    a = ap.parse_args()
    if a.adjoint:
        adjoint_pairs(a.adjoint, a.steps)
        return
    if a.long:
        long_chains([int(x) for x in a.long.split(",")])
        return
    wl = synth.config1(seed=2, n_queries=max(a.queries, 1), n_refs=a.refs)
    q, r = synth.pack(wl.queries[:a.queries]), synth.pack(wl.refs)
    opts = Options.speed(13) if a.speed13 else Options()
    import time
    with GTalignB200(0, 0, opts) as g:
        res = g.process_block(q, r, scorethld=0.5, alignments=False)
        t0 = time.perf_counter()
        res = g.process_block(q, r, scorethld=0.5, alignments=False)
        wall = time.perf_counter() - t0
    print("pairs", q.n * r.n, "launches", res.launches, "wall ms %.1f" % (1000 * wall),
          "stage ms (summed over concurrent sub-batches)", [round(x, 1) for x in res.timings_ms.tolist()])


def adjoint_pairs(npairs: int, steps: int, nbase: int = 50_000):
    """Adjoint polishing of `npairs` pairs with fixed 1:1 alignments (lengths
    U(60,600)): a synthetic chain against a rigidly moved copy with 1.5 A
    noise, started from a transform 0.05 rad / 0.5 A off.  `nbase` chains are
    generated on the host and reused with fresh rotations and noise drawn on
    the device.  Prints pairs/s and the TM-score gain distribution."""
    import time
    import numpy as np
    import torch
    from .adjoint import polish
    rng = np.random.default_rng(5)
    lens = rng.integers(60, 601, size=nbase)
    base = synth.random_chains(rng, lens, "a")
    xb = torch.from_numpy(np.concatenate([c.xyz for c in base]).astype(np.float32)).cuda()
    lb = torch.from_numpy(lens.astype(np.int64)).cuda()
    ob = torch.cumsum(lb, 0) - lb
    reps = (npairs + nbase - 1) // nbase
    idx = torch.arange(npairs, device="cuda") % nbase
    n = lb[idx].to(torch.int32)
    off = torch.cumsum(n.long(), 0) - n.long()
    N = int(n.sum())
    pid = torch.repeat_interleave(torch.arange(npairs, device="cuda"), n.long(), output_size=N)
    src = ob[idx][pid] + (torch.arange(N, device="cuda") - off[pid])
    g = torch.Generator(device="cuda").manual_seed(7)
    q = xb[src].contiguous()

    def rotations(m, scale=None):
        a = torch.randn(m, 3, device="cuda", generator=g)
        if scale is not None:
            a = a * scale
        else:
            a = a / a.norm(dim=1, keepdim=True) * (torch.rand(m, 1, device="cuda", generator=g) * 3.14159)
        th = a.norm(dim=1).clamp_min(1e-12)[:, None, None]
        k = a / th[:, :, 0]
        K = torch.zeros(m, 3, 3, device="cuda")
        K[:, 0, 1], K[:, 0, 2], K[:, 1, 0] = -k[:, 2], k[:, 1], k[:, 2]
        K[:, 1, 2], K[:, 2, 0], K[:, 2, 1] = -k[:, 0], -k[:, 1], k[:, 0]
        I = torch.eye(3, device="cuda").expand(m, 3, 3)
        return I + torch.sin(th) * K + (1 - torch.cos(th)) * (K @ K)

    R = rotations(npairs)
    t = torch.randn(npairs, 3, device="cuda", generator=g) * 10
    r = torch.einsum("nij,nj->ni", R[pid], q) + t[pid] + torch.randn(N, 3, device="cuda", generator=g) * 1.5
    R0 = rotations(npairs, scale=0.05) @ R
    t0 = t + torch.randn(npairs, 3, device="cuda", generator=g) * 0.5
    tfm = torch.cat([R0.reshape(npairs, 9), t0], 1).contiguous()
    d0 = (1.24 * torch.clamp(n.float() - 15, min=1).pow(1.0 / 3.0) - 1.8).clamp_min(0.5)
    tfm_w = tfm.clone()
    polish(q, r, off, n, tfm_w, d0, steps)          # warm-up
    torch.cuda.synchronize()
    tfm_w = tfm.clone()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    tb, ta = polish(q, r, off, n, tfm_w, d0, steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    gain = ((ta - tb) / n.float()).cpu().numpy()
    print("pairs", npairs, "residues", N, "steps", steps, "ms %.1f" % ms,
          "pairs/s %.0f" % (npairs / (ms / 1000.0)),
          "TM gain mean %.4f median %.4f max %.4f" % (gain.mean(), np.median(gain), gain.max()),
          "never lower %s" % bool((gain >= 0).all()),
          "raised %.3f" % float((gain > 0).mean()), flush=True)


def long_chains(lengths):
    """One gtb_process_block call per long-chain pair (gtalign defaults,
    --no-detailed-search, -s 0.5): wall time, TM-scores and stage timings."""
    import time
    import numpy as np
    from .shard import subset
    wl = synth.config2(seed=3, lengths=tuple(lengths))
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    with GTalignB200(0, 0, Options()) as g:
        g.process_block(subset(q, np.array([0])), subset(r, np.array([0])), scorethld=0.5,
                        alignments=False)
        for i in range(q.n):
            qi, ri = subset(q, np.array([i])), subset(r, np.array([i]))
            t0 = time.perf_counter()
            res = g.process_block(qi, ri, scorethld=0.5, alignments=False)
            wall = time.perf_counter() - t0
            print("length", lengths[i], "wall ms %.1f" % (1000 * wall),
                  "tm %.4f %.4f rmsd %.3f aligned %d" % (res.alndata[0, 0, 9], res.alndata[0, 0, 10],
                                                        res.alndata[0, 0, 8], res.alndata[0, 0, 4]),
                  "stage ms", [round(x, 1) for x in res.timings_ms.tolist()], flush=True)


if __name__ == "__main__":
    main()
