#!/usr/bin/env python
"""Benchmark: pairs/s of the batched superposition search on B200.

Workload (seeded synthetic; no public dataset): 16 query C-alpha traces
(lengths U(80,800)) against 200,000 reference traces (log-normal lengths,
median 250, sigma_log 0.6, clipped to 30..2000; 5% members of homolog
families), i.e. 3.2M query-reference pairs per step, with gtalign's default
per-pair options except the spatial-index detailed search
(--no-detailed-search; refinement 1, depth 2, convergence 18,
--pre-score 0.4, -s 0.5).

One step = the full stage sequence (seed -> refinement -> DP <-> refinement
loops -> final superposition/production scores) over one query chunk (2
queries, the reference's --dev-queries-per-chunk default) x all 200,000
references; the default 8 timed steps cover the whole 3.2M-pair workload.  `value` is measured with the structure blocks resident in HBM
(gtb_process_resident, results left on the device); `e2e` through the
public call gtb_process_block with pinned host buffers (host->device copy of
the blocks and device->host copy of the per-pair result records inside the
timed region).  Inputs (about 0.6 GB of coordinates and the pair state) are
larger than L2 between steps.

--impl reference times the reference's own CPU implementation (its OpenMP
build compiled from source under oracle/_ref/, or, when that binary is
absent, the oracle port) on this host's cores over a bounded sample of the
same workload.

Multi-GPU (torchrun): pairs are independent; every rank aligns its own
seeded workload of the same size (weak scaling, no data-path collective);
the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# k_findfrag DRAM read + write per pair (ncu, 2 queries x 40,000 references:
# 102.29 MB + 5.99 MB for 13,333 pairs)
FINDFRAG_DRAM_BYTES_PER_PAIR = (102.29e6 + 5.99e6) / 13333

METRIC = "pairs/s on 1 B200 at |dTM|<=1e-4; batched+adjoint vs plain; HBM % of peak"
UNIT = "pairs/s"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during a region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(nq: int, nr: int, seed: int):
    from gtalign_alpha_b200 import synth
    wl = synth.config1(seed=seed, n_queries=nq, n_refs=nr)
    return wl, synth.pack(wl.queries), synth.pack(wl.refs)


# -------------------------------------------------------------------- ours
def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    dev = local
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from gtalign_alpha_b200 import build as gb
    gb.build()
    from gtalign_alpha_b200.api import GTalignB200, Options, pack_fields, load_library
    L = load_library()

    t0 = time.time()
    wl, q, r = make_workload(args.nqueries, args.nrefs, args.seed + 1000 * rank)
    gen_s = time.time() - t0
    npairs = q.n * r.n
    opts = Options()  # gtalign defaults, detailed search off
    g = GTalignB200(dev, 0, opts)
    from gtalign_alpha_b200.shard import subset
    nchunk = (q.n + args.qchunk - 1) // args.qchunk
    qchunks = [subset(q, np.arange(c * args.qchunk, min(q.n, (c + 1) * args.qchunk))) for c in range(nchunk)]
    qbs = [pack_fields(c) for c in qchunks]
    rb = pack_fields(r)

    # resident blocks for `value`
    rblk = ctypes.c_void_p()
    L.gtb_block_upload.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.gtb_block_free.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.gtb_process_resident.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    qblks = [ctypes.c_void_p() for _ in qbs]
    for blk, pk in list(zip(qblks, qbs)) + [(rblk, rb)]:
        st = L.gtb_block_upload(g.handle, pk.beg, pk.end, ctypes.byref(blk))
        if st != 0:
            raise RuntimeError(L.gtb_last_error(g.handle).decode())
    maxpairs = max(c.n for c in qchunks) * r.n
    d_out = torch.empty(maxpairs * 16, dtype=torch.float32, device=dev)
    d_tfm = torch.empty(maxpairs * 12, dtype=torch.float32, device=dev)
    step_pairs = [c.n * r.n for c in qchunks]

    def step_resident(k):
        st = L.gtb_process_resident(g.handle, ctypes.c_float(0.5), qblks[k % nchunk], rblk,
                                    ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_tfm.data_ptr()), None)
        if st != 0:
            raise RuntimeError(L.gtb_last_error(g.handle).decode())
        return int(L.gtb_last_launch_count(g.handle))

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    for k in range(args.warmup):
        step_resident(k)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = 0
    stage_ms = np.zeros(7)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        e0.record()
        done_pairs = 0
        for k in range(args.steps):
            launches += step_resident(k)
            done_pairs += step_pairs[k % nchunk]
            tm = np.zeros(7, np.float32)
            L.gtb_last_timings(g.handle, tm.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
            stage_ms += tm
        e1.record()
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = ws * done_pairs / (ms / 1000.0)

    # e2e through gtb_process_block with pinned host buffers
    pin = {}
    for nm, pk in [("q%d" % c, qb) for c, qb in enumerate(qbs)] + [("r", rb)]:
        arrs = []
        for a in pk.arrays:
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            t.numpy()[:] = a.view(np.uint8).ravel()
            arrs.append(t)
        beg = (ctypes.c_void_p * 10)()
        end = (ctypes.c_void_p * 10)()
        for f, t in enumerate(arrs):
            beg[f] = t.data_ptr()
            end[f] = t.data_ptr() + t.numel()
        pin[nm] = (arrs, beg, end)
    h_out = torch.empty(maxpairs * 16, dtype=torch.float32, pin_memory=True)
    h_tfm = torch.empty(maxpairs * 12, dtype=torch.float32, pin_memory=True)
    from gtalign_alpha_b200.api import _CResults
    res = _CResults(h_out.data_ptr(), h_tfm.data_ptr(), None, None, None, None)

    def step_e2e(k):
        qk = "q%d" % (k % nchunk)
        st = L.gtb_process_block(g.handle, ctypes.c_float(0.5), pin[qk][1], pin[qk][2],
                                 pin["r"][1], pin["r"][2], ctypes.byref(res))
        if st != 0:
            raise RuntimeError(L.gtb_last_error(g.handle).decode())

    step_e2e(0)
    torch.cuda.synchronize()
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    e2e_pairs = 0
    for k in range(args.steps):
        step_e2e(k)
        e2e_pairs += step_pairs[k % nchunk]
    e3.record()
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = ws * e2e_pairs / (ms_e2e / 1000.0)
    h2d = int(np.mean([sum(a.nbytes for a in qb.arrays) for qb in qbs])) + sum(a.nbytes for a in rb.arrays)
    d2h = int(np.mean(step_pairs)) * (16 + 12) * 4

    # the batched form with adjoint polishing of the final transforms
    # (polish_steps=5): the same resident steps, timed the same way, and the
    # score gain against the unpolished outputs of the last step
    adjoint = None
    if args.polish_steps > 0:
        adjoint = adjoint_run(L, dev, qblks, rblk, nchunk, step_pairs, args, maxpairs,
                              d_out, barrier, ws, qchunks, r)

    # the plain form: the same kernels at one pair per call (1 query x 1
    # reference through gtb_process_block with host buffers), on a sample
    plain = plain_sample(g, L, q, r, args.plain_pairs, args.seed) if args.plain_pairs > 0 else None
    if plain is not None:
        plain["batched_vs_plain"] = value / plain["value"]
        if adjoint is not None:
            plain["batched_adjoint_vs_plain"] = adjoint["value"] / plain["value"]

    # roofline of the dominant stage (fraction of the step per stage)
    hbm_peak, peak_kind = peaks()
    st_ms = stage_ms / args.steps
    # algorithmic bytes of the seed (scan) stage: every reference coordinate
    # read once per query block, query coordinates, and a 64-byte record per pair
    # per step (one query chunk): every reference residue once, the chunk's
    # queries, a 64-byte record per pair; the step's seed launches (one per
    # sub-batch) split these bytes, and stage_ms[0] sums their durations
    algo_bytes = 12 * r.total + 12 * q.total / nchunk + 64 * done_pairs / args.steps
    seed_ms = float(st_ms[0])
    achieved = algo_bytes / (seed_ms / 1000.0) / 1e9 if seed_ms > 0 else 0.0
    # DRAM bytes of one seed launch, scaled by pairs from an ncu capture of a
    # smaller case of the same workload (profiles/top_kernels_c1_2x40000.md)
    step_pairs_avg = done_pairs / args.steps
    nsub = max(1, min(6, int(step_pairs_avg) // 16384))
    traffic = FINDFRAG_DRAM_BYTES_PER_PAIR * step_pairs_avg / nsub
    algo_launch = algo_bytes / nsub
    roof = {"bound": "hbm", "kernel": "k_findfrag (stage-1 seed scan)",
            "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "peak_source": peak_kind,
            "traffic": traffic, "traffic_unit": "bytes per launch (scaled from ncu)",
            "algorithmic_bytes_per_launch": algo_launch,
            "stage_ms": {"seed": float(st_ms[0]), "refine_init": float(st_ms[1]),
                         "dp_refine_loops": float(st_ms[2]), "final": float(st_ms[5]),
                         "total": float(st_ms[6])}}

    # CPU baseline sample (rank 0, N=1 only)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(wl, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (f64 rotation solve)", "data": "synthetic (seeded C-alpha traces)",
            "config": {"workload": "16 queries x %d references (log-normal lengths, median 250)" % args.nrefs,
                       "pairs_per_gpu": npairs, "step": "%d queries x %d references" % (args.qchunk, args.nrefs),
                       "options": "gtalign defaults with --no-detailed-search, -s 0.5",
                       "l2": "inputs larger than L2 (%.0f MB of reference coordinates)" % (12 * r.total / 1e6),
                       "parallelism": "dp%d (independent pairs)" % ws},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roof,
            "adjoint": adjoint,
            "plain": plain,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "workload_gen_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    for blk in qblks:
        L.gtb_block_free(g.handle, blk)
    L.gtb_block_free(g.handle, rblk)
    g.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------- reference
def ref_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "gtalign")
    return p if os.path.exists(p) else None


def run_reference_sample(wl, nq: int, nref: int, threads: int):
    """Time the reference CPU build (or the oracle port) on nq queries x nref
    references of the workload.  Returns (pairs, seconds, kind)."""
    from gtalign_alpha_b200 import synth
    binp = ref_binary()
    sub = synth.Workload(wl.queries[:nq], wl.refs[:nref], wl.seed)
    if binp:
        d = tempfile.mkdtemp(prefix="gtref")
        try:
            synth.write_dirs(sub, d + "/q", d + "/r")
            cmd = [binp, "--qrs=" + d + "/q", "--rfs=" + d + "/r", "-o", d + "/out", "--outfmt=1",
                   "--cpu-threads=%d" % threads, "--cpu-threads-reading=1", "--no-detailed-search",
                   "--dev-queries-per-chunk=%d" % max(1, nq)]
            subprocess.run(cmd, capture_output=True, check=True)
            secs = 0.0
            seen = set()
            for f in os.listdir(d + "/out"):
                J = json.load(open(os.path.join(d, "out", f)))["gtalign_search"]
                t = J["search_statistics"]["query_batch_execution_time"]
                if t not in seen:
                    seen.add(t)
                    secs += t
            return nq * nref, secs, "reference"
        finally:
            shutil.rmtree(d, ignore_errors=True)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    q, r = synth.pack(sub.queries), synth.pack(sub.refs)
    t = time.time()
    pyoracle.process_block(q, r, pyoracle.opts_from(refinement=1, convergence=18, prescore=0.4,
                                                    scorethld=0.5), nthreads=threads)
    return nq * nref, time.time() - t, "port"


def adjoint_run(L, dev, qblks, rblk, nchunk, step_pairs, args, maxpairs, d_ref, barrier, ws,
                qchunks, r):
    """pairs/s of the resident steps with polish_steps on, and the score
    gain of the polished transforms over the unpolished ones."""
    import torch
    from gtalign_alpha_b200.api import GTalignB200, Options
    k_last = (args.steps - 1) % nchunk
    ref = d_ref[:step_pairs[k_last] * 16].view(-1, 16).cpu().numpy()
    gp = GTalignB200(dev, 0, Options(polish_steps=args.polish_steps))
    d_out = torch.empty(maxpairs * 16, dtype=torch.float32, device=dev)
    d_tfm = torch.empty(maxpairs * 12, dtype=torch.float32, device=dev)

    def step(k):
        st = L.gtb_process_resident(gp.handle, ctypes.c_float(0.5), qblks[k % nchunk], rblk,
                                    ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_tfm.data_ptr()), None)
        if st != 0:
            raise RuntimeError(L.gtb_last_error(gp.handle).decode())

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    done = 0
    for k in range(args.steps):
        step(k)
        done += step_pairs[k % nchunk]
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    pol = d_out[:step_pairs[k_last] * 16].view(-1, 16).cpu().numpy()
    gp.close()
    # score by the shorter structure's length: the polishing objective
    lq = np.repeat(qchunks[k_last].lens, r.n)
    lr = np.tile(r.lens, qchunks[k_last].n)
    col = np.where(lq <= lr, 9, 10)
    rows = np.arange(len(col))
    ok = ref[:, 9] > 0
    a = ref[rows, col][ok]
    b = pol[rows, col][ok]
    gain = b - a
    return {"value": ws * done / (ms / 1000.0), "unit": UNIT, "polish_steps": args.polish_steps,
            "pairs_reported": int(ok.sum()), "pairs_gained": int((gain > 1e-6).sum()),
            "tm_gain_mean": float(gain.mean()) if ok.any() else 0.0,
            "tm_gain_max": float(gain.max()) if ok.any() else 0.0,
            "never_lower": bool((gain >= -1e-6).all())}


def plain_sample(g, L, q, r, npairs: int, seed: int):
    """pairs/s of one gtb_process_block call per pair on a seeded sample of
    the workload's pairs (blocks packed beforehand; the calls are timed)."""
    import torch
    from gtalign_alpha_b200.api import _CResults, pack_fields
    from gtalign_alpha_b200.shard import subset
    rng = np.random.default_rng(seed + 77)
    qi = rng.integers(0, q.n, npairs)
    ri = rng.integers(0, r.n, npairs)
    blocks = [(pack_fields(subset(q, np.array([a]))), pack_fields(subset(r, np.array([b]))))
              for a, b in zip(qi, ri)]
    out = np.zeros(16, np.float32)
    tfm = np.zeros(12, np.float32)
    res = _CResults(out.ctypes.data, tfm.ctypes.data, None, None, None, None)

    def one(qb, rb):
        st = L.gtb_process_block(g.handle, ctypes.c_float(0.5), qb.beg, qb.end, rb.beg, rb.end,
                                 ctypes.byref(res))
        if st != 0:
            raise RuntimeError(L.gtb_last_error(g.handle).decode())

    for qb, rb in blocks[:3]:
        one(qb, rb)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for qb, rb in blocks:
        one(qb, rb)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    return {"value": npairs / secs, "unit": UNIT,
            "sample": "%d seeded pairs of the workload, one gtb_process_block call (1 query x "
                      "1 reference, host buffers) per pair" % npairs}


def cpu_baseline_sample(wl, args):
    threads = os.cpu_count() or 1
    nref = args.cpu_sample_refs
    pairs, secs, kind = run_reference_sample(wl, 1, nref, threads)
    return {"value": pairs / secs, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": "1 query (L=%d) x %d references of the workload, default options with "
                      "--no-detailed-search; %.1f s" % (wl.queries[0].length, nref, secs)}


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from gtalign_alpha_b200 import synth
    wl = synth.config1(seed=args.seed, n_queries=args.nqueries, n_refs=args.cpu_sample_refs * 2)
    for _ in range(args.warmup):
        run_reference_sample(wl, 1, 50, threads)
    tot_pairs, tot_s, kind = 0, 0.0, "reference"
    for k in range(args.steps):
        qi = k % args.nqueries
        sub = synth.Workload(wl.queries[qi:qi + 1], wl.refs, wl.seed)
        pairs, secs, kind = run_reference_sample(sub, 1, args.cpu_sample_refs, threads)
        tot_pairs += pairs
        tot_s += secs
    v = tot_pairs / tot_s
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded C-alpha traces)",
            "config": {"workload": "16 queries x %d references (log-normal lengths, median 250)" % args.nrefs,
                       "options": "gtalign defaults with --no-detailed-search",
                       "parallelism": "host cores"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": "per step 1 query x %d references of the workload" % args.cpu_sample_refs},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nrefs", type=int, default=200_000)
    ap.add_argument("--nqueries", type=int, default=16)
    ap.add_argument("--qchunk", type=int, default=2, help="queries per step (the reference's --dev-queries-per-chunk)")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-sample-refs", type=int, default=2000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--polish-steps", type=int, default=5,
                    help="adjoint polishing steps of the second timed form (0: skip)")
    ap.add_argument("--plain-pairs", type=int, default=300,
                    help="pairs timed in the one-pair-per-call form (0: skip)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
