#!/usr/bin/env python
"""Benchmark: pairs/s of the batched superposition search on B200.

Workload (seeded synthetic; no public dataset): 16 query C-alpha traces
(lengths U(80,800)) against 200,000 reference traces (log-normal lengths,
median 250, sigma_log 0.6, clipped to 30..2000; 5% members of homolog
families), i.e. 3.2M query-reference pairs, with gtalign's default per-pair
options except the spatial-index detailed search (--no-detailed-search;
refinement 1, depth 2, convergence 18, --pre-score 0.4, -s 0.5).

One step = the full stage sequence (seed -> refinement -> DP <-> refinement
loops -> final superposition/production scores) over one query chunk (2
queries, the reference's --dev-queries-per-chunk default) x all 200,000
references.  Legs of one run:

* autotune (before any timing, --autotune 1): gtb_autotune picks the launch
  shapes (seed offsets per CTA, CTAs per long refinement pair, DP pairs per
  CTA wavefront, pairs per sub-batch) on the first step's block; every
  handle then uses them.  They change no result.
* value (headline): the batched form with adjoint polishing of the final
  transforms (5 projected-gradient steps), structure blocks resident in HBM
  (gtb_process_resident, results left on the device).  The per-pair numeric
  error records (|FP32 path - FP64 recomputation| of both TM-scores and the
  RMSD) of every timed pair are kept and their maxima reported; the run
  fails when a TM-score error exceeds 1e-4 or an RMSD error 1e-3 A.
* unpolished: the same steps without polishing (the reference's results).
* e2e: the public call gtb_process_block with pinned host buffers: the
  host->device copy of the blocks, the device->host copy of the records,
  transforms, numeric errors and alignment rows (the reference's alnsmem
  layout) inside the timed region.
* plain: the same kernels at one pair per call (1 query x 1 reference).
* long_chain: the long-chain configuration (8 assembly pairs of
  5,000-37,860 residues, one call per pair) with alignment rows; the
  reference's GPU build on the 12,000 and 37,860 pairs.
* adjoint: 1,000,000 fixed-alignment pairs (lengths U(60,600)) polished
  with 10 projected-gradient steps of the TM-score adjoint.
* roofline: the HBM roofline of the stage-1 seed scan, and the FP32 SIMT
  roofline of the whole step from device-counted algorithmic work.
* cpu_baseline: the reference's CPU build (oracle/_ref/gtalign, compiled
  from its sources) on this host's cores over a bounded sample of the same
  workload, all 16 queries.
* reference_gpu: the reference's own GPU build (oracle/_ref/gpu/gtalign,
  compiled for sm_100a from its sources by oracle/Makefile.refgpu) on the
  same B200, over the first query chunk x a sample of the references, timed
  by its "query batch execution time" (the GPU bar for this path); and
  from_files: the same sample's files read by this library's reader and
  aligned, wall clock against the reference process's.
* clustering: the all-against-all clustering configuration at 1,000
  structures (config4's generator): the set aligned against itself with the
  clustering run's coverage prefilter, linked by gtb_cluster; the
  reference's GPU build (--cls) on the same structures, wall clock both.
* default_options: gtalign's default options (--speed 9, the spatial-index
  detailed search on) on the same workload, --defaults-steps steps over the
  first query chunks, and the reference's GPU build at those options.
* reader: the host PDB reader (gtb_read_pdb) on the first --reader-files
  references written as files, all host threads.

Inputs (about 0.6 GB of coordinates and the pair state) are larger than L2
between steps.  --impl reference times the reference's own CPU
implementation the same way.

Multi-GPU (torchrun): pairs are independent; the 200,000 references are split
over the ranks by cost (sum Lq*Lr, longest first; shard.ShardPlan) and every
rank aligns each query chunk with its share (strong scaling, no data-path
collective); the timing is the max over ranks; the e2e leg gathers the
records on rank 0 (shard.search_sharded).
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

# k_findfrag DRAM read + write per pair (ncu, one seed launch of the benchmark
# step, 66,667 pairs: profiles/findfrag_dram_c1_2x200000.md)
FINDFRAG_DRAM_BYTES_PER_PAIR = (336.93e6 + 8.44e6) / 66667

METRIC = "pairs/s on 1 B200 at |dTM|<=1e-4; batched+adjoint vs plain; HBM % of peak"
UNIT = "pairs/s"
# algorithmic FP32 work per unit (the per-pass figure of the scoring/covariance
# pass: transform 18, distance 6, TM term 3 incl. one divide, covariance 15 +
# 6 squares; and per DP cell)
FLOPS_PER_VISIT = 48
FLOPS_PER_DP_CELL = 12
NSM_B200 = 148
FP32_LANES_PER_SM = 128
TOL_TM, TOL_RMSD = 1e-4, 1e-3


_T0 = time.time()


def progress(msg: str) -> None:
    """A timestamped line on stderr (the JSON line stays alone on stdout)."""
    print("[bench %7.1fs] %s" % (time.time() - _T0, msg), file=sys.stderr, flush=True)


def lib_options(args, polish: int):
    """The library's options of the run: a --speed preset 0..12 (9 is the
    command line's default, the detailed search on), or 13: the defaults
    with --no-detailed-search; -s 0.5."""
    from gtalign_alpha_b200.api import Options
    if args.speed == 13:
        return Options(polish_steps=polish)      # defaults with --no-detailed-search
    return Options.speed(args.speed, polish_steps=polish)


def cli_options(args):
    """The same options on the reference's command line."""
    return ["--no-detailed-search"] if args.speed == 13 else ["--speed=%d" % args.speed]


def options_text(args) -> str:
    return ("gtalign defaults with --no-detailed-search, -s 0.5" if args.speed == 13
            else "gtalign defaults (--speed %d: the spatial-index detailed search on), -s 0.5" % args.speed)


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


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


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


def _max_over_ranks(x: float, ws: int, dev) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(x: float, ws: int, dev) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# -------------------------------------------------------------------- ours
class Resident:
    """Timed resident steps (gtb_process_resident) of one handle over the
    query chunks x this rank's references, with per-step device buffers for
    the records, transforms and numeric errors of every timed pair."""

    def __init__(self, L, g, qblks, rblk, step_pairs, maxpairs, steps, dev):
        import torch
        self.L, self.g, self.qblks, self.rblk = L, g, qblks, rblk
        self.step_pairs = step_pairs
        self.nchunk = len(qblks)
        nbuf = min(steps, self.nchunk)
        self.out = torch.empty((nbuf, maxpairs * 16), dtype=torch.float32, device=dev)
        self.tfm = torch.empty((nbuf, maxpairs * 12), dtype=torch.float32, device=dev)
        self.err = torch.zeros((nbuf, maxpairs * 4), dtype=torch.float32, device=dev)
        self.maxerr = torch.zeros(3, dtype=torch.float32, device=dev)
        self.nrmsd_over = torch.zeros((), dtype=torch.int64, device=dev)

    def step(self, k):
        import torch
        b = k % self.out.shape[0]
        c = k % self.nchunk
        st = self.L.gtb_process_resident(self.g.handle, ctypes.c_float(0.5), self.qblks[c], self.rblk,
                                         ctypes.c_void_p(self.out[b].data_ptr()),
                                         ctypes.c_void_p(self.tfm[b].data_ptr()),
                                         ctypes.c_void_p(self.err[b].data_ptr()))
        if st != 0:
            raise RuntimeError(self.L.gtb_last_error(self.g.handle).decode())
        n = self.step_pairs[c]
        e = self.err[b, :n * 4].view(n, 4)
        # every timed pair's error, reduced on the device (no host sync)
        torch.maximum(self.maxerr, e[:, :3].amax(dim=0), out=self.maxerr)
        self.nrmsd_over += (e[:, 2] > TOL_RMSD).sum()
        return int(self.L.gtb_last_launch_count(self.g.handle))

    def records(self, k):
        b = k % self.out.shape[0]
        n = self.step_pairs[k % self.nchunk]
        return self.out[b, :n * 16].view(n, 16).cpu().numpy()


def timed_steps(res: Resident, args, ws, dev, barrier, clocks=False, work=False):
    import torch
    for k in range(args.warmup):
        res.step(k)
    res.maxerr.zero_()
    res.nrmsd_over.zero_()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches, done = 0, 0
    stage_ms = np.zeros(7)
    wk = np.zeros(4, np.float64)
    kms = np.zeros(4, np.float64)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = Clocks(dev) if clocks else None
    if clk:
        clk.__enter__()
    e0.record()
    for k in range(args.steps):
        launches += res.step(k)
        done += res.step_pairs[k % res.nchunk]
        tm = np.zeros(7, np.float32)
        res.L.gtb_last_timings(res.g.handle, tm.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        stage_ms += tm
        if work:
            wk += res.g.last_work().astype(np.float64)
            kms += res.g.last_kernel_ms().astype(np.float64)
    e1.record()
    torch.cuda.synchronize()
    if clk:
        clk.__exit__()
    barrier()
    torch.cuda.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), ws, dev)
    allpairs = _sum_over_ranks(done, ws, dev)
    me = res.maxerr.cpu().numpy()
    return {"ms": ms, "pairs": allpairs, "launches": launches, "stage_ms": stage_ms / args.steps,
            "work": wk / args.steps, "kernel_ms": kms / args.steps, "maxerr": [float(x) for x in me],
            "nrmsd_over": int(res.nrmsd_over.item()),
            "clocks": clk.summary() if clk else None}


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
    from gtalign_alpha_b200.api import GTalignB200, Options, pack_fields, load_library, _CResults
    from gtalign_alpha_b200.shard import ShardPlan, subset, search_sharded
    L = load_library()

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    t0 = time.time()
    progress("generating the workload")
    wl, q, r_all = make_workload(args.nqueries, args.nrefs, args.seed)
    plan = ShardPlan(r_all, q.lens, rank, ws)
    r = plan.refs
    gen_s = time.time() - t0
    nchunk = (q.n + args.qchunk - 1) // args.qchunk
    qchunks = [subset(q, np.arange(c * args.qchunk, min(q.n, (c + 1) * args.qchunk))) for c in range(nchunk)]
    qbs = [pack_fields(c) for c in qchunks]
    rb = pack_fields(r)
    gp = GTalignB200(dev, 0, lib_options(args, args.polish_steps))
    g0 = GTalignB200(dev, 0, lib_options(args, 0))

    # resident blocks (uploaded once, used by both handles on this device)
    L.gtb_block_upload.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.gtb_block_free.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.gtb_process_resident.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    rblk = ctypes.c_void_p()
    qblks = [ctypes.c_void_p() for _ in qbs]
    for blk, pk in list(zip(qblks, qbs)) + [(rblk, rb)]:
        st = L.gtb_block_upload(gp.handle, pk.beg, pk.end, ctypes.byref(blk))
        if st != 0:
            raise RuntimeError(L.gtb_last_error(gp.handle).decode())
    step_pairs = [c.n * r.n for c in qchunks]
    maxpairs = max(step_pairs)
    legs = set(args.legs.split(","))

    # launch shapes picked by the library's autotuner on the first step's
    # block (outside the timed region), then used by every handle
    tuning = None
    if args.autotune:
        progress("autotune (launch shapes, on the first step's block)")
        t0 = time.time()
        best, tms, tried = gp.autotune(qblks[0], rblk, scorethld=0.5, trials=1)
        g0.set_tuning(best)
        tuning = {"picked": best.as_dict(), "ms_per_call": tms, "s": time.time() - t0,
                  "tried": [dict(t, ms=round(m, 2)) for t, m in tried]}

    # headline: batched + adjoint polishing, resident
    progress("headline (batched + adjoint, resident)")
    rp = Resident(L, gp, qblks, rblk, step_pairs, maxpairs, args.steps, dev)
    gp.set_kernel_timing(True)          # per-family device time for the FP32 roofline
    A = timed_steps(rp, args, ws, dev, barrier, clocks=True, work=True)
    gp.set_kernel_timing(False)
    value = A["pairs"] / (A["ms"] / 1000.0)
    ms_step = A["ms"] / args.steps
    # the metric's qualifier: every timed pair's TM-scores within TOL_TM of
    # the FP64 recomputation.  The RMSD is the reference's FP32 value (from
    # sums of squares, bit-identical to the oracle); its error against FP64
    # is reported, not gated.
    acc_ok = A["maxerr"][0] <= TOL_TM and A["maxerr"][1] <= TOL_TM

    # the unpolished form (the reference's results) and the polishing gain
    unpol = None
    if "unpolished" in legs:
        progress("unpolished")
        r0 = Resident(L, g0, qblks, rblk, step_pairs, maxpairs, args.steps, dev)
        B = timed_steps(r0, args, ws, dev, barrier)
        ok0 = B["maxerr"][0] <= TOL_TM and B["maxerr"][1] <= TOL_TM
        acc_ok = acc_ok and ok0
        k_last = args.steps - 1
        a, b = r0.records(k_last), rp.records(k_last)
        c = qchunks[k_last % nchunk]
        lq, lr = np.repeat(c.lens, r.n), np.tile(r.lens, c.n)
        col = np.where(lq <= lr, 9, 10)          # polishing objective: d0 of the shorter length
        rows = np.arange(len(col))
        rep = a[:, 9] > 0
        gain = b[rows, col][rep] - a[rows, col][rep]
        unpol = {"value": B["pairs"] / (B["ms"] / 1000.0), "unit": UNIT, "ms_per_step": B["ms"] / args.steps,
                 "max_err_tm": max(B["maxerr"][:2]), "max_err_rmsd": B["maxerr"][2],
                 "polish_gain_last_step": {
                     "pairs_reported": int(rep.sum()), "pairs_gained": int((gain > 1e-6).sum()),
                     "tm_gain_mean": float(gain.mean()) if rep.any() else 0.0,
                     "tm_gain_max": float(gain.max()) if rep.any() else 0.0,
                     "never_lower": bool((gain >= -1e-6).all())}}

    # e2e through gtb_process_block (host buffers), polished form
    e2e = None
    if "e2e" in legs:
        progress("e2e")
        e2e = e2e_run(L, gp, qbs, rb, qchunks, r, step_pairs, maxpairs, args, ws, rank, dev, barrier,
                      q, r_all, plan)

    # the plain form: one pair per call
    plain = None
    if "plain" in legs and args.plain_pairs > 0 and rank == 0:
        progress("plain")
        plain = plain_sample(gp, L, q, r, args.plain_pairs, args.seed)
        plain["batched_adjoint_vs_plain"] = value / ws / plain["value"]
        if unpol is not None:
            plain["batched_vs_plain"] = unpol["value"] / ws / plain["value"]

    # rooflines
    hbm_peak, peak_kind = peaks()
    st_ms = A["stage_ms"]
    # HBM roofline of the stage-1 seed scan: per step every reference residue
    # once (12 B), the chunk's queries, a 64-byte record per pair; the step's
    # seed launches (one per sub-batch) split these bytes and stage_ms[0]
    # sums their durations
    step_pairs_avg = A["pairs"] / ws / args.steps
    algo_bytes = 12 * r.total + 12 * q.total / nchunk + 64 * step_pairs_avg
    seed_ms = float(st_ms[0])
    achieved = algo_bytes / (seed_ms / 1000.0) / 1e9 if seed_ms > 0 else 0.0
    sub_pairs = tuning["picked"]["sub_pairs"] if tuning else 16384
    nsub = max(1, min(6, int(step_pairs_avg) // sub_pairs))
    traffic = FINDFRAG_DRAM_BYTES_PER_PAIR * step_pairs_avg / nsub
    clocks = A["clocks"]
    sm_mhz = clocks["sm_mhz"] if clocks else 1965.0
    fp32_peak = NSM_B200 * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
    wk, kms = A["work"], A["kernel_ms"]
    fl = {"seed": FLOPS_PER_VISIT * wk[0], "refine": FLOPS_PER_VISIT * wk[1],
          "dp": FLOPS_PER_DP_CELL * (wk[2] + wk[3])}
    fl_step = sum(fl.values())
    fp32_ach = fl_step / (ms_step / 1000.0) / 1e12
    # per kernel family: its algorithmic flops over its summed launch
    # durations (CUDA events on the launching streams; the detailed search's
    # slot-score DP cells are timed with its own kernels)
    fam = {"k_findfrag (seed)": (FLOPS_PER_VISIT * wk[0], kms[0]),
           "k_refine (refinement passes)": (FLOPS_PER_VISIT * wk[1], kms[1]),
           "k_dp / k_dp_wave (DP)": (FLOPS_PER_DP_CELL * wk[2], kms[2])}
    per_kernel = {}
    for name, (f, t) in fam.items():
        a = f / (t / 1000.0) / 1e12 if t > 0 else 0.0
        per_kernel[name] = {"flops_per_step": f, "ms_per_step": t, "achieved": a,
                            "frac": a / fp32_peak}
    if kms[3] > 0:
        # the detailed search's own kernels (local SS alignment, configuration
        # search, slot scores): time only, their work is not a FP32 count
        per_kernel["k_f3_* (detailed search)"] = {"ms_per_step": kms[3],
                                                  "slot_score_dp_cells": wk[3]}
    roof = {"bound": "hbm", "kernel": "k_findfrag (stage-1 seed scan)",
            "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": traffic, "traffic_unit": "bytes per launch (ncu, one seed launch of the bench step)",
            "algorithmic_bytes_per_launch": algo_bytes / nsub,
            "fp32": {"bound": "fp32 SIMT", "achieved": fp32_ach, "unit": "TFLOP/s",
                     "peak": fp32_peak, "frac": fp32_ach / fp32_peak,
                     "peak_source": "148 SMs x 128 FP32 lanes x 2 (FMA) x %.0f MHz (median SM clock "
                                    "sampled during the timed steps)" % sm_mhz,
                     "scope": "whole step (every kernel), per-step algorithmic flops / ms_per_step",
                     "per_kernel": per_kernel,
                     "per_kernel_note": "summed launch durations of concurrent sub-batch streams "
                                        "overlap, so these fractions are lower bounds",
                     "flops_per_step": fl_step,
                     "flops_per_step_by_kernel": fl,
                     "units_per_step": {"seed_position_visits": wk[0], "refine_position_visits": wk[1],
                                        "dp_cells": wk[2], "detailed_search_dp_cells": wk[3]},
                     "flops_per_unit": {"position_visit": FLOPS_PER_VISIT, "dp_cell": FLOPS_PER_DP_CELL}},
            "stage_ms": {"seed": float(st_ms[0]), "refine_init": float(st_ms[1]),
                         "dp_refine_loops": float(st_ms[2]), "final": float(st_ms[5]),
                         "total": float(st_ms[6])}}

    long_chain = adjoint = cpu = refgpu = clustering = defaults = reader = None
    if rank == 0 and ws == 1:
        if "reader" in legs:
            progress("host reader")
            try:
                reader = reader_run(wl, args, r_all)
            except Exception as e:                   # a host-side leg must not lose the line
                reader = {"unavailable": "%s: %s" % (type(e).__name__, str(e)[:200])}
        if "refgpu" in legs:
            progress("reference GPU build")
            refgpu = reference_gpu_sample(wl, args, value)
        if "defaults" in legs and args.speed == 13:
            progress("default options (--speed 9)")
            defaults = defaults_run(L, args, wl, qbs, rb, step_pairs, maxpairs, dev, legs)
        if "cluster" in legs:
            progress("clustering run")
            clustering = cluster_run(args)
        if "long" in legs:
            progress("long chains")
            long_chain = long_chain_run(gp, args)
        if "adjoint" in legs:
            progress("adjoint polishing")
            adjoint = adjoint_pairs(args.adjoint_pairs, args.adjoint_steps)
        if "cpu" in legs:
            progress("reference CPU build sample")
            cpu = cpu_baseline_sample(wl, args)
        progress("done")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak",
            "vs_baseline": None,
            "dtype": "f32 (f64 rotation solve)", "data": "synthetic (seeded C-alpha traces)",
            "config": {"workload": "16 queries x %d references (log-normal lengths, median 250)" % args.nrefs,
                       "pairs": q.n * r_all.n,
                       "step": "%d queries x %d references%s" % (args.qchunk, args.nrefs,
                                                                 " (split over the ranks)" if ws > 1 else ""),
                       "form": "batched + adjoint polishing (%d steps)" % args.polish_steps,
                       "options": options_text(args),
                       "l2": "inputs larger than L2 (%.0f MB of reference coordinates)" % (12 * r_all.total / 1e6),
                       "parallelism": "dp%d (references split by cost, independent pairs)" % ws,
                       "launch_shapes": tuning["picked"] if tuning else "defaults (--autotune 0)"},
            "autotune": tuning,
            "accuracy": {"max_err_tm": max(A["maxerr"][:2]), "max_err_rmsd": A["maxerr"][2],
                         "tolerance_tm": TOL_TM, "ok": bool(acc_ok),
                         "pairs_rmsd_err_over_1e-3": A["nrmsd_over"],
                         "pairs_timed": A["pairs"],
                         "scope": "every timed pair: |FP32 search path - FP64 recomputation|; "
                                  "gated on the TM-scores (the metric's |dTM|<=1e-4); the RMSD "
                                  "is the reference's FP32 sums-of-squares value, its FP64 error "
                                  "reported"},
            "e2e": e2e,
            "gpu_launches": A["launches"],
            "roofline": roof,
            "unpolished": unpol,
            "plain": plain,
            "long_chain": long_chain,
            "adjoint": adjoint,
            "cpu_baseline": cpu,
            "reference_gpu": refgpu,
            "default_options": defaults,
            "reader": reader,
            "clustering": clustering,
            "clocks": clocks,
            "workload_gen_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    for blk in qblks:
        L.gtb_block_free(gp.handle, blk)
    L.gtb_block_free(gp.handle, rblk)
    gp.close()
    g0.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if not acc_ok:
        sys.exit(3)


def e2e_run(L, g, qbs, rb, qchunks, r, step_pairs, maxpairs, args, ws, rank, dev, barrier, q, r_all, plan):
    """Steps through gtb_process_block with pinned host inputs and outputs,
    alignment rows included; at N > 1 through shard.search_sharded (records
    gathered on rank 0 every step)."""
    import torch
    from gtalign_alpha_b200.api import _CResults
    from gtalign_alpha_b200.shard import search_sharded
    nchunk = len(qbs)
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
    # with the detailed search the reader's index trees travel with the blocks
    # (made once, as the reader makes them with the blocks)
    ndx = {}
    if args.speed != 13:
        from gtalign_alpha_b200.api import build_index
        for nm, soa in [("q%d" % c, qc) for c, qc in enumerate(qchunks)] + [("r", r)]:
            arrs = []
            for a in build_index(soa):
                t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
                t.numpy()[:] = a.view(np.uint8).ravel()
                arrs.append(t)
            ndx[nm] = (arrs, (ctypes.c_void_p * 6)(*[t.data_ptr() for t in arrs]))
    h_out = torch.empty(maxpairs * 16, dtype=torch.float32, pin_memory=True)
    h_tfm = torch.empty(maxpairs * 12, dtype=torch.float32, pin_memory=True)
    h_err = torch.empty(maxpairs * 4, dtype=torch.float32, pin_memory=True)
    asz = max(int(L.gtb_alns_size(pin["q%d" % c][1], pin["q%d" % c][2], pin["r"][1], pin["r"][2]))
              for c in range(nchunk))
    h_alns = np.empty(asz, np.uint8)
    res = _CResults(h_out.data_ptr(), h_tfm.data_ptr(), h_alns.ctypes.data, h_err.data_ptr(), None, None)
    d2h_rows = []
    maxerr = np.zeros(3)

    def process(k):
        qk = "q%d" % (k % nchunk)
        if ndx:
            st = L.gtb_process_block_ndx(g.handle, ctypes.c_float(0.5), pin[qk][1], pin[qk][2],
                                         ndx[qk][1], pin["r"][1], pin["r"][2], ndx["r"][1],
                                         ctypes.byref(res))
        else:
            st = L.gtb_process_block(g.handle, ctypes.c_float(0.5), pin[qk][1], pin[qk][2],
                                     pin["r"][1], pin["r"][2], ctypes.byref(res))
        if st != 0:
            raise RuntimeError(L.gtb_last_error(g.handle).decode())
        n = step_pairs[k % nchunk]
        rec = h_out[:n * 16].numpy().reshape(n, 16)
        # bytes of the alignment rows the call copied: 5 rows of (columns + 1)
        # per reported pair, and an 8-byte offset per pair
        alen = rec[:, 4]
        d2h_rows.append(int((5 * (alen[alen > 0] + 1)).sum()) + 8 * n)
        e = h_err[:n * 4].numpy().reshape(n, 4)[:, :3].max(axis=0)
        np.maximum(maxerr, e, out=maxerr)
        return rec

    def one_step(k):
        if ws == 1:
            return process(k)
        fn = lambda qs, rs: (process(k).reshape(qs.n, rs.n, 16), h_tfm[:qs.n * rs.n * 12].numpy().reshape(qs.n, rs.n, 12))
        return search_sharded(qchunks[k % nchunk], r_all, fn, rank, ws, plan=plan)

    for k in range(max(1, args.warmup)):
        one_step(k)
    torch.cuda.synchronize()
    barrier()
    d2h_rows.clear()
    maxerr[:] = 0
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    done = 0
    for k in range(args.steps):
        one_step(k)
        done += step_pairs[k % nchunk]
    e3.record()
    torch.cuda.synchronize()
    ms = _max_over_ranks(e2.elapsed_time(e3), ws, dev)
    allpairs = _sum_over_ranks(done, ws, dev)
    h2d = int(np.mean([sum(a.nbytes for a in qb.arrays) for qb in qbs])) + sum(a.nbytes for a in rb.arrays)
    if ndx:
        h2d += int(np.mean([sum(t.numel() for t in ndx["q%d" % c][0]) for c in range(nchunk)]))
        h2d += sum(t.numel() for t in ndx["r"][0])
    d2h = int(np.mean(step_pairs)) * (16 + 12 + 4) * 4 + int(np.mean(d2h_rows))
    return {"value": allpairs / (ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms / args.steps,
            "max_err_tm": float(max(maxerr[:2])), "max_err_rmsd": float(maxerr[2]),
            "includes": "H2D of both blocks; D2H of records, transforms, numeric errors and "
                        "alignment rows (reference layout); polished form"}


def long_chain_run(g, args):
    """The long-chain configuration: 8 assembly pairs (5,000-37,860 residues),
    one gtb_process_block call per pair with alignment rows; wall time per
    pair (host clock around the call, which includes its copies)."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.shard import subset
    lengths = tuple(int(x) for x in args.long_lengths.split(","))
    wl = synth.config2(seed=3, lengths=lengths)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    warm = synth.config2(seed=4, lengths=(2000,))
    g.process_block(synth.pack(warm.queries), synth.pack(warm.refs), scorethld=0.5)
    per = []
    tot = 0.0
    g.set_kernel_timing(True)       # the per-family split of each pair's device time
    for i in range(q.n):
        qi, ri = subset(q, np.array([i])), subset(r, np.array([i]))
        t0 = time.perf_counter()
        res = g.process_block(qi, ri, scorethld=0.5, alignments=True)
        wall = time.perf_counter() - t0
        tot += wall
        rec = res.alndata[0, 0]
        kms = g.last_kernel_ms()
        per.append({"length": int(lengths[i]), "wall_s": wall, "tm_q": float(rec[9]), "tm_r": float(rec[10]),
                    "rmsd": float(rec[8]), "aligned": int(rec[4]),
                    "err_tm": float(res.numerr[0, 0, :2].max()), "err_rmsd": float(res.numerr[0, 0, 2]),
                    "kernel_ms": {"seed": float(kms[0]), "refine": float(kms[1]), "dp": float(kms[2])}})
    g.set_kernel_timing(False)
    out = {"value": q.n / tot, "unit": "pairs/s", "total_s": tot, "pairs": per,
           "form": "batched + adjoint polishing (%d steps), alignment rows" % args.polish_steps,
           "published_reference": "GTalign on a T4: 65.12 s for a 37,860-residue pair (other "
                                  "structures, other GPU; not comparable as a ratio)"}
    if "refgpu" in args.legs.split(",") and args.long_refgpu_lengths:
        progress("reference GPU build on long chains")
        pick = {int(x) for x in args.long_refgpu_lengths.split(",")}
        out["reference_gpu"] = []
        for i in range(q.n):
            if lengths[i] not in pick:
                continue
            try:
                out["reference_gpu"].append(long_chain_reference_gpu(wl.queries[i], wl.refs[i], per[i], args))
            except Exception as e:                   # a comparison must not lose the line
                out["reference_gpu"].append({"length": int(lengths[i]),
                                             "unavailable": "%s: %s" % (type(e).__name__, str(e)[:200])})
    return out


def long_chain_reference_gpu(qc, rc, ours, args):
    """The reference's GPU build on one long pair (the same structures as PDB
    files; --dev-max-length and --dev-queries-total-length-per-chunk raised
    to the pair's length so that it is not skipped): its query batch
    execution time and wall time against this library's wall time for the
    pair (which includes the host copies and alignment rows)."""
    from gtalign_alpha_b200 import synth
    binp = os.path.join(ROOT, "oracle", "_ref", "gpu", "gtalign")
    if not os.path.exists(binp):
        return {"unavailable": "oracle/_ref/gpu/gtalign not built (make -f oracle/Makefile.refgpu)"}
    L = max(qc.length, rc.length)
    d = tempfile.mkdtemp(prefix="gtreflong")
    try:
        qf, rf = os.path.join(d, "q.pdb"), os.path.join(d, "r.pdb")
        synth.write_pdb(qc, qf)
        synth.write_pdb(rc, rf)
        cmd = [binp, "--qrs=" + qf, "--rfs=" + rf, "-o", d + "/out", "--outfmt=1", "--dev-N=1",
               "--dev-max-length=%d" % L, "--dev-queries-total-length-per-chunk=%d" % L,
               "-s", "0"] + cli_options(args)
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, timeout=args.refgpu_timeout)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return {"length": ours["length"],
                    "unavailable": "reference GPU build exited %d: %s" % (p.returncode, p.stderr.decode()[-300:])}
        secs, tmq = 0.0, None
        for f in os.listdir(d + "/out"):
            J = json.load(open(os.path.join(d, "out", f)))["gtalign_search"]
            secs += J["search_statistics"]["query_batch_execution_time"]
            for h in J["search_results"]:
                tmq = float(h["hit_record"]["alignment"]["tmscore_query"])
        if tmq is None:
            return {"length": ours["length"], "wall_s": wall,
                    "unavailable": "no alignment reported (stderr: %s)" % p.stderr.decode()[-300:]}
        return {"length": ours["length"], "wall_s": wall, "batch_s": secs, "tm_q": tmq,
                "ours_wall_s": ours["wall_s"], "ours_tm_q": ours["tm_q"],
                "reference_batch_over_ours_wall": secs / ours["wall_s"] if ours["wall_s"] > 0 else None}
    except subprocess.TimeoutExpired:
        return {"length": ours["length"],
                "unavailable": "reference GPU build did not finish within %d s" % args.refgpu_timeout}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def adjoint_pairs(npairs: int, steps: int, nbase: int = 50_000):
    """Adjoint polishing of `npairs` pairs with fixed 1:1 alignments (lengths
    U(60,600)): a synthetic chain against a rigidly moved copy with 1.5 A
    noise, started from a transform 0.05 rad / 0.5 A off.  `nbase` chains are
    generated on the host and reused with fresh rotations and noise drawn on
    the device.  Returns pairs/s and the TM-score gain distribution."""
    import torch
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.adjoint import polish
    rng = np.random.default_rng(5)
    lens = rng.integers(60, 601, size=nbase)
    base = synth.random_chains(rng, lens, "a")
    xb = torch.from_numpy(np.concatenate([c.xyz for c in base]).astype(np.float32)).cuda()
    lb = torch.from_numpy(lens.astype(np.int64)).cuda()
    ob = torch.cumsum(lb, 0) - lb
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
    for _ in range(3):
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
    return {"value": npairs / (ms / 1000.0), "unit": "pairs/s", "pairs": npairs, "residues": N,
            "steps": steps, "ms": ms,
            "tm_gain_mean": float(gain.mean()), "tm_gain_median": float(np.median(gain)),
            "tm_gain_max": float(gain.max()), "never_lower": bool((gain >= 0).all()),
            "raised_frac": float((gain > 0).mean()),
            "workload": "fixed 1:1 alignments, lengths U(60,600), started 0.05 rad / 0.5 A off"}


# ---------------------------------------------------------------- reference
def ref_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "gtalign")
    return p if os.path.exists(p) else None


# Runs of the reference CPU build that stalled (every thread waiting on a
# futex, no progress: an intermittent deadlock of its worker threads, seen on
# about one call in six with 8 threads and 250 references) and were restarted.
REF_STALLS = {"stalled": 0, "calls": 0}
REF_CALL_LIMIT_S = 20          # a call of the samples here takes a few seconds


def run_reference_sample(wl, nq: int, nref: int, threads: int, args):
    """Time the reference CPU build (or the oracle port) on the first nq
    queries x nref references of the workload.  Returns (pairs, seconds, kind).
    The time is the build's own "query batch execution time"; a call that
    stalls is killed after REF_CALL_LIMIT_S and run again (REF_STALLS)."""
    from gtalign_alpha_b200 import synth
    binp = ref_binary()
    sub = synth.Workload(wl.queries[:nq], wl.refs[:nref], wl.seed)
    if binp:
        d = tempfile.mkdtemp(prefix="gtref")
        try:
            synth.write_dirs(sub, d + "/q", d + "/r")
            cmd = [binp, "--qrs=" + d + "/q", "--rfs=" + d + "/r", "-o", d + "/out", "--outfmt=1",
                   "--cpu-threads=%d" % threads, "--cpu-threads-reading=1",
                   "--dev-queries-per-chunk=%d" % max(1, nq)] + cli_options(args)
            for attempt in range(5):
                REF_STALLS["calls"] += 1
                shutil.rmtree(d + "/out", ignore_errors=True)
                try:
                    subprocess.run(cmd, capture_output=True, check=True, timeout=REF_CALL_LIMIT_S)
                    break
                except subprocess.TimeoutExpired:
                    REF_STALLS["stalled"] += 1
                    progress("reference CPU build stalled; run again (%d)" % REF_STALLS["stalled"])
            else:
                raise RuntimeError("the reference CPU build stalled 5 times in a row")
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
    ndx = {}
    if args.speed != 13:
        from gtalign_alpha_b200.api import build_index
        ndx = dict(qndx=build_index(q), rndx=build_index(r))
    lo = lib_options(args, 0)
    pyoracle.process_block(q, r, pyoracle.opts_from(refinement=lo.refinement, convergence=lo.convergence,
                                                    prescore=lo.prescore, scorethld=0.5, depth=lo.depth,
                                                    addsearchbyss=lo.addsearchbyss,
                                                    nodetailedsearch=lo.nodetailedsearch,
                                                    trigger=lo.trigger, nbranches=lo.nbranches),
                           nthreads=threads, **ndx)
    return nq * nref, time.time() - t, "port"


def cluster_run(args):
    """The all-against-all clustering configuration at a bounded size: the
    set of config4 (args.cluster_n structures, log-normal lengths, 30% in
    families of 10) aligned against itself in query blocks with the
    clustering run's coverage prefilter, at --speed 13 as the reference
    recommends for clustering, then linked (complete linkage, TM-score 0.5)
    by gtb_cluster; and the reference's GPU build on the same structures
    (--cls over the file list).  Times are wall clock of the whole run
    (device work, transfers, linkage; for the reference also its reading)."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import GTalignB200, Options, cluster
    wl = synth.config4(seed=4, n=args.cluster_n)
    chains = wl.queries
    n = len(chains)
    allsoa = synth.pack(chains)
    types = np.arange(n, dtype=np.int32)
    rec = np.zeros((n, n, 16), np.float32)
    qblock = 64
    with GTalignB200(0, 0, Options.speed(13, clsfilter=1, clscoverage=0.7)) as g:
        # warm-up on the first block (allocations, kernel load)
        g.process_block(synth.pack(chains[:qblock]), allsoa, scorethld=0.5, alignments=False,
                        numerr=False, qtypes=types[:qblock], rtypes=types)
        t0 = time.perf_counter()
        reported = 0
        for q0 in range(0, n, qblock):
            q1 = min(n, q0 + qblock)
            res = g.process_block(synth.pack(chains[q0:q1]), allsoa, scorethld=0.5, alignments=False,
                                  numerr=False, qtypes=types[q0:q1], rtypes=types)
            rec[q0:q1] = res.alndata
            reported += int((res.alndata[..., 4] > 0).sum())
        t1 = time.perf_counter()
    cl = cluster(rec, allsoa.lens, ids=[c.name for c in chains], linkage=0, threshold=0.5, coverage=0.7)
    t2 = time.perf_counter()
    ours = [frozenset(chains[k].name for k in c) for c in cl.clusters]
    out = {"value": n * n / (t2 - t0), "unit": "candidate pairs/s",
           "structures": n, "pairs_reported": reported, "align_s": t1 - t0, "link_s": t2 - t1,
           "clusters": len(ours),
           "workload": "config4: %d structures, log-normal lengths (median 220), 30%% in families of 10; "
                       "--speed 13, --cls-threshold 0.5, complete linkage, coverage 0.7" % n}
    binp = os.path.join(ROOT, "oracle", "_ref", "gpu", "gtalign")
    if not os.path.exists(binp):
        out["reference_gpu"] = {"unavailable": "oracle/_ref/gpu/gtalign not built"}
        return out
    d = tempfile.mkdtemp(prefix="gtclsb")
    try:
        files = []
        for c in chains:
            files.append(os.path.join(d, c.name + ".pdb"))
            synth.write_pdb(c, files[-1])
        cmd = [binp, "--cls=" + ",".join(files), "-o", os.path.join(d, "o"), "--speed=13", "--dev-N=1",
               "--cls-threshold=0.5", "--cls-algorithm=0"]
        t = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, timeout=args.refgpu_timeout)
        wall = time.perf_counter() - t
        if p.returncode != 0:
            out["reference_gpu"] = {"unavailable": "reference --cls run failed (rc %d)" % p.returncode}
            return out
        text = open(os.path.join(d, "o", "gtalignclusters.lst")).read().splitlines()
        last = max(k for k, ln in enumerate(text) if ln.startswith("===="))
        ref = []
        for ln in text[last + 1:]:
            names = [w.split("_")[0] for w in ln.split() if w.startswith("s")]
            if names:
                ref.append(frozenset(names))
        same = sum(len(c) for c in set(ours) & set(ref))
        out["reference_gpu"] = {"wall_s": wall, "value": n * n / wall, "unit": "candidate pairs/s",
                                "clusters": len(ref), "structures_in_identical_clusters": same,
                                "ours_vs_reference_gpu": (n * n / (t2 - t0)) / (n * n / wall)}
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def reader_run(wl, args, r_all):
    """The host reader (gtb_read_pdb): the first --reader-files references
    of the workload written as PDB files, then read back on every host
    thread (the files just written, so from the page cache); files,
    residues and bytes per second, and the time the whole reference set
    would take at that rate."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import read_pdb
    nf = min(args.reader_files, len(wl.refs))
    d = tempfile.mkdtemp(prefix="gtreader")
    try:
        paths = []
        for i in range(nf):
            paths.append(os.path.join(d, "r%06d.pdb" % i))
            synth.write_pdb(wl.refs[i], paths[-1])
        nbytes = sum(os.path.getsize(p) for p in paths)
        read_pdb(paths[:64])                                  # library and threads warm
        t0 = time.perf_counter()
        rb = read_pdb(paths, threads=0)
        dt = time.perf_counter() - t0
        ok = rb.soa.n == nf and int(rb.soa.total) == int(sum(c.length for c in wl.refs[:nf]))
        return {"value": nf / dt, "unit": "files/s", "residues_per_s": rb.soa.total / dt,
                "mb_per_s": nbytes / dt / 1e6, "threads": os.cpu_count(), "files": nf,
                "all_structures_read": bool(ok),
                "reference_set_s_at_this_rate": r_all.n / (nf / dt),
                "sample": "the first %d references of the workload as PDB files (%.0f MB), "
                          "page cache warm" % (nf, nbytes / 1e6)}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def defaults_run(L, args, wl, qbs, rb, step_pairs, maxpairs, dev, legs):
    """gtalign's default options (--speed 9: the spatial-index detailed search
    on) on the headline workload, one GPU: a handle of its own (the blocks
    uploaded again, with their index trees), one warm-up step, then
    --defaults-steps resident polished steps over the first query chunks,
    every timed pair's TM-score error checked; and the reference's GPU build
    at the same options on its sample."""
    import copy
    from gtalign_alpha_b200.api import GTalignB200
    a9 = copy.copy(args)
    a9.speed, a9.steps, a9.warmup = 9, args.defaults_steps, 1
    g9 = GTalignB200(dev, 0, lib_options(a9, args.polish_steps))
    blks = []
    try:
        t0 = time.time()
        for pk in list(qbs) + [rb]:
            blk = ctypes.c_void_p()
            st = L.gtb_block_upload(g9.handle, pk.beg, pk.end, ctypes.byref(blk))
            if st != 0:
                raise RuntimeError(L.gtb_last_error(g9.handle).decode())
            blks.append(blk)
        upload_s = time.time() - t0
        res = Resident(L, g9, blks[:-1], blks[-1], step_pairs, maxpairs, a9.steps, dev)
        D = timed_steps(res, a9, 1, dev, lambda: None)
        v = D["pairs"] / (D["ms"] / 1000.0)
        out = {"value": v, "unit": UNIT, "ms_per_step": D["ms"] / a9.steps, "steps": a9.steps,
               "options": options_text(a9), "form": "batched + adjoint polishing (%d steps), resident"
               % args.polish_steps, "max_err_tm": max(D["maxerr"][:2]),
               "ok": bool(max(D["maxerr"][:2]) <= TOL_TM),
               "upload_and_index_s": upload_s,
               "note": "the first query chunks only (they hold the longest queries); the "
                       "headline's 8 steps cover all 16"}
        if "refgpu" in legs:
            progress("reference GPU build at the default options")
            out["reference_gpu"] = reference_gpu_sample(wl, a9, v)
        return out
    finally:
        for blk in blks:
            L.gtb_block_free(g9.handle, blk)
        g9.close()


def from_files_run(d, args, ref_wall):
    """The reference GPU build's sample the way a user runs it, from the
    structure files to the results, this library's way: the host reader
    (gtb_read_pdb) on the same query and reference files, then one
    gtb_process_block call with alignment rows (the reference's results,
    unpolished; no output files written).  Host wall time from the first
    file read to the results in host memory; the handle is created before."""
    import glob
    from gtalign_alpha_b200.api import GTalignB200, read_pdb
    try:
        qf = sorted(glob.glob(os.path.join(d, "q", "*.pdb")))
        rf = sorted(glob.glob(os.path.join(d, "r", "*.pdb")))
        with GTalignB200(0, 0, lib_options(args, 0)) as g:
            read_pdb(qf)                                   # the reader's first call
            t0 = time.perf_counter()
            q = read_pdb(qf, maxlen=65535)
            r = read_pdb(rf, maxlen=65535)
            res = g.process_packed(q.packed, r.packed, scorethld=0.5, alignments=True)
            wall = time.perf_counter() - t0
        return {"wall_s": wall, "pairs": q.soa.n * r.soa.n, "reported": int((res.alndata[..., 9] > 0).sum()),
                "reference_wall_s": ref_wall, "reference_wall_over_ours": ref_wall / wall,
                "scope": "ours: read the files, align, results and alignment rows in host memory; "
                         "reference: its whole process (reading, device setup, search, JSON output)"}
    except Exception as e:                                 # a missing piece must not lose the line
        return {"unavailable": "%s: %s" % (type(e).__name__, str(e)[:200])}


def reference_gpu_sample(wl, args, value):
    """The reference's GPU build on this device: the first query chunk (2
    queries) x the first refgpu_refs references of the workload, default
    options with --no-detailed-search.  pairs/s from its "query batch
    execution time" (device work, host reading excluded) and from the wall
    time of the process."""
    from gtalign_alpha_b200 import synth
    binp = os.path.join(ROOT, "oracle", "_ref", "gpu", "gtalign")
    if not os.path.exists(binp):
        return {"unavailable": "oracle/_ref/gpu/gtalign not built (make -f oracle/Makefile.refgpu)"}
    nq, nref = args.qchunk, args.refgpu_refs
    sub = synth.Workload(wl.queries[:nq], wl.refs[:nref], wl.seed)
    d = tempfile.mkdtemp(prefix="gtrefgpu")
    try:
        synth.write_dirs(sub, d + "/q", d + "/r")
        cmd = [binp, "--qrs=" + d + "/q", "--rfs=" + d + "/r", "-o", d + "/out", "--outfmt=1",
               "--dev-queries-per-chunk=%d" % nq, "--dev-N=1",
               "--cpu-threads-reading=4"] + cli_options(args)
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, timeout=args.refgpu_timeout)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return {"unavailable": "reference GPU build exited %d: %s" % (p.returncode, p.stderr.decode()[-300:])}
        secs, seen = 0.0, set()
        for f in os.listdir(d + "/out"):
            J = json.load(open(os.path.join(d, "out", f)))["gtalign_search"]
            t = J["search_statistics"]["query_batch_execution_time"]
            if t not in seen:
                seen.add(t)
                secs += t
        v = nq * nref / secs
        out = {"value": v, "unit": UNIT, "wall_s": wall, "batch_s": secs,
               "sample": "%d queries x %d references of the workload, %s" % (nq, nref, options_text(args)),
               "ours_vs_reference_gpu": value / v}
        out["from_files"] = from_files_run(d, args, wall)
        return out
    except subprocess.TimeoutExpired:
        return {"unavailable": "reference GPU build did not finish within %d s" % args.refgpu_timeout}
    finally:
        shutil.rmtree(d, ignore_errors=True)


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
                      "1 reference, host buffers) per pair, polished form" % npairs}


def cpu_baseline_sample(wl, args):
    """The reference CPU build over all the workload's queries, each against
    the first cpu_sample_refs / 4 references (one call per query, as the
    reference arm cycles queries)."""
    threads = os.cpu_count() or 1
    from gtalign_alpha_b200 import synth
    nref = max(50, args.cpu_sample_refs // 4)
    pairs, secs, kind = 0, 0.0, "reference"
    for qi in range(len(wl.queries)):
        sub = synth.Workload(wl.queries[qi:qi + 1], wl.refs, wl.seed)
        p, s, kind = run_reference_sample(sub, 1, nref, threads, args)
        pairs += p
        secs += s
    return {"value": pairs / secs, "unit": UNIT, "cores": threads, "kind": kind, "cpu": cpu_model(),
            "sample": "each of the %d queries x the first %d references of the workload, %s; "
                      "%.1f s in all" % (len(wl.queries), nref, options_text(args), secs),
            "stalled_runs_restarted": dict(REF_STALLS)}


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from gtalign_alpha_b200 import synth
    wl = synth.config1(seed=args.seed, n_queries=args.nqueries, n_refs=args.cpu_sample_refs * 2)
    for _ in range(args.warmup):
        run_reference_sample(wl, 1, 50, threads, args)
    tot_pairs, tot_s, kind = 0, 0.0, "reference"
    for k in range(args.steps):
        qi = k % args.nqueries
        sub = synth.Workload(wl.queries[qi:qi + 1], wl.refs, wl.seed)
        pairs, secs, kind = run_reference_sample(sub, 1, args.cpu_sample_refs, threads, args)
        tot_pairs += pairs
        tot_s += secs
    v = tot_pairs / tot_s
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded C-alpha traces)",
            "config": {"workload": "16 queries x %d references (log-normal lengths, median 250)" % args.nrefs,
                       "options": options_text(args),
                       "parallelism": "host cores"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind, "cpu": cpu_model(),
                             "sample": "per step 1 query (cycling over the 16) x %d references of the "
                                       "workload" % args.cpu_sample_refs,
                             "stalled_runs_restarted": dict(REF_STALLS)},
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
    ap.add_argument("--autotune", type=int, default=1,
                    help="pick the launch shapes with gtb_autotune before the timed steps (0: defaults)")
    ap.add_argument("--speed", type=int, default=13, choices=list(range(14)),
                    help="the command line's --speed preset 0..12 (9: its default); 13: its "
                         "defaults with --no-detailed-search")
    ap.add_argument("--cpu-sample-refs", type=int, default=2000)
    ap.add_argument("--polish-steps", type=int, default=5,
                    help="adjoint polishing steps of the headline (batched + adjoint) form")
    ap.add_argument("--plain-pairs", type=int, default=300,
                    help="pairs timed in the one-pair-per-call form")
    ap.add_argument("--long-lengths", default="5000,8000,12000,16000,20000,25000,30000,37860")
    ap.add_argument("--adjoint-pairs", type=int, default=1_000_000)
    ap.add_argument("--adjoint-steps", type=int, default=10)
    ap.add_argument("--refgpu-refs", type=int, default=10000,
                    help="references in the reference GPU build's sample (x the first query chunk)")
    ap.add_argument("--refgpu-timeout", type=int, default=600)
    ap.add_argument("--long-refgpu-lengths", default="12000,37860",
                    help="long-chain pairs also run through the reference's GPU build (empty: none)")
    ap.add_argument("--cluster-n", type=int, default=1000,
                    help="structures of the all-against-all clustering leg")
    ap.add_argument("--legs", default="unpolished,e2e,plain,long,adjoint,cpu,refgpu,cluster,defaults,reader",
                    help="legs besides the headline: unpolished,e2e,plain,long,adjoint,cpu,refgpu,"
                         "cluster,defaults,reader")
    ap.add_argument("--reader-files", type=int, default=4000,
                    help="PDB files of the host-reader leg")
    ap.add_argument("--defaults-steps", type=int, default=2,
                    help="timed steps of the default-options leg (--speed 9)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
