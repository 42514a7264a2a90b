#!/usr/bin/env python
"""Benchmark of the OTF operator path on B200.

Default workload (N=1): the sigma-build microbenchmark, sigma = H c on 16
spatial orbitals with 8 alpha + 8 beta electrons (12870^2 = 165,636,900
determinants, UInt32 strings), seeded synthetic integrals, c ~ N(0,1)
normalised.  One step = one sigma application.  FP64 is the headline; the
FP32-bulk/FP64-accumulate sigma is timed beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload sigma|davidson|vqe]

N > 1 (torchrun, one rank per GPU): one sigma is split into N beta-column
bands (strong scaling); each rank computes its band from the whole input and
the bands are all-gathered over NCCL, so every rank ends the step with the
whole sigma.  The step time is the max over ranks.

--impl reference times the reference's own CPU implementation
(libotf_native built from the reference sources into oracle/_ref) on the
box's host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SIGMA_CFGS = {
    "16o": dict(norb=16, na=8, nb=8, seed=0),   # the sigma microbenchmark, 16 orbitals 8a+8b (the headline line)
    "15o": dict(norb=15, na=7, nb=8, seed=0),   # a smaller case of the same kernels, for ncu captures
}
SIGMA_CFG = SIGMA_CFGS["16o"]
METRIC = "sigma H*c builds per second (FP64), 16 orbitals 8a+8b"
UNIT = "sigma/s"
FP64_NOMINAL_TFLOPS = 37.0   # B200 FP64 (non-tensor) nominal; no measured figure on this pool


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# workload description (shared by both arms)
# ---------------------------------------------------------------------------

def pair_counts(net, norb, na, nb):
    """Exact connected (dst, src) pairs per group for one symmetry block
    (orbsym = 0): a string s connects under X-mask x iff popc(s & x) = popc(x)/2."""
    def conn(mask, n):
        k = bin(int(mask)).count("1")
        if k % 2:
            return 0
        return math.comb(k, k // 2) * math.comb(norb - k, n - k // 2) if n - k // 2 >= 0 else 0
    ca = {}
    cb = {}
    out = np.zeros(net.ngs)
    for g in range(net.ngs):
        ax, bx = int(net.axs[g]), int(net.bxs[g])
        if ax not in ca:
            ca[ax] = conn(ax, na)
        if bx not in cb:
            cb[bx] = conn(bx, nb)
        out[g] = ca[ax] * cb[bx]
    return out


def algorithmic_flops(net, pairs):
    """(2r + 1) flops per connected pair of a rank-r group: r products and r-1
    sums for the coefficient, one multiply and one add into the accumulator."""
    return float(np.sum(pairs * (2 * net.ranks + 1)))


def subnetwork(net, keep):
    """OTF network restricted to the groups `keep` (original order kept)."""
    from binsim_b200 import network as nw
    groups = [net.group(int(g)) for g in keep]
    out = [(ax, bx, r, za, zb, wa, wb) for (ax, bx, r, za, zb, wa, wb) in groups]
    return nw._pack(out, net.norb, net.orbsym)


# ---------------------------------------------------------------------------
# CPU baseline worker (no torch in this process: the reference's OpenMP)
# ---------------------------------------------------------------------------

def cpu_worker(args):
    from binsim_b200 import network as nw
    from oracle.oracle import RefLibs, ref_available
    if not ref_available():
        print(json.dumps({"unavailable": "oracle/_ref not built"}))
        return
    ref = RefLibs()
    cfg = SIGMA_CFGS[args.sigma_size]
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    pairs = pair_counts(net, cfg["norb"], cfg["na"], cfg["nb"])
    rb, dim = ref.basis(cfg["norb"], cfg["na"], cfg["nb"])
    rng = np.random.default_rng(1)
    x = rng.normal(size=dim)
    x /= np.linalg.norm(x)
    y = np.zeros(dim)
    import ctypes as C
    P = lambda a: a.ctypes.data_as(C.c_void_p)

    def run(keep):
        sub = subnetwork(net, keep)
        rn = ref.network(sub)
        t0 = time.perf_counter()
        ref.otf.hvec_gather_contract_otf_f64(rb, rn, P(x), P(y))
        dt = time.perf_counter() - t0
        ref.otf.destroy_network_otf_f64(rn)
        return dt, float(pairs[keep].sum())

    full = float(pairs.sum())
    threads = int(os.environ.get("OMP_NUM_THREADS", "0"))
    if args.cpu_full:
        # warm-up (OpenMP threads, first touch of the output): a sigma of every
        # 200th group, untimed
        run(np.arange(0, net.ngs, 200))
        # whole sigma, every group: the reference's contract_network_otf as the
        # Julia host calls it (one network, one hvec_gather_contract_otf_f64)
        rn = ref.network(net)
        times = []
        t_start = time.perf_counter()
        while True:
            t0 = time.perf_counter()
            ref.otf.hvec_gather_contract_otf_f64(rb, rn, P(x), P(y))
            times.append(time.perf_counter() - t0)
            spent = time.perf_counter() - t_start
            if len(times) >= max(1, args.cpu_reps) or spent + times[-1] > args.cpu_seconds:
                break
        ref.otf.destroy_network_otf_f64(rn)
        dt = float(np.median(times))
        print(json.dumps({"value": 1.0 / dt, "sec_per_sigma": dt, "sample_pairs": full, "full_pairs": full,
                          "sample_groups": int(net.ngs), "stride": 1, "sample_seconds": dt, "reps": len(times),
                          "times": times, "threads": threads, "full": True}))
        return
    off = np.flatnonzero(net.type_codes() != 0)
    # probe with a small stride, then size the sample to ~args.cpu_seconds
    stride = max(1, len(off) // 40)
    keep = off[::stride]
    dt, pr = run(keep)
    rate = pr / max(dt, 1e-9)
    target = args.cpu_seconds * rate
    stride = max(1, int(pairs[off].sum() / max(target, 1.0)))
    keep = off[::stride]
    times = []
    for _ in range(max(1, args.cpu_reps)):
        y[:] = 0.0
        dt, pr = run(keep)
        times.append(dt)
    dt = float(np.median(times))
    sec_per_sigma = dt * full / pr
    if args.cpu_out:
        # the sampled sub-network's reference sigma, for the GPU parity check
        np.save(os.path.join(args.cpu_out, "keep.npy"), keep)
        np.save(os.path.join(args.cpu_out, "sigma_ref.npy"), y)
    print(json.dumps({
        "value": 1.0 / sec_per_sigma, "sec_per_sigma": sec_per_sigma, "sample_pairs": pr, "full_pairs": full,
        "sample_groups": int(len(keep)), "stride": int(stride), "sample_seconds": dt, "reps": len(times),
        "threads": threads,
    }))


def run_cpu_baseline(args, full=False, out_dir=None, seconds=None, reps=None):
    """The reference's sigma on the host cores in a worker process (no torch):
    a sample of the groups scaled by pair counts, or with full=True whole sigmas
    (reps of them, as many as fit in `seconds`, at least one).  out_dir: the
    sampled run saves its groups and its sigma there."""
    try:
        import psutil
        cores = psutil.cpu_count(logical=False) or os.cpu_count()
    except Exception:
        cores = os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close", OMP_PLACES="cores")
    env.pop("CUDA_VISIBLE_DEVICES", None)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker",
           "--cpu-seconds", str(args.cpu_seconds if seconds is None else seconds),
           "--cpu-reps", str(args.cpu_reps if reps is None else reps), "--sigma-size", args.sigma_size]
    if full:
        cmd.append("--cpu-full")
    if out_dir:
        cmd += ["--cpu-out", out_dir]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0:
        log(r.stderr[-2000:])
        return None, cores
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line), cores


def cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def profile_traffic(name):
    """Figures of a committed ncu summary (profiles/<name>.json), or None."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", name + ".json")))
    except Exception:
        return None


def sigma_roofline(net, pairs, cfg, dim, stages, hbm, fp64_peak, world, ms, dmma_peak=None):
    """Roofline of the dominant kernel of the structured sigma, from the per-stage
    CUDA-event times measured in this run.  Returns (roofline dict, launches per sigma)."""
    if not stages:
        return ({"bound": "hbm", "achieved": dim * 16.0 / world / (ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                 "frac": None, "traffic": None, "note": "whole sigma (no per-stage times on this path)"}, None)
    launches = int(sum(v[1] for v in stages.values()))
    # stages -> kernels: both pure-spin stages launch pure_rows_kernel
    kern = {}
    for k, (t, n) in stages.items():
        name = "pure_rows" if k in ("pure_alpha", "pure_beta") else k
        t0, n0 = kern.get(name, (0.0, 0))
        kern[name] = (t0 + t, n0 + n)
    top = max(kern, key=lambda k: kern[k][0])
    t_ms, n_launch = kern[top]
    per_launch_s = t_ms * 1e-3 / max(1, n_launch)
    nA, nB = math.comb(cfg["norb"], cfg["na"]), math.comb(cfg["norb"], cfg["nb"])
    types = net.type_codes()
    if top == "mixed_gemm":
        # compulsory bytes of the GEMM stage: each source row of c~ read once, the
        # intermediate Z[a'][j][b] (M = connected alpha singles per row) written once
        M = cfg["na"] * (cfg["norb"] - cfg["na"])
        bytes_total = dim * 8.0 + nA * M * nB * 8.0
        flops_total = float(np.sum(pairs[types == 3] * (2 * net.ranks[types == 3] + 1)))
        # the GEMMs as executed: 64-row passes x every F excitation x every column
        nF = math.comb(cfg["norb"], 2)
        dense_total = 2.0 * nA * (64 * math.ceil(M / 64)) * nF * nB
    elif top == "pure_rows":
        # per launch (one spin side) the compulsory HBM bytes are one read of the
        # input (c~ or its transpose) and one write of the result; the source-row
        # re-reads of the row AXPYs are served by L2 (see l2_bytes)
        bytes_total = 2 * dim * 16.0
        sel = (types == 1) | (types == 2)
        flops_total = float(np.sum(pairs[sel] * (2 * net.ranks[sel] + 1)))
    else:
        bytes_total = dim * 16.0
        flops_total = 0.0
    if top != "mixed_gemm":
        dense_total = None
    achieved = bytes_total / max(1, n_launch) / per_launch_s / 1e9
    prof = profile_traffic(f"sigma_{top}_15o7a8b")
    traffic = None
    if prof and prof.get("dram_bytes_per_launch") and prof.get("units_per_launch"):
        # scale the captured launch (15 orbitals) by the determinants one launch covers here
        units_here = dim / max(1, n_launch)
        traffic = prof["dram_bytes_per_launch"] * units_here / prof["units_per_launch"]
    roof = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm if hbm else None, "traffic": traffic,
            "launches_per_sigma": n_launch, "ms_per_launch": per_launch_s * 1e3,
            "fp64_tflops": flops_total / max(1, n_launch) / per_launch_s / 1e12,
            "fp64_frac_of_measured_fma_peak": flops_total / max(1, n_launch) / per_launch_s / 1e12 / fp64_peak,
            "fp64_dense_gemm_tflops": (dense_total / max(1, n_launch) / per_launch_s / 1e12) if dense_total else None,
            "dense_frac_of_measured_dmma_peak": (dense_total / max(1, n_launch) / per_launch_s / 1e12 / dmma_peak)
            if dense_total and dmma_peak else None,
            "note": "dominant kernel of the structured sigma, timed live per launch with CUDA events; achieved = "
                    "its compulsory HBM bytes per launch / launch time, of the measured HBM copy peak; the kernel "
                    "is bound by the tensor cores' FP64 (DMMA) pipe, see dense_frac_of_measured_dmma_peak (the dense "
                    "GEMM as executed against the measured DMMA peak); traffic = ncu dram bytes of a 15-orbital "
                    "launch scaled by determinants per launch"}
    return roof, launches


def gpu_sigma(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from binsim_b200 import cuotf, network as nw

    torch.cuda.set_device(local_rank)
    cfg = SIGMA_CFGS[args.sigma_size]
    t0 = time.time()
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    pairs = pair_counts(net, cfg["norb"], cfg["na"], cfg["nb"])
    flops = algorithmic_flops(net, pairs)
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    H = cuotf.CuNetwork(net)
    f = cuotf.CuOTFFunctions(B, H)
    log(f"[rank {rank}] setup {time.time() - t0:.1f}s dim={B.dim} groups={net.ngs}")
    dim = B.dim
    rng = np.random.default_rng(1)
    xh = rng.normal(size=dim)
    xh /= np.linalg.norm(xh)
    x = torch.from_numpy(xh).cuda()
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    shard = None
    if world > 1:
        # beta-column bands per rank, then an NCCL all-gather of the bands: every
        # rank ends the step holding the whole sigma (the next step's input)
        from binsim_b200.shard import ColumnShardedSigma
        shard = ColumnShardedSigma(f.hvec_cols, math.comb(cfg["norb"], cfg["na"]), math.comb(cfg["norb"], cfg["nb"]))

    def step(mixed=False):
        if world == 1:
            (f.hvec_mixed if mixed else f.hvec)(x, y)
        else:
            shard(x, y, mixed=mixed)
    path = f.sigma_path()
    log(f"[rank {rank}] sigma path {path}")

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        torch.cuda.synchronize()
        return ms

    with Clocks(local_rank) as clk:
        ms = timed(step, args.steps, args.warmup)
    ms_mixed = timed(lambda: step(True), args.steps, max(1, args.warmup))
    # mixed-precision error vs FP64 on this rank's rows
    step(False)
    y64 = y.clone()
    step(True)
    err_mixed = float((y - y64).abs().max() / y64.abs().max())

    # per-stage device times of one sigma (CUDA events around every launch of
    # the structured path), FP64 and FP32 bulk; the median of 3 runs per stage
    stages, stages32 = None, None
    if world == 1 and path[0] == 1:
        runs = [f.sigma_stage_times(x, y) for _ in range(3)]
        stages = {k: (float(np.median([r[k][0] for r in runs])), runs[0][k][1]) for k in runs[0]}
        runs = [f.sigma_stage_times(x, y, mixed=True) for _ in range(3)]
        stages32 = {k: (float(np.median([r[k][0] for r in runs])), runs[0][k][1]) for k in runs[0]}
    fp64_peak = cuotf.fma_peak(True)
    fp32_peak = cuotf.fma_peak(False)
    dmma_peak = cuotf.fma_peak(dmma=True)

    # e2e through the public API with host buffers: H2D c, sigma, D2H sigma
    xpin = torch.from_numpy(xh).pin_memory()
    ypin = torch.empty(dim, dtype=torch.float64).pin_memory()

    def e2e_step():
        x.copy_(xpin, non_blocking=True)
        step(False)
        ypin.copy_(y, non_blocking=True)
    ms_e2e_serial = timed(e2e_step, max(1, args.steps // 2), 1)
    # the public host-vector call: every step copies its input in and its result
    # out, the copies of neighbouring steps overlapped with the sigma between them
    ms_e2e = None
    if world == 1:
        ksteps = max(1, args.steps)
        f.hvec_host([xpin], [ypin])   # warm-up (device buffers of the pipeline)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f.hvec_host([xpin] * ksteps, [ypin] * ksteps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1) / ksteps
        host_err = float(np.abs(ypin.numpy() - y.cpu().numpy()).max() / np.abs(y.cpu().numpy()).max())
    else:
        ms_e2e = ms_e2e_serial
        host_err = None

    result = None
    if rank == 0:
        pk = peaks()
        hbm = pk.get("hbm_gbs")
        tflops = flops / world / (ms * 1e-3) / 1e12
        roof, launches = sigma_roofline(net, pairs, cfg, dim, stages, hbm, fp64_peak, world, ms, dmma_peak)
        if launches is None:
            launches = count_launches(step)
        result = {
            "metric": METRIC if args.sigma_size == "16o" else
            f"sigma H*c builds per second (FP64), {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b",
            "value": 1000.0 / ms, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"sigma microbenchmark: H*c, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, "
                                   f"{dim:,} dets, UInt32 strings, seeded synthetic integrals (seed {cfg['seed']}), "
                                   "c ~ N(0,1) normalised",
                       "dim": dim, "groups": int(net.ngs), "pair_updates": float(pairs.sum()),
                       "l2": f"inputs larger than L2 (c and sigma are {dim * 8 / 1e9:.2f} GB each)",
                       "sharding": (f"{world} beta-column bands of one sigma + NCCL all-gather of the bands "
                                    f"({shard.exchange_bytes() / 1e9:.2f} GB received per rank per step)")
                       if world > 1 else "single GPU"},
            "e2e": {"value": 1000.0 / ms_e2e, "unit": UNIT, "h2d_bytes_per_step": dim * 8,
                    "d2h_bytes_per_step": dim * 8, "ms_per_step": ms_e2e,
                    "path": "bsim_hvec_host over pinned host vectors: per step H2D of c, sigma, D2H of sigma; "
                            "copies of neighbouring steps overlap the sigma between them" if world == 1 else
                            "H2D, sharded sigma, D2H in sequence",
                    "serial_ms_per_step": ms_e2e_serial,
                    "max_rel_diff_host_vs_device_result": host_err},
            "mixed": {"value": 1000.0 / ms_mixed, "unit": UNIT, "ms_per_step": ms_mixed,
                      "dtype": "f32 bulk, f64 accumulate", "max_rel_err_vs_fp64": err_mixed,
                      "speedup_vs_fp64": ms / ms_mixed},
            "roofline": roof,
            "compute_roofline": {"bound": "fp64 CUDA cores", "achieved": tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                                 "frac": tflops / fp64_peak, "flops_per_sigma": flops,
                                 "note": "whole sigma: (2r+1) flops per connected pair of a rank-r group; peak = "
                                         "FP64 FMA-chain throughput measured on this GPU by bsim_fma_peak (no FP64 "
                                         "figure in MEASURED_PEAKS.json)"},
            "stages_ms": {k: round(v[0], 3) for k, v in stages.items()} if stages else None,
            "stages_ms_fp32_bulk": {k: round(v[0], 3) for k, v in stages32.items()} if stages32 else None,
            "fp32_fma_peak_tflops": fp32_peak,
            "fp64_dmma_peak_tflops": dmma_peak,
            "pair_updates_per_s": float(pairs.sum()) / (ms * 1e-3),
            "sigma_path": {"path": path[0], "reason": path[1], "residual_groups": path[2]},
            "gpu_launches": launches * args.steps if launches else None,
            "clocks": clk.summary(),
        }
    return result, net


def sampled_parity(args, net, sample_dir):
    """The GPU sigma (FP64 and FP32 bulk) of the sub-network the CPU leg ran
    through the reference's hvec_gather_contract_otf_f64 (op/hvec.hpp:481-496),
    on the same input, against the reference's result."""
    import torch
    from binsim_b200 import cuotf
    cfg = SIGMA_CFGS[args.sigma_size]
    keep = np.load(os.path.join(sample_dir, "keep.npy"))
    yref = np.load(os.path.join(sample_dir, "sigma_ref.npy"))
    sub = subnetwork(net, keep)
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(sub))
    rng = np.random.default_rng(1)   # the CPU leg's input
    xh = rng.normal(size=B.dim)
    xh /= np.linalg.norm(xh)
    x = torch.from_numpy(xh).cuda()
    y = torch.empty_like(x)
    scale = float(np.abs(yref).max())
    out = {"groups": int(len(keep)), "of_groups": int(net.ngs), "sigma_path": f.sigma_path()[0],
           "max_abs_ref": scale,
           "note": "the CPU leg's sampled sub-network (every k-th off-diagonal group), same input c: GPU sigma "
                   "vs the reference's hvec_gather_contract_otf_f64 on the host; rel = abs / max|sigma_ref|"}
    for name, fn in (("fp64", f.hvec), ("fp32_bulk", f.hvec_mixed)):
        fn(x, y)
        d = float(np.abs(y.cpu().numpy() - yref).max())
        out[name] = {"max_abs_err_vs_reference": d, "max_rel_err_vs_reference": d / scale}
    del f, B, x, y
    torch.cuda.empty_cache()
    return out


def davidson_pair(size):
    """One FP64 and one mixed Davidson solve of the lowest root at a DAV_CFGS size,
    each timed with CUDA events after a warm-up sigma of its precision (a solve is
    tens of sigmas): seconds, iterations, energies."""
    import torch
    from binsim_b200 import cuotf, network as nw
    cfg = DAV_CFGS[size]
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    diags = torch.zeros(B.dim, dtype=torch.float64, device="cuda")
    f.get_diags(diags)
    v0 = torch.zeros_like(diags)
    v0[B.hf_index()] = 1.0
    x, y = torch.empty_like(v0), torch.empty_like(v0)
    f.hvec(v0, y)
    f.hvec_mixed(v0, y)
    out = {}
    for mixed in (False, True):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = f.davidson(v0.clone(), diags, x, tol=DAV_TOL, maxiter=500, ncv=cfg["ncv"], maxspace=cfg["maxspace"],
                        mixed=mixed)
        e1.record()
        torch.cuda.synchronize()
        out["mixed" if mixed else "fp64"] = {"seconds": e0.elapsed_time(e1) * 1e-3, "iterations": st["iterations"],
                                            "energy": st["energy"]}
    del f, B, net, diags, v0, x, y
    torch.cuda.empty_cache()
    return {"workload": f"FCI Davidson, lowest root, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, seeded synthetic "
                        f"integrals (seed {cfg['seed']}), HF start, subspace {cfg['maxspace']}, restart to {cfg['ncv']}, "
                        f"residual tol {DAV_TOL}",
            "fp64_s": out["fp64"]["seconds"], "mixed_s": out["mixed"]["seconds"],
            "mixed_speedup_vs_fp64": out["fp64"]["seconds"] / out["mixed"]["seconds"],
            "fp64_iterations": out["fp64"]["iterations"], "mixed_iterations": out["mixed"]["iterations"],
            "abs_energy_diff_eh": abs(out["fp64"]["energy"] - out["mixed"]["energy"]),
            "solves_timed": "one per precision, after a warm-up sigma of each",
            "target": "mixed >= 1.5x faster than FP64 within 1e-8 Eh"}


def task_targets(args):
    """The task's two targets at their named sizes, for the default line: FCI
    Davidson at 12 orbitals 6a+6b (FP64 and mixed, time to the root, energy error
    against the reference's CPU Davidson) and, where sigma dominates the step, at
    16 orbitals 8a+8b; VQE energy + adjoint gradient at 14 orbitals 7a+7b with 2000
    generators (against the reference-style backgrad sweep and the per-parameter
    gradient by central differences)."""
    import copy
    import torch
    a = copy.copy(args)
    a.steps, a.warmup, a.dav_size = 3, 3, "12o"
    t0 = time.time()
    dav = gpu_davidson(a)
    torch.cuda.empty_cache()
    dav16 = davidson_pair("16o")
    t1 = time.time()
    vqe = gpu_vqe(a)
    torch.cuda.empty_cache()
    t2 = time.time()
    pp = vqe["adjoint_vs_per_parameter"]
    return {
        "fci_davidson_12o": {
            "workload": dav["config"]["workload"], "fp64_s": dav["fp64"]["seconds"],
            "mixed_s": dav["mixed"]["seconds"], "mixed_speedup_vs_fp64": dav["mixed"]["speedup_vs_fp64"],
            "fp64_abs_err_vs_oracle_eh": dav["fp64"]["abs_err_vs_oracle"],
            "mixed_abs_err_vs_oracle_eh": dav["mixed"]["abs_err_vs_oracle"],
            "fp64_iterations": dav["fp64"]["iterations"], "mixed_iterations": dav["mixed"]["iterations"],
            "mixed_sigma_fp32": dav["mixed"]["sigma_fp32"], "mixed_sigma_fp64": dav["mixed"]["sigma_fp64"],
            "oracle_energy": dav["oracle_energy"], "reference_cpu_s": (dav.get("cpu_baseline") or {}).get("value"),
            "solves_timed": dav["steps"], "target": "mixed >= 1.5x faster than FP64 within 1e-8 Eh"},
        "fci_davidson_16o": dav16,
        "vqe_14o": {
            "workload": vqe["config"]["workload"], "evals_per_s": vqe["value"], "ms_per_eval": vqe["ms_per_step"],
            "energy": vqe["energy"],
            "reference_sweep_ms": vqe["adjoint_vs_reference_sweep"]["sweep_ms"],
            "adjoint_vs_reference_sweep": vqe["adjoint_vs_reference_sweep"]["speedup"],
            "max_abs_grad_diff_vs_sweep": vqe["adjoint_vs_reference_sweep"]["max_abs_grad_diff"],
            "per_parameter_gradient_ms": pp["fd_ms"], "adjoint_vs_per_parameter": pp["speedup"],
            "per_parameter_sample": pp["sample"], "max_abs_fd_err": pp["max_abs_fd_err"],
            "target": "adjoint >= 10x faster than the per-parameter gradient at 1e-7 agreement"},
        "seconds": {"davidson": round(t1 - t0, 1), "vqe": round(t2 - t1, 1)},
    }


def count_launches(fn, prefix="bsim::"):
    """Kernels of this library launched by one call of fn, counted in an
    untimed pass under the CUDA activity tracer."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    try:
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
    except Exception as e:  # tracer unavailable
        log(f"launch count unavailable: {e}")
        return None
    n = 0
    for ev in prof.events():
        if prefix in ev.name and getattr(ev, "device_type", None) is not None and "CUDA" in str(ev.device_type):
            n += 1
    return n


def timed_events(fn, k, w):
    """Device time of k calls of fn after w warm-up calls (CUDA events on the
    current stream, synchronised on both sides); ms per call."""
    import torch
    for _ in range(w):
        fn()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / k


# ---------------------------------------------------------------------------
# Band overhead of the sharded sigma, measured on one GPU
# ---------------------------------------------------------------------------

def gpu_bands(args):
    """The per-rank unit of the N-GPU sigma (bsim_hvec_cols, one beta-column
    band) timed band by band on one GPU for N = 2, 4, 8: the sum over the N bands
    against one whole sigma is the work the split adds (with a band, the beta
    same-spin doubles go through the row lists instead of the intermediate-string
    GEMM), and the largest band bounds the N-GPU step before its all-gather."""
    import torch
    from binsim_b200 import cuotf, network as nw
    from binsim_b200.shard import column_bands
    cfg = SIGMA_CFGS[args.sigma_size]
    torch.cuda.set_device(0)
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    nA, nB = math.comb(cfg["norb"], cfg["na"]), math.comb(cfg["norb"], cfg["nb"])
    rng = np.random.default_rng(1)
    xh = rng.normal(size=B.dim)
    xh /= np.linalg.norm(xh)
    x = torch.from_numpy(xh).cuda()
    y = torch.empty_like(x)
    steps, warm = max(1, args.steps), max(3, args.warmup)
    out = {}
    for mixed in (False, True):
        key = "fp32_bulk" if mixed else "fp64"
        whole = timed_events(lambda: (f.hvec_mixed if mixed else f.hvec)(x, y), steps, warm)
        per_n = {}
        for n in (2, 4, 8):
            bands = column_bands(nB, n)
            ms = [timed_events(lambda lo=lo, hi=hi: f.hvec_cols(x, y, lo, hi, mixed=mixed), steps, 1)
                  for lo, hi in bands if hi > lo]
            per_n[str(n)] = {"bands_ms": [round(v, 3) for v in ms], "sum_ms": sum(ms), "max_ms": max(ms),
                             "overhead_vs_whole": sum(ms) / whole - 1.0, "ideal_speedup": whole / max(ms)}
        out[key] = {"whole_ms": whole, "splits": per_n}
    return {"metric": "sigma band overhead on one GPU", "unit": "ms", "n_gpus": 1, "steps": steps, "warmup": warm,
            "config": {"workload": f"sigma, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, beta-column bands of "
                                   f"{nB} columns (starts on multiples of 128), {nA} alpha rows"},
            "bands": out}


# ---------------------------------------------------------------------------
# FCI Davidson workload: time to the lowest root, FP64 vs FP32-bulk mixed
# ---------------------------------------------------------------------------

DAV_CFGS = {
    # the plain FP64 FCI Davidson workload, 12 orbitals 6a+6b, subspace 8
    "12o": dict(norb=12, na=6, nb=6, seed=0, maxspace=8, ncv=3),
    # the sigma microbenchmark's space, where sigma dominates the step
    "16o": dict(norb=16, na=8, nb=8, seed=0, maxspace=8, ncv=3),
}
DAV_TOL = 1e-5          # residual norm (jl/davidson.jl convergence test); energy error checked against 1e-8 Eh
DAV_METRIC = "FCI Davidson time to the lowest root within 1e-8 Eh (FP64 path)"


def gpu_davidson(args):
    import torch
    from binsim_b200 import cuotf, network as nw
    cfg = DAV_CFGS[args.dav_size]
    torch.cuda.set_device(0)
    t0 = time.time()
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    dim = B.dim
    diags = torch.zeros(dim, dtype=torch.float64, device="cuda")
    f.get_diags(diags)
    hf = B.hf_index()
    v0h = np.zeros(dim)
    v0h[hf] = 1.0
    v0 = torch.from_numpy(v0h).cuda()
    x = torch.empty_like(v0)
    y = torch.empty_like(v0)
    f.hvec(v0, y)           # builds the sigma plan outside the timed region
    f.hvec_mixed(v0, y)
    torch.cuda.synchronize()
    log(f"davidson setup {time.time() - t0:.1f}s dim={dim} sigma path {f.sigma_path()}")
    stats = {}

    def run(mixed, tol=DAV_TOL):
        def go():
            stats[mixed] = f.davidson(v0.clone(), diags, x, tol=tol, maxiter=500, ncv=cfg["ncv"],
                                      maxspace=cfg["maxspace"], mixed=mixed)
        return go
    # tight FP64 energy: the GPU FP64 path to a 1e-9 residual
    run(False, 1e-9)()
    e_tight = stats[False]["energy"]
    steps, warm = max(1, args.steps), max(3, args.warmup)
    ms64 = timed_events(run(False), steps, warm)
    st64 = dict(stats[False])
    ms32 = timed_events(run(True), steps, warm)
    st32 = dict(stats[True])
    launches = count_launches(run(False))
    # e2e: host start vector and diagonal in, host eigenvector out, per solve
    v0pin = torch.from_numpy(v0h).pin_memory()
    dpin = diags.cpu().pin_memory()
    xpin = torch.empty(dim, dtype=torch.float64).pin_memory()

    def e2e():
        v0.copy_(v0pin, non_blocking=True)
        diags.copy_(dpin, non_blocking=True)
        run(False)()
        xpin.copy_(x, non_blocking=True)
    ms_e2e = timed_events(e2e, steps, 1)
    cpu = None
    if not args.no_cpu_baseline and args.dav_size == "12o":
        cpu = run_cpu_davidson(args)
    e_oracle = cpu["energy"] if cpu and "energy" in cpu else e_tight
    sig = dim * 16.0
    res = {
        "metric": DAV_METRIC, "value": ms64 * 1e-3, "unit": "s", "n_gpus": 1, "steps": steps, "warmup": warm,
        "ms_per_step": ms64, "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"FCI Davidson, lowest root, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, "
                               f"{dim:,} dets, UInt32 strings, seeded synthetic integrals (seed {cfg['seed']}), "
                               f"HF start, subspace {cfg['maxspace']}, restart to {cfg['ncv']}, residual tol {DAV_TOL}",
                   "dim": dim, "l2": "vectors larger than L2" if sig > 126e6 else "vectors fit in L2"},
        "fp64": {"seconds": ms64 * 1e-3, "iterations": st64["iterations"], "sigma_fp64": st64["sigma_fp64"],
                 "energy": st64["energy"], "abs_err_vs_oracle": abs(st64["energy"] - e_oracle)},
        "mixed": {"seconds": ms32 * 1e-3, "iterations": st32["iterations"], "sigma_fp64": st32["sigma_fp64"],
                  "sigma_fp32": st32["sigma_fp32"], "energy": st32["energy"],
                  "abs_err_vs_oracle": abs(st32["energy"] - e_oracle), "speedup_vs_fp64": ms64 / ms32},
        "oracle_energy": {"value": e_oracle, "source": "reference CPU Davidson (libotf_native + libdiag), "
                                                       "residual 1e-9" if cpu and "energy" in cpu else
                          "GPU FP64 Davidson to residual 1e-9 (parity-tested path)"},
        "e2e": {"value": ms_e2e * 1e-3, "unit": "s", "h2d_bytes_per_step": 2 * dim * 8, "d2h_bytes_per_step": dim * 8,
                "ms_per_step": ms_e2e},
        "gpu_launches": launches * steps if launches is not None else None,
    }
    if cpu:
        res["cpu_baseline"] = {"value": cpu.get("seconds"), "unit": "s", "cores": cpu.get("cores"),
                               "kind": "reference", "sample": cpu.get("sample")}
    return res


# ---------------------------------------------------------------------------
# Block Davidson workload: lowest 2 roots, FP32 subspace + FP64 refinement
# ---------------------------------------------------------------------------

BLOCK_CFGS = {
    # 18 orbitals 8a+8b (1.91e9 dets): 6 FP32 subspace vectors (7.66 GB each) plus their
    # sigmas, FP64 roots; FP64 block Davidson with 6 kept vectors does not fit in HBM
    "18o": dict(norb=18, na=8, nb=8, seed=0, nroots=2, maxspace=6, ncv=2, modes=("mixed",), scratch_gb=4.0,
                maxiter=160),
    # the same solver at 16 orbitals, where both precisions fit: the FP64/mixed comparison
    "16o": dict(norb=16, na=8, nb=8, seed=0, nroots=2, maxspace=6, ncv=2, modes=("fp64", "mixed"), scratch_gb=24.0,
                maxiter=400),
}
BLOCK_TOL = 1e-5
BLOCK_METRIC = "FCI block Davidson time to the lowest 2 roots (FP64 residual norms < 1e-5)"


def gpu_block_davidson(args):
    import torch
    from binsim_b200 import cuotf, network as nw
    cfg = BLOCK_CFGS[args.block_size]
    os.environ["BSIM_SIGMA_SCRATCH_GB"] = str(cfg["scratch_gb"])
    torch.cuda.set_device(0)
    t0 = time.time()
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    dim, k = B.dim, cfg["nroots"]
    log(f"block davidson: network {net.ngs} groups, dim {dim:,}, setup {time.time() - t0:.1f}s")
    X = torch.zeros((k, dim), dtype=torch.float64, device="cuda")
    f.get_diags(X[0])                      # FP64 diagonal, kept in FP32 for the preconditioner
    d32 = X[0].float()
    X[0].zero_()
    starts, saved = [], []
    for _ in range(k):                     # the k lowest-diagonal determinants
        i = int(torch.argmin(d32))
        starts.append(i)
        saved.append(float(d32[i]))
        d32[i] = float("inf")
    for i, v in zip(starts, saved):
        d32[i] = v

    def reset():
        X.zero_()
        for j, i in enumerate(starts):
            X[j, i] = 1.0
    # warm-up: plan build and both sigma precisions (the scratch reaches its FP64 size)
    reset()
    t1 = time.time()
    for _ in range(max(1, args.warmup)):
        f.hvec(X[0], X[1])
        f.hvec_mixed(X[0], X[1])
    torch.cuda.synchronize()
    log(f"sigma path {f.sigma_path()}, warm-up {time.time() - t1:.1f}s")
    # full-size checks on random vectors u, v: <v|H u> = <u|H v> (FP64), and the
    # FP32-bulk sigma against the FP64 one
    g = torch.Generator(device="cuda").manual_seed(1)
    X[0].normal_(generator=g)
    X[0] /= X[0].norm()
    v = torch.empty(dim, dtype=torch.float64, device="cuda").normal_(generator=g)
    v /= v.norm()
    y = torch.empty_like(v)
    f.hvec(X[0], X[1])
    f.hvec(v, y)
    a, b = float(torch.dot(v, X[1])), float(torch.dot(X[0], y))
    f.hvec_mixed(X[0], y)
    checks = {"symmetry_rel": abs(a - b) / abs(a),
              "fp32_bulk_vs_fp64_rel": float((y - X[1]).abs().max() / X[1].abs().max())}
    del v, y
    torch.cuda.empty_cache()
    log(f"full-size checks {checks}")
    stages = {}
    for mixed in (False, True):
        reset()
        tm = f.sigma_stage_times(X[0], X[1], mixed=mixed)
        stages["fp32" if mixed else "fp64"] = {"total_ms": float(sum(v[0] for v in tm.values())),
                                               "stages_ms": {kk: round(v[0], 3) for kk, v in tm.items()}}
    out = {}
    for mode in cfg["modes"]:
        reset()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = f.davidson_block(X, d32, k, tol=BLOCK_TOL, maxiter=cfg["maxiter"], ncv=cfg["ncv"],
                              maxspace=cfg["maxspace"], mixed=(mode == "mixed"), verbose=args.verbose)
        e1.record()
        torch.cuda.synchronize()
        st["seconds"] = e0.elapsed_time(e1) * 1e-3
        st["free_gb_before"] = free0 / 1e9
        out[mode] = st
        log(f"{mode}: {st}")
    main = out["mixed"]
    res = {
        "metric": BLOCK_METRIC, "value": main["seconds"], "unit": "s", "n_gpus": 1, "steps": 1,
        "warmup": f"{max(1, args.warmup)} sigma applications per precision (one solve takes minutes)",
        "ms_per_step": main["seconds"] * 1e3, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 subspace / f64 refinement", "data": "synthetic",
        "config": {"workload": f"mixed-precision block Davidson, lowest {k} roots, {cfg['norb']} orbitals "
                               f"{cfg['na']}a+{cfg['nb']}b, {dim:,} dets, UInt32 strings, seeded synthetic "
                               f"integrals (seed {cfg['seed']}), start: the {k} lowest-diagonal determinants, "
                               f"{cfg['maxspace']} FP32 subspace vectors kept, restart to {cfg['ncv']}, FP32 "
                               f"diagonal preconditioner, FP64 residual tol {BLOCK_TOL}",
                   "dim": dim, "l2": "vectors larger than L2"},
        "sigma_ms": stages, "sigma_checks": checks, "solves": out,
    }
    if "fp64" in out:
        res["fp64_vs_mixed"] = {"speedup": out["fp64"]["seconds"] / main["seconds"],
                                "max_abs_energy_diff": max(abs(a - b) for a, b in
                                                           zip(out["fp64"]["energies"], main["energies"]))}
    return res


# ---------------------------------------------------------------------------
# VQE workload: energy + full gradient by the adjoint sweep
# ---------------------------------------------------------------------------

VQE_CFG = dict(norb=14, na=7, nb=7, seed=0, n_gen=2000, amp=0.05, ckpt=64)
VQE_METRIC = "VQE UCCGSD energy + adjoint gradient evaluations per second"


def vqe_problem(cfg):
    from binsim_b200 import network as nw
    # grouping + SVD compression in the library's native builder (the 36-orbital
    # Hamiltonian and pool take ~65 s less than with the numpy builder)
    ham = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"], native=True)
    pool = nw.ucc_pool(cfg["norb"], native=True)
    op_idx, param_idx, th = nw.draw_generators(pool, cfg["n_gen"], seed=cfg["seed"], amp_sigma=cfg["amp"])
    return ham, pool, op_idx, param_idx, th


def gpu_vqe(args):
    import torch
    from binsim_b200 import cuotf
    cfg = VQE_CFG
    torch.cuda.set_device(0)
    t0 = time.time()
    ham, pool, op_idx, param_idx, th = vqe_problem(cfg)
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(ham), cuotf.CuNetwork(pool.network))
    dim = B.dim
    ref_idx, ref_val = np.array([B.hf_index()]), np.array([1.0])
    lv = torch.empty(dim, dtype=torch.float64, device="cuda")
    rv = torch.empty_like(lv)
    f.hvec(lv.zero_(), rv)
    torch.cuda.synchronize()
    log(f"vqe setup {time.time() - t0:.1f}s dim={dim} components={len(op_idx)} params={len(th)}")
    out = {}

    def adjoint():
        out["adj"] = f.energy_grad(op_idx, param_idx, th, ref_idx, ref_val, lv, rv, ckpt_every=cfg["ckpt"])
    steps, warm = max(1, args.steps), max(3, args.warmup)
    with Clocks(0) as clk:
        ms_adj = timed_events(adjoint, steps, warm)
    E, g, var = out["adj"]
    launches = count_launches(adjoint)

    # the reference's energy_objective (jl/vqe.jl:1-21) step by step through the
    # legacy entry points: one expm per component, hvec, one backgrad per
    # component with its host round trip
    def ref_sweep():
        lv.zero_()
        lv[int(ref_idx[0])] = 1.0
        for i, p in zip(op_idx, param_idx):
            f.expm(int(i) + 1, float(th[p]), lv)
        f.hvec(lv, rv)
        ln = float(lv @ lv)
        gg = np.zeros(len(th))
        for i, p in zip(op_idx[::-1], param_idx[::-1]):
            gg[p] += f.backgrad(int(i) + 1, float(th[p]), lv, rv) * 2 / ln
        out["sweep"] = gg
    ms_sweep = timed_events(ref_sweep, 1, 1)

    # plain per-parameter gradient: central differences, two energies per parameter
    def energy(t):
        f.prepare_state(op_idx, param_idx, t, ref_idx, ref_val, lv)
        f.hvec(lv, rv)
        return float(lv @ rv) / float(lv @ lv)
    ms_energy = timed_events(lambda: energy(th), steps, 1)
    # measured on a sample: the central-difference gradient of the 8 steepest
    # parameters (16 energies), timed with CUDA events, scaled to every parameter
    h = 1e-5
    fd_params = [int(p) for p in np.argsort(-np.abs(g))[:8]]
    fd = {}

    def fd_sample():
        for p in fd_params:
            tp, tm = th.copy(), th.copy()
            tp[p] += h
            tm[p] -= h
            fd[p] = (energy(tp) - energy(tm)) / (2 * h)
    ms_fd_sample = timed_events(fd_sample, 1, 0)
    fd_err = max(abs(fd[p] - g[p]) for p in fd_params)
    ms_fd = ms_fd_sample * len(th) / len(fd_params)
    # e2e: parameters from the host, energy and gradient back to the host (the call does both)
    res = {
        "metric": VQE_METRIC, "value": 1000.0 / ms_adj, "unit": "evals/s", "n_gpus": 1, "steps": steps,
        "warmup": warm, "ms_per_step": ms_adj, "higher_is_better": True, "scaling": "replicas",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"VQE energy + gradient, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, {dim:,} dets, "
                               f"{cfg['n_gen']} spin-adapted generalised singles/doubles drawn with seed {cfg['seed']} "
                               f"({len(op_idx)} spin-orbital components), amplitudes N(0, {cfg['amp']}^2), HF reference, "
                               f"checkpoint every {cfg['ckpt']} generators",
                   "dim": dim, "components": int(len(op_idx)), "params": int(len(th)),
                   "l2": "state vectors 94 MB each; two of them plus checkpoints exceed L2"},
        "energy": E, "variance": var,
        "adjoint_vs_reference_sweep": {"sweep_ms": ms_sweep, "speedup": ms_sweep / ms_adj,
                                       "max_abs_grad_diff": float(np.abs(out["sweep"] - g).max()),
                                       "note": "jl/vqe.jl energy_objective on this library's legacy entry points"},
        "adjoint_vs_per_parameter": {"fd_ms": ms_fd, "energy_ms": ms_energy, "speedup": ms_fd / ms_adj,
                                     "max_abs_fd_err": fd_err, "fd_params": fd_params,
                                     "fd_grads": [float(g[p]) for p in fd_params],
                                     "sample": f"central differences (h = 1e-5) of the {len(fd_params)} steepest "
                                               f"parameters measured ({ms_fd_sample:.1f} ms for "
                                               f"{2 * len(fd_params)} energies), scaled by {len(th)} / "
                                               f"{len(fd_params)} parameters",
                                     "note": "the plain per-parameter gradient: 2 energies per parameter"},
        "e2e": {"value": 1000.0 / ms_adj, "unit": "evals/s", "h2d_bytes_per_step": int(8 * (len(th) + 2 * len(op_idx))),
                "d2h_bytes_per_step": int(8 * (len(th) + 2)), "ms_per_step": ms_adj,
                "note": "the public call takes host parameters and returns host energy and gradient"},
        "gpu_launches": launches * steps if launches is not None else None,
        "clocks": clk.summary(),
    }
    return res


# ---------------------------------------------------------------------------
# ADAPT workload: pool-gradient screening on UInt64 strings, plus the adjoint gradient
# ---------------------------------------------------------------------------

# 36 orbitals 3a+3b (7140^2 determinants): 516K Hamiltonian groups, 840K pool
# components; --adapt-norb 20 gives a quick case of the same operator mix
ADAPT_CFG = dict(norb=36, na=3, nb=3, seed=0, n_gen=40, amp=0.05, ckpt=8)
ADAPT_METRIC = "ADAPT pool screening: spin-adapted pool gradients per second (UInt64 strings)"


def adapt_problem(cfg):
    from binsim_b200 import network as nw
    t0 = time.time()
    # grouping + SVD compression in the library's native builder (the 36-orbital
    # Hamiltonian and pool take ~65 s less than with the numpy builder)
    ham = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"], native=True)
    pool = nw.ucc_pool(cfg["norb"], native=True)
    op_idx, param_idx, th = nw.draw_generators(pool, cfg["n_gen"], seed=cfg["seed"], amp_sigma=cfg["amp"])
    log(f"adapt problem built in {time.time() - t0:.1f}s: {ham.ngs} Hamiltonian groups, {pool.network.ngs} pool "
        f"components, {len(pool.components)} generators")
    return ham, pool, op_idx, param_idx, th


def adapt_cfg(args):
    cfg = dict(ADAPT_CFG)
    cfg["norb"] = args.adapt_norb
    return cfg


def gpu_adapt(args):
    """ADAPT-VQE screening (reference ADAPT use of batch_grad: theta = 0, l = psi,
    r = H psi, op/batchgrad.hpp:529-540): the commutator expectation of every
    spin-adapted pool generator = sum of its components' gradients; then the
    adjoint energy gradient of the 40-generator ansatz that made psi."""
    import torch
    from binsim_b200 import cuotf
    cfg = adapt_cfg(args)
    torch.cuda.set_device(0)
    ham, pool, op_idx, param_idx, th = adapt_problem(cfg)
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"], string_bits=64)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(ham, string_bits=64), cuotf.CuNetwork(pool.network, string_bits=64))
    dim = B.dim
    ref_idx, ref_val = np.array([B.hf_index()]), np.array([1.0])
    psi = torch.empty(dim, dtype=torch.float64, device="cuda")
    hpsi = torch.empty_like(psi)
    ngs = pool.network.ngs
    zeros = torch.zeros(ngs, dtype=torch.float64, device="cuda")
    grads = torch.empty(ngs, dtype=torch.float64, device="cuda")
    f.prepare_state(op_idx, param_idx, th, ref_idx, ref_val, psi)
    # generator gradient = sum over its components (products at theta = 0)
    comp_gen = np.zeros(ngs, np.int64)
    for gi, comps in enumerate(pool.components):
        comp_gen[comps] = gi
    comp_gen_t = torch.from_numpy(comp_gen).cuda()
    gen_grads = torch.zeros(len(pool.components), dtype=torch.float64, device="cuda")

    def screen():
        f.hvec(psi, hpsi)
        f.batchgrad(psi, hpsi, grads, zeros)
        gen_grads.zero_().index_add_(0, comp_gen_t, grads)
    # first call: builds the sigma plan and the theta = 0 route (pool classification,
    # hole tables, density scratch) outside the timed region
    t0 = time.time()
    f.hvec(psi, hpsi)
    f.batchgrad(psi, hpsi, grads, zeros)
    torch.cuda.synchronize()
    first_call_s = time.time() - t0
    steps, warm = max(1, args.steps), max(3, args.warmup)
    with Clocks(0) as clk:
        ms = timed_events(screen, steps, warm)
        ms_h = timed_events(lambda: f.hvec(psi, hpsi), steps, 1)
        ms_bg = timed_events(lambda: f.batchgrad(psi, hpsi, grads, zeros), steps, 1)
    launches = count_launches(screen)
    g = gen_grads.cpu().numpy()
    top = np.argsort(-np.abs(g))[:5]
    # adjoint gradient of the ansatz that made psi
    lv, rv = torch.empty_like(psi), torch.empty_like(psi)
    out = {}

    def adjoint():
        out["a"] = f.energy_grad(op_idx, param_idx, th, ref_idx, ref_val, lv, rv, ckpt_every=cfg["ckpt"])
    ms_adj = timed_events(adjoint, steps, 1)
    E, ga, _ = out["a"]
    density = None
    if args.pool_density:
        # the pair-list gradient beside the theta = 0 route: every theta 1e-300 sends
        # every group to the pair lists (the same work as at theta = 0, gradients equal
        # to rounding)
        tiny = torch.full_like(zeros, 1e-300)
        grads_p = torch.empty_like(grads)
        ms_pl = timed_events(lambda: f.batchgrad(psi, hpsi, grads_p, tiny), max(1, min(steps, 2)), 1)
        f.batchgrad(psi, hpsi, grads, zeros)
        torch.cuda.synchronize()
        a_, b_ = grads.cpu().numpy(), grads_p.cpu().numpy()
        # GEMM flops as launched: Tab (n^2 x n^2 over one-hole alpha x beta strings) and the
        # two same-spin tables (pairs x pairs over two-hole strings x the other spin's strings)
        from math import comb
        n_, na_, nb_ = cfg["norb"], cfg["na"], cfg["nb"]
        npair = n_ * (n_ - 1) // 2
        flops = 2.0 * (n_ * n_) ** 2 * comb(n_, na_ - 1) * comb(n_, nb_ - 1)
        flops += 2.0 * npair ** 2 * (comb(n_, na_ - 2) * comb(n_, nb_) if na_ >= 2 else 0)
        flops += 2.0 * npair ** 2 * (comb(n_, nb_ - 2) * comb(n_, na_) if nb_ >= 2 else 0)
        dmma = cuotf.fma_peak(dmma=True)
        kind, _, _ = cuotf.pool_plan(pool.network)
        density = {"ms": ms_bg, "pair_list_ms": ms_pl, "speedup_vs_pair_list": ms_pl / ms_bg,
                   "first_call_s": first_call_s, "gemm_flops": flops,
                   "tflops": flops / (ms_bg * 1e-3) / 1e12, "fp64_dmma_peak_tflops": dmma,
                   "frac_of_measured_dmma_peak": flops / (ms_bg * 1e-3) / 1e12 / dmma,
                   "general_groups": int((kind < 0).sum()),
                   "max_abs_diff_vs_pair_list": float(np.abs(a_ - b_).max()),
                   "max_abs_grad": float(np.abs(b_).max()),
                   "note": "batchgrad at theta = 0 takes the transition-density route; the pair lists are timed "
                           "with every theta = 1e-300"}
    res = {
        "metric": ADAPT_METRIC, "value": len(pool.components) / (ms * 1e-3), "unit": "generators/s", "n_gpus": 1,
        "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "replicas",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"ADAPT screening: {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, {dim:,} dets, "
                               f"UInt64 strings (ranked addressing), {ham.ngs} Hamiltonian groups, pool of "
                               f"{len(pool.components)} spin-adapted generalised singles/doubles ({ngs} components), "
                               f"state from {cfg['n_gen']} seeded generators, amplitudes N(0, {cfg['amp']}^2); one "
                               "step = H psi + every component's gradient at theta = 0 + the per-generator sums",
                   "dim": dim, "pool_generators": len(pool.components), "pool_components": ngs,
                   "hamiltonian_groups": int(ham.ngs)},
        "sigma_ms": ms_h, "batchgrad_ms": ms_bg,
        "top_generators": [{"label": [str(v) for v in pool.labels[int(i)]], "grad": float(g[int(i)])} for i in top],
        "adjoint": {"ms": ms_adj, "energy": E, "params": int(len(th)), "max_abs_grad": float(np.abs(ga).max())},
        "e2e": {"value": len(pool.components) / (ms * 1e-3), "unit": "generators/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(8 * len(pool.components)), "ms_per_step": ms,
                "note": "psi resident on the device between ADAPT iterations; the generator gradients are read back"},
        "gpu_launches": launches * steps if launches is not None else None,
        "clocks": clk.summary(),
    }
    if density is not None:
        res["pool_density"] = density
    if not args.no_cpu_baseline:
        cpu = run_cpu_adapt(args, ham, pool, psi.cpu().numpy(), hpsi.cpu().numpy(), grads.cpu().numpy())
        if cpu and "seconds" in cpu:
            res["cpu_baseline"] = {"value": len(pool.components) / cpu["seconds"], "unit": "generators/s",
                                   "cores": cpu["cores"], "kind": "port", "sample": cpu["sample"]}
            res["parity_vs_oracle"] = {"max_abs_diff": cpu["max_abs_diff"], "components_checked": cpu["checked"]}
    return res


def cpu_adapt_worker(args):
    """The oracle (C restatement of op/batchgrad.hpp over UInt64 strings with the
    reference's sorted-list string search) on a bounded sample of pool components
    and Hamiltonian groups; also checks the sampled components' GPU gradients."""
    from oracle.oracle import Oracle
    import pickle
    cfg = adapt_cfg(args)
    with open(args.adapt_state, "rb") as fh:
        st = pickle.load(fh)
    ham, pool = st["ham"], st["pool"]
    O = Oracle()
    Bo = O.basis(cfg["norb"], cfg["na"], cfg["nb"])
    psi, hpsi, gpu = st["psi"], st["hpsi"], st["grads"]
    ngs = pool.network.ngs
    stride = max(1, ngs // args.adapt_sample)
    keep = np.arange(0, ngs, stride)
    sub = subnetwork(pool.network, keep)
    No = O.network(sub)
    t0 = time.perf_counter()
    g = O.batchgrad(Bo, No, np.zeros(len(keep)), psi, hpsi)
    t_bg = (time.perf_counter() - t0) * ngs / len(keep)
    hstride = max(1, ham.ngs // args.adapt_sample)
    hkeep = np.arange(0, ham.ngs, hstride)
    Ho = O.network(subnetwork(ham, hkeep))
    t0 = time.perf_counter()
    O.hvec(Bo, Ho, psi)
    t_h = (time.perf_counter() - t0) * ham.ngs / len(hkeep)
    print(json.dumps({"seconds": t_bg + t_h, "max_abs_diff": float(np.abs(g - gpu[keep]).max()),
                      "checked": int(len(keep)), "bg_sample": int(len(keep)), "h_sample": int(len(hkeep)),
                      "t_batchgrad": t_bg, "t_hvec": t_h}))


def run_cpu_adapt(args, ham, pool, psi, hpsi, grads):
    import pickle
    import tempfile
    with tempfile.NamedTemporaryFile(suffix=".pkl", delete=False) as fh:
        pickle.dump({"ham": ham, "pool": pool, "psi": psi, "hpsi": hpsi, "grads": grads}, fh)
        path = fh.name
    try:
        out, cores = run_cpu_worker(args, ["--workload", "adapt", "--adapt-state", path,
                                           "--adapt-sample", str(args.adapt_sample),
                                           "--adapt-norb", str(args.adapt_norb)])
    finally:
        os.unlink(path)
    if out is None or "seconds" not in out:
        return out
    out["cores"] = cores
    out["sample"] = (f"oracle (C restatement, UInt64 strings, OpenMP) on a stride of the {args.adapt_norb}-orbital pool "
                     f"giving {out['bg_sample']} components and {out['h_sample']} Hamiltonian "
                     f"groups, times scaled by the group counts; the reference's basis library is UInt32-only, "
                     f"so no reference code runs this space; {cpu_model()}")
    return out


def cpu_davidson_worker(args):
    from binsim_b200 import network as nw
    from oracle.oracle import RefLibs, ref_available
    if not ref_available():
        print(json.dumps({"unavailable": "oracle/_ref not built"}))
        return
    cfg = DAV_CFGS[args.dav_size]
    R = RefLibs()
    net = nw.hamiltonian_network(cfg["norb"], seed=cfg["seed"])
    b, dim = R.basis(cfg["norb"], cfg["na"], cfg["nb"])
    n = R.network(net)
    d = R.diag_elems(b, n, dim)
    v0 = np.zeros(dim)
    v0[R.det_index(b, (1 << cfg["na"]) - 1, (1 << cfg["nb"]) - 1, dim)] = 1.0
    t0 = time.perf_counter()
    e, _, it, ns = R.davidson(b, n, v0, d, tol=DAV_TOL, ncv=cfg["ncv"], maxspace=cfg["maxspace"])
    sec = time.perf_counter() - t0
    out = {"seconds": sec, "energy_at_tol": e, "iterations": it, "sigma": ns}
    if args.dav_oracle:
        e2, _, _, _ = R.davidson(b, n, v0, d, tol=1e-9, ncv=cfg["ncv"], maxspace=cfg["maxspace"])
        out["energy"] = e2
    print(json.dumps(out))


def cpu_vqe_worker(args):
    """The reference's energy_objective (jl/vqe.jl:1-21) on libotf_native: a
    bounded prefix of the forward expm sweep and of the backgrad sweep, one full
    hvec, scaled to the whole component sequence."""
    import ctypes as C
    from oracle.oracle import RefLibs, ref_available
    if not ref_available():
        print(json.dumps({"unavailable": "oracle/_ref not built"}))
        return
    cfg = VQE_CFG
    R = RefLibs()
    ham, pool, op_idx, param_idx, th = vqe_problem(cfg)
    b, dim = R.basis(cfg["norb"], cfg["na"], cfg["nb"])
    hn, pn = R.network(ham), R.network(pool.network)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    lv = np.zeros(dim)
    lv[R.det_index(b, (1 << cfg["na"]) - 1, (1 << cfg["nb"]) - 1, dim)] = 1.0
    rv = np.zeros(dim)
    k = min(len(op_idx), args.vqe_sample)
    t0 = time.perf_counter()
    for i in range(k):
        R.otf.expm_contract_otf_f64(b, pn, int(op_idx[i]), float(th[param_idx[i]]), P(lv))
    t_exp = time.perf_counter() - t0
    t0 = time.perf_counter()
    R.otf.hvec_gather_contract_otf_f64(b, hn, P(lv), P(rv))
    t_h = time.perf_counter() - t0
    t0 = time.perf_counter()
    for i in reversed(range(k)):
        R.otf.backgrad_contract_otf_f64(b, pn, int(op_idx[i]), float(th[param_idx[i]]), P(lv), P(rv))
    t_bg = time.perf_counter() - t0
    n = len(op_idx)
    sec = (t_exp + t_bg) * n / k + t_h
    print(json.dumps({"seconds": sec, "sample_components": k, "components": n, "t_expm": t_exp, "t_backgrad": t_bg,
                      "t_hvec": t_h}))


def run_cpu_worker(args, extra):
    cores = physical_cores()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close", OMP_PLACES="cores")
    env.pop("CUDA_VISIBLE_DEVICES", None)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker"] + extra
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0:
        log(r.stderr[-2000:])
        return None, cores
    return json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1]), cores


def run_cpu_vqe(args):
    out, cores = run_cpu_worker(args, ["--workload", "vqe", "--vqe-sample", str(args.vqe_sample)])
    if out is None or "seconds" not in out:
        return out
    out["cores"] = cores
    out["sample"] = (f"reference energy_objective on libotf_native: first {out['sample_components']} of "
                     f"{out['components']} components of the expm and backgrad sweeps, scaled by the component count, "
                     f"plus one full hvec; {cpu_model()}")
    return out


def run_cpu_davidson(args, oracle_energy=True):
    out, cores = run_cpu_worker(args, ["--workload", "davidson", "--dav-size", args.dav_size] +
                                (["--dav-oracle"] if oracle_energy else []))
    if out is None or "seconds" not in out:
        return out
    out["cores"] = cores
    out["sample"] = (f"whole solve: reference Davidson driver (jl/davidson.jl restated over libdiag) with "
                     f"libotf_native sigma, residual tol {DAV_TOL}, {out.get('iterations')} iterations; {cpu_model()}")
    return out


def physical_cores():
    try:
        import psutil
        return psutil.cpu_count(logical=False) or os.cpu_count()
    except Exception:
        return os.cpu_count()


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default="sigma", choices=["sigma", "davidson", "vqe", "adapt", "block", "bands"])
    ap.add_argument("--block-size", default="16o", choices=sorted(BLOCK_CFGS))
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--adapt-state", default="")
    ap.add_argument("--adapt-sample", type=int, default=400)
    ap.add_argument("--adapt-norb", type=int, default=ADAPT_CFG["norb"])
    ap.add_argument("--pool-density", action="store_true",
                    help="adapt: also time the pair-list pool gradient and compare it with the theta = 0 "
                         "density route batchgrad takes")
    ap.add_argument("--dav-size", default="12o", choices=sorted(DAV_CFGS))
    ap.add_argument("--sigma-size", default="16o", choices=sorted(SIGMA_CFGS))
    ap.add_argument("--dav-oracle", action="store_true")
    ap.add_argument("--vqe-sample", type=int, default=200)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--cpu-reps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-worker", action="store_true")
    ap.add_argument("--cpu-full", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--cpu-out", default="", help=argparse.SUPPRESS)
    ap.add_argument("--no-targets", action="store_true",
                    help="default line: skip the Davidson (12 and 16 orbitals) and VQE (14 orbitals) figures")
    args = ap.parse_args()

    if args.cpu_worker:
        {"sigma": cpu_worker, "davidson": cpu_davidson_worker, "vqe": cpu_vqe_worker,
         "adapt": cpu_adapt_worker}[args.workload](args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        reference_arm(args)
        return

    if args.workload != "sigma":
        # Davidson and VQE are single-state solves: one GPU (further ranks would be replicas)
        if rank != 0:
            return
        result = {"davidson": gpu_davidson, "vqe": gpu_vqe, "adapt": gpu_adapt,
                  "block": gpu_block_davidson, "bands": gpu_bands}[args.workload](args)
        if args.workload == "vqe" and not args.no_cpu_baseline:
            cpu = run_cpu_vqe(args)
            if cpu and "seconds" in cpu:
                result["cpu_baseline"] = {"value": 1.0 / cpu["seconds"], "unit": "evals/s", "cores": cpu["cores"],
                                          "kind": "reference", "sample": cpu["sample"]}
        print(json.dumps(result))
        return

    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    try:
        result, net = gpu_sigma(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline:
            import shutil
            import tempfile
            tmp = tempfile.mkdtemp(prefix="bsim_ref_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
            try:
                res, cores = run_cpu_baseline(args, out_dir=tmp if world == 1 else None)
                if res and "value" in res:
                    result["cpu_baseline"] = {
                        "value": res["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                        "sample": f"reference libotf_native sigma on every {res['stride']}-th off-diagonal group "
                                  f"({res['sample_pairs']:.3e} of {res['full_pairs']:.3e} pair updates, "
                                  f"{res['sample_seconds']:.1f} s), scaled by exact pair counts; {cpu_model()}"}
                    if world == 1:
                        result["parity_vs_reference"] = sampled_parity(args, net, tmp)
                else:
                    result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                                              "sample": "unavailable: oracle/_ref not built"}
            finally:
                shutil.rmtree(tmp, ignore_errors=True)
        if world == 1 and not args.no_targets and args.sigma_size == "16o":
            result["targets"] = task_targets(args)
        print(json.dumps(result))


REF_SIGMA_SECONDS = 150.0


def reference_gpu_sigma(cfg):
    """The reference's own GPU library (src/extern/cuotf.cu built unchanged for
    sm_100a into oracle/_ref/libcuotf_ref.so) on the same sigma, driven through
    its C-ABI with the reference's host handles, as jl/cuda/cunetwork.jl does."""
    try:
        from oracle import time_ref_gpu
        r = time_ref_gpu.time_sigma(cfg["norb"], compare=False)
        return {"seconds_per_sigma": r["reference_gpu_s"], "value": 1.0 / r["reference_gpu_s"], "unit": UNIT,
                "reps": r["reps"], "what": r["what"],
                "note": "reference libcuotf hvec_cuda, legacy default stream, wall time around reps with "
                        "sync_device_cuda"}
    except Exception as e:   # library not built, or no GPU
        return {"unavailable": f"{type(e).__name__}: {str(e)[:200]}"}


def reference_arm(args):
    """The reference's own CPU implementation of the workload, on the host cores."""
    base = {"impl": "reference", "n_gpus": args.gpus, "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    if args.workload == "sigma":
        # whole sigmas of the full network, as many as fit in REF_SIGMA_SECONDS
        # (at least one; ~70 s each at 16 orbitals on 16 cores)
        res, cores = run_cpu_baseline(args, full=True, seconds=REF_SIGMA_SECONDS, reps=max(1, args.steps))
        if res is None or "unavailable" in res:
            print(json.dumps({"impl": "reference", "unavailable": (res or {}).get("unavailable", "worker failed")}))
            return
        cfg = SIGMA_CFGS[args.sigma_size]
        sample = (f"reference libotf_native hvec_gather_contract_otf_f64 over the whole network ({res['sample_groups']} "
                  f"groups, {res['full_pairs']:.3e} pair updates per sigma), {res['reps']} sigma(s) measured "
                  f"(median), {res['threads']} OpenMP threads; {cpu_model()}")
        line = dict(base, metric=METRIC, value=res["value"], unit=UNIT, steps=res["reps"],
                    requested_steps=args.steps,
                    warmup="1 untimed sigma of every 200th group (threads, first touch)",
                    ms_per_step=res["sec_per_sigma"] * 1e3, higher_is_better=True, scaling="strong",
                    config={"workload": f"sigma microbenchmark: H*c, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b, "
                                        "seeded synthetic integrals (seed 0), c ~ N(0,1) normalised"},
                    seconds_per_sigma=res["times"],
                    cpu_baseline={"value": res["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                                  "sample": sample},
                    e2e={"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        if args.gpus == 1:
            line["reference_gpu"] = reference_gpu_sigma(cfg)
    elif args.workload == "davidson":
        if args.dav_size != "12o":
            print(json.dumps({"impl": "reference", "unavailable": "the CPU reference solve of the 16-orbital space "
                                                                  "takes tens of minutes; timed on 12 orbitals only"}))
            return
        cpu = run_cpu_davidson(args, oracle_energy=False)
        if not cpu or "seconds" not in cpu:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
            return
        cfg = DAV_CFGS[args.dav_size]
        line = dict(base, metric=DAV_METRIC, value=cpu["seconds"], unit="s", steps=1, warmup=0,
                    ms_per_step=cpu["seconds"] * 1e3, higher_is_better=False, scaling="strong",
                    config={"workload": f"FCI Davidson, lowest root, {cfg['norb']} orbitals {cfg['na']}a+{cfg['nb']}b"},
                    cpu_baseline={"value": cpu["seconds"], "unit": "s", "cores": cpu["cores"], "kind": "reference",
                                  "sample": cpu["sample"]},
                    e2e={"value": cpu["seconds"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    elif args.workload == "block":
        print(json.dumps({"impl": "reference", "unavailable": "the reference's Davidson driver (jl/davidson.jl) follows "
                                                              "one root; it has no block solver for the lowest 2 roots, "
                                                              "and one reference sigma at 18 orbitals takes ~2,900 s on "
                                                              "the host cores"}))
        return
    elif args.workload == "bands":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no sharded sigma (single process, "
                                                              "one device)"}))
        return
    elif args.workload == "adapt":
        print(json.dumps({"impl": "reference", "unavailable": "the reference's basis library is UInt32-only and its "
                                                              "dense string map overflows at 36 orbitals "
                                                              "(basis.hpp:271); the GPU line carries the oracle port "
                                                              "as cpu_baseline"}))
        return
    else:
        cpu = run_cpu_vqe(args)
        if not cpu or "seconds" not in cpu:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
            return
        v = 1.0 / cpu["seconds"]
        line = dict(base, metric=VQE_METRIC, value=v, unit="evals/s", steps=1, warmup=0,
                    ms_per_step=cpu["seconds"] * 1e3, higher_is_better=True, scaling="replicas",
                    config={"workload": "VQE energy + gradient, 14 orbitals 7a+7b, 2000 generators"},
                    cpu_baseline={"value": v, "unit": "evals/s", "cores": cpu["cores"], "kind": "reference",
                                  "sample": cpu["sample"]},
                    e2e={"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line))


if __name__ == "__main__":
    main()
