#!/usr/bin/env python
"""Benchmark of the OTF operator path on B200.

Default workload (N=1): the sigma-build microbenchmark, sigma = H c on 16
spatial orbitals with 8 alpha + 8 beta electrons (12870^2 = 165,636,900
determinants, UInt32 strings), seeded synthetic integrals, c ~ N(0,1)
normalised.  One step = one sigma application.  FP64 is the headline; the
FP32-bulk/FP64-accumulate sigma is timed beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload sigma|davidson|vqe]

N > 1 (torchrun, one rank per GPU): the destination tiles of one sigma are
split into N contiguous row bands (strong scaling, input replicated on every
rank, no data-path collective); the step time is the max over ranks.

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

SIGMA_CFG = dict(norb=16, na=8, nb=8, seed=0)
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
    cfg = SIGMA_CFG
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
        dt, pr = run(keep)
        times.append(dt)
    dt = float(np.median(times))
    full = float(pairs.sum())
    sec_per_sigma = dt * full / pr
    print(json.dumps({
        "value": 1.0 / sec_per_sigma, "sec_per_sigma": sec_per_sigma, "sample_pairs": pr, "full_pairs": full,
        "sample_groups": int(len(keep)), "stride": int(stride), "sample_seconds": dt, "reps": len(times),
        "threads": int(os.environ.get("OMP_NUM_THREADS", "0")),
    }))


def run_cpu_baseline(args):
    try:
        import psutil
        cores = psutil.cpu_count(logical=False) or os.cpu_count()
    except Exception:
        cores = os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close", OMP_PLACES="cores")
    env.pop("CUDA_VISIBLE_DEVICES", None)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", "--cpu-seconds", str(args.cpu_seconds),
           "--cpu-reps", str(args.cpu_reps)]
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


def profile_traffic():
    """DRAM bytes per sigma launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "sigma_tile_kernel_16o8e.json")
    try:
        return json.load(open(p)).get("dram_bytes_per_launch")
    except Exception:
        return None


def gpu_sigma(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from binsim_b200 import cuotf, network as nw

    torch.cuda.set_device(local_rank)
    cfg = SIGMA_CFG
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
    ntiles = f.num_tiles()
    lo, hi = rank * ntiles // world, (rank + 1) * ntiles // world
    stream = torch.cuda.current_stream()

    def step(mixed=False):
        if world == 1:
            (f.hvec_mixed if mixed else f.hvec)(x, y)
        else:
            f.hvec_tiles(x, y, lo, hi, mixed=mixed)
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

    # e2e through the public API with host buffers: H2D c, sigma, D2H sigma
    xpin = torch.from_numpy(xh).pin_memory()
    ypin = torch.empty(dim, dtype=torch.float64).pin_memory()

    def e2e_step():
        x.copy_(xpin, non_blocking=True)
        step(False)
        ypin.copy_(y, non_blocking=True)
    ms_e2e = timed(e2e_step, max(1, args.steps // 2), 1)

    result = None
    if rank == 0:
        pk = peaks()
        hbm = pk.get("hbm_gbs")
        bytes_alg = dim * 16.0 / world        # c read + sigma written per launch (rows of this rank)
        achieved = bytes_alg / (ms * 1e-3) / 1e9
        traffic = profile_traffic()
        tflops = flops / world / (ms * 1e-3) / 1e12
        result = {
            "metric": METRIC, "value": 1000.0 / ms, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "sigma microbenchmark (config 1): H*c, 16 orbitals 8a+8b, 165,636,900 dets, "
                                   "UInt32 strings, seeded synthetic integrals (seed 0), c ~ N(0,1) normalised",
                       "dim": dim, "groups": int(net.ngs), "pair_updates": float(pairs.sum()),
                       "l2": "inputs larger than L2 (c and sigma are 1.33 GB each)",
                       "sharding": f"{world} row bands of one sigma" if world > 1 else "single GPU"},
            "e2e": {"value": 1000.0 / ms_e2e, "unit": UNIT, "h2d_bytes_per_step": dim * 8,
                    "d2h_bytes_per_step": dim * 8, "ms_per_step": ms_e2e},
            "mixed": {"value": 1000.0 / ms_mixed, "unit": UNIT, "ms_per_step": ms_mixed,
                      "dtype": "f32 bulk, f64 accumulate", "max_rel_err_vs_fp64": err_mixed,
                      "speedup_vs_fp64": ms / ms_mixed},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if hbm else None, "traffic": traffic,
                         "note": "compulsory bytes dim*(8+8) per sigma, of measured HBM copy peak; sigma is "
                                 "bound by FP64 issue and gathers, see compute_roofline"},
            "compute_roofline": {"bound": "fp64", "achieved": tflops, "peak": FP64_NOMINAL_TFLOPS,
                                 "unit": "TFLOP/s", "frac": tflops / FP64_NOMINAL_TFLOPS,
                                 "flops_per_sigma": flops, "note": "(2r+1) flops per connected pair; "
                                                                   "peak is the nominal FP64 figure"},
            "pair_updates_per_s": float(pairs.sum()) / (ms * 1e-3),
            "sigma_path": {"path": path[0], "reason": path[1], "residual_groups": path[2]},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
        }
    return result


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default="sigma", choices=["sigma"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--cpu-reps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-worker", action="store_true")
    args = ap.parse_args()

    if args.cpu_worker:
        cpu_worker(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        res, cores = run_cpu_baseline(args)
        if res is None or "unavailable" in res:
            print(json.dumps({"impl": "reference", "unavailable": (res or {}).get("unavailable", "worker failed")}))
            return
        sample = (f"reference libotf_native hvec_gather_contract_otf_f64 on every {res['stride']}-th off-diagonal "
                  f"group ({res['sample_groups']} groups, {res['sample_pairs']:.3e} of {res['full_pairs']:.3e} pair "
                  f"updates), scaled by exact pair counts; {cpu_model()}")
        line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": res["reps"], "warmup": 1, "ms_per_step": res["sec_per_sigma"] * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": "sigma microbenchmark (config 1): H*c, 16 orbitals 8a+8b"},
                "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    try:
        result = gpu_sigma(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline:
            res, cores = run_cpu_baseline(args)
            if res and "value" in res:
                result["cpu_baseline"] = {
                    "value": res["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                    "sample": f"reference libotf_native sigma on every {res['stride']}-th off-diagonal group "
                              f"({res['sample_pairs']:.3e} of {res['full_pairs']:.3e} pair updates, "
                              f"{res['sample_seconds']:.1f} s), scaled by exact pair counts; {cpu_model()}"}
            else:
                result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                                          "sample": "unavailable: oracle/_ref not built"}
        print(json.dumps(result))


if __name__ == "__main__":
    main()
