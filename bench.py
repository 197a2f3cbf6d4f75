"""Benchmark of the reordered-SpMV path on B200.

Workload (default): R-MAT scale 22 (4,194,304 rows), edge factor 16,
a=.57 b=.19 c=.19, seed 1, duplicates merged, FP32 values and x uniform in
[-1, 1]; pGOrder (gorder4, window 5) permutation applied on the GPU; one step =
one MERBIT FP32 SpMV (SIGMA 14, 256 threads) of the reordered matrix with the
matrix and x resident in HBM. The streamed matrix (~0.5 GB) is larger than
L2, so no flush is needed between steps.

metric: achieved HBM GB/s = algorithmic bytes per SpMV
        4(n+1) + 8 nnz + 4n (x) + 4n (y), divided by the device time.
e2e:    the same metric through the C-ABI with host buffers: each step copies
        x from pinned host memory, permutes it (x' = P x), runs the SpMV,
        un-permutes y (y = P^T y') and copies y back to pinned host memory.
--impl reference: the CPU baseline of this path (the reference has no CPU
        SpMV; this is the OpenMP FP32 CSR SpMV restatement from oracle/) on all
        host cores, same matrix, metric and unit.

Multi-GPU (torchrun): every rank runs the same workload on its own GPU
(replicas, weak scaling); value = sum over ranks of the bytes / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "matrix-reorder_b200"))

HBM_FALLBACK_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def spmv_bytes(n: int, nnz: int, val_bytes: int = 4) -> int:
    return 4 * (n + 1) + nnz * (4 + val_bytes) + 4 * n + 4 * n


def traffic_from_profiles(name: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/<name>)."""
    p = os.path.join(REPO, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_spmv:"):
                return int(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clk", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.out.close()
        rows = [r.split(",") for r in open(self.out.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(rows)}


def build_workload(M, scale: int, ef: int, seed: int, cache_dir: str | None):
    """R-MAT + pGOrder permutation (host), cached in cache_dir for other ranks."""
    key = f"rmat_s{scale}_ef{ef}_seed{seed}"
    if cache_dir:
        f = os.path.join(cache_dir, key + ".npz")
        if os.path.exists(f):
            d = np.load(f)
            return d["rp"], d["ci"], d["v"], d["x"], d["perm"], {"cached": True}
    t0 = time.time()
    rp, ci, v = M.gen_rmat(scale=scale, edge_factor=ef, seed=seed)
    t_gen = time.time() - t0
    n = rp.size - 1
    x = M.uniform(n, seed=seed + 1000)
    t0 = time.time()
    new2old = M.pgorder(rp, ci, vsize=0, width=5)
    t_ord = time.time() - t0
    perm = np.empty(n, np.int32)
    perm[new2old] = np.arange(n, dtype=np.int32)
    if cache_dir:
        np.savez(os.path.join(cache_dir, key + ".npz"), rp=rp, ci=ci, v=v, x=x, perm=perm)
    return rp, ci, v, x, perm, {"gen_s": round(t_gen, 2), "pgorder_s": round(t_ord, 2),
                                "pgorder_vsize": M.pgorder_width(n, ci.size)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    """CPU baseline arm: OpenMP FP32 CSR SpMV restatement on all host cores."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import mrb200 as M
    import pyoracle as O

    rp, ci, v, x, perm, _ = build_workload(M, args.scale, args.edge_factor, args.seed, None)
    # the same reordered matrix the GPU arm runs
    brp, bci, bv = O.permute_csr(rp, ci, v, perm)
    xp = np.empty_like(x)
    xp[perm] = x
    n, nnz = brp.size - 1, bci.size
    y = np.empty(n, np.float32)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        O.spmv_f32_omp(brp, bci, bv, xp, y, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        used = O.spmv_f32_omp(brp, bci, bv, xp, y, threads)
    dt = time.perf_counter() - t0
    b = spmv_bytes(n, nnz)
    val = b * args.steps / dt / 1e9
    line = {
        "metric": "spmv_hbm_gbs", "value": round(val, 2), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"rmat_s{args.scale}_ef{args.edge_factor} pGOrder-reordered CSR SpMV", "n_rows": n,
                   "nnz": nnz, "seed": args.seed},
        "cpu_baseline": {"value": round(val, 2), "unit": "GB/s", "cores": used, "kind": "port",
                         "sample": f"{args.steps} full FP32 CSR SpMVs of the reordered matrix (OpenMP restatement; "
                                   "the reference has no CPU SpMV)"},
        "e2e": {"value": round(val, 2), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def time_cpu_baseline(brp, bci, bv, xp, budget_s: float = 10.0):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as O
    n = brp.size - 1
    y = np.empty(n, np.float32)
    threads = os.cpu_count() or 1
    O.spmv_f32_omp(brp, bci, bv, xp, y, threads)  # warm
    reps, t0 = 0, time.perf_counter()
    while True:
        used = O.spmv_f32_omp(brp, bci, bv, xp, y, threads)
        reps += 1
        if time.perf_counter() - t0 >= budget_s or reps >= 200:
            break
    dt = time.perf_counter() - t0
    return spmv_bytes(n, bci.size) * reps / dt / 1e9, used, reps


def run_ours(args):
    import torch
    import mrb200 as M

    ws, rank, local = dist_env()
    dist = ws > 1
    if dist:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cache = tempfile.gettempdir() if dist else None
    if dist:
        if rank == 0:
            build_workload(M, args.scale, args.edge_factor, args.seed, cache)
        tdist.barrier()
    rp, ci, v, x, perm, setup = build_workload(M, args.scale, args.edge_factor, args.seed, cache)
    n, nnz = rp.size - 1, ci.size
    st = torch.cuda.current_stream()
    d = lambda a: torch.from_numpy(a).to(dev)
    rp_d, ci_d, v_d, x_d, perm_d = d(rp), d(ci), d(v), d(x), d(perm)
    A = M.view(rp_d, ci_d, v_d)
    # device permutation B = P A P^T
    brp = torch.empty_like(rp_d)
    bci = torch.empty_like(ci_d)
    bv = torch.empty_like(v_d)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    M.permute_csr(A, perm_d, brp, bci, bv)
    torch.cuda.synchronize()
    setup["permute_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    B = M.view(brp, bci, bv)
    xp = torch.empty_like(x_d)
    M.permute_vector(perm_d, x_d, xp, inverse=False)
    yp = torch.empty_like(x_d)
    hub_cache = True
    if args.tune:
        # the project's autotuner picks sigma (tile = 32 x sigma merge items),
        # threads per CTA and the hub cache on this matrix (setup, untimed)
        t0 = time.perf_counter()
        args.sigma, args.block, flags, _ = M.autotune(B, xp, yp, reps=5)
        hub_cache = (flags & 1) == 0
        setup["autotune_s"] = round(time.perf_counter() - t0, 2)
    t0 = time.perf_counter()
    plan = M.MerbitPlan(B, sigma=args.sigma, block=args.block, hub_cache=hub_cache)
    torch.cuda.synchronize()
    setup["plan_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    bytes_step = spmv_bytes(n, nnz)

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    # companion numbers (untimed for the headline): CSR and MERBIT before/after reordering
    details = {}
    if not args.quick:
        yd = torch.empty_like(x_d)
        details["csr_orig_gbs"] = round(bytes_step / timed(lambda: M.spmv_csr(A, x_d, yd), 50, 5) / 1e6, 1)
        details["csr_reordered_gbs"] = round(bytes_step / timed(lambda: M.spmv_csr(B, xp, yp), 50, 5) / 1e6, 1)
        plan_a = M.MerbitPlan(A, sigma=args.sigma, block=args.block)
        details["merbit_orig_gbs"] = round(bytes_step / timed(lambda: plan_a.spmv(x_d, yd), 50, 5) / 1e6, 1)
        plan_a.close()
        plan_nh = M.MerbitPlan(B, sigma=args.sigma, block=args.block, hub_cache=False)
        details["merbit_reordered_no_hub_cache_gbs"] = round(
            bytes_step / timed(lambda: plan_nh.spmv(xp, yp), 50, 5) / 1e6, 1)
        plan_nh.close()
        # the reference's fixed configuration: SIGMA 14, 256 threads (src/class.cu:1409-1410)
        plan_r = M.MerbitPlan(B, sigma=14, block=256, hub_cache=False)
        details["merbit_reordered_sigma14_block256_gbs"] = round(
            bytes_step / timed(lambda: plan_r.spmv(xp, yp), 50, 5) / 1e6, 1)
        plan_r.close()
    inf = plan.info()
    details["hub_columns"] = inf.hub_columns
    details["hub_coverage"] = round(inf.hub_coverage, 4)

    # ---- headline: K MERBIT SpMVs on the reordered matrix ----
    for _ in range(args.warmup):
        plan.spmv(xp, yp)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.15)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        plan.spmv(xp, yp)
    e1.record(st)
    torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    clocks = sampler.stop()
    ms_total = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms_total], device=dev)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    value = ws * bytes_step * args.steps / (ms_total / 1e3) / 1e9

    # ---- e2e: host buffers through the C-ABI ----
    k_e2e = max(1, min(args.steps, args.e2e_steps))
    x_h = torch.from_numpy(x).pin_memory()
    y_h = torch.empty(n, dtype=torch.float32).pin_memory()
    x_in = torch.empty_like(x_d)
    y_out = torch.empty_like(x_d)

    def e2e_step():
        x_in.copy_(x_h, non_blocking=True)
        M.permute_vector(perm_d, x_in, xp, inverse=False)
        plan.spmv(xp, yp)
        M.permute_vector(perm_d, yp, y_out, inverse=True)
        y_h.copy_(y_out, non_blocking=True)

    for _ in range(3):
        e2e_step()
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(st)
    for _ in range(k_e2e):
        e2e_step()
    f1.record(st)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1)
    if dist:
        t = torch.tensor([ms_e2e], device=dev)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_val = ws * bytes_step * k_e2e / (ms_e2e / 1e3) / 1e9
    # self-check of the e2e result: against the plain CSR kernel on the
    # original (unreordered) matrix
    y_csr = torch.empty_like(x_d)
    M.spmv_csr(A, x_d, y_csr)
    torch.cuda.synchronize()
    got, ref = y_h.to(dev).double(), y_csr.double()
    check = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))

    peak, peak_kind = peaks()
    achieved = bytes_step / (ms_step / 1e3) / 1e9
    traffic = traffic_from_profiles(f"merbit_spmv_rmat_s{args.scale}.md")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes_per_spmv": bytes_step,
                "kernels_timed": "one MERBIT SpMV (persistent kernel with fused fix-up, or grid kernel + fix-up)"}

    cpu = None
    if rank == 0 and not args.quick and args.cpu_budget > 0:
        brp_h, bci_h, bv_h = brp.cpu().numpy(), bci.cpu().numpy(), bv.cpu().numpy()
        gbs, cores, reps = time_cpu_baseline(brp_h, bci_h, bv_h, xp.cpu().numpy(), args.cpu_budget)
        cpu = {"value": round(gbs, 2), "unit": "GB/s", "cores": cores, "kind": "port",
               "sample": f"{reps} full FP32 CSR SpMVs of the same reordered matrix (OpenMP restatement; "
                         "the reference has no CPU SpMV)"}

    plan.close()
    if rank == 0:
        line = {
            "metric": "spmv_hbm_gbs", "value": round(value, 1), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"rmat_s{args.scale}_ef{args.edge_factor} pGOrder-reordered MERBIT FP32 SpMV",
                       "n_rows": n, "nnz": nnz, "seed": args.seed, "sigma": args.sigma, "block": args.block,
                       "hub_cache": bool(hub_cache), "tuned": bool(args.tune),
                       "parallelism": f"replicas x{ws}",
                       "l2": "inputs larger than L2 (matrix stream ~%d MB per step)" % (bytes_step // 2**20)},
            "roofline": roofline,
            "e2e": {"value": round(e2e_val, 1), "unit": "GB/s", "h2d_bytes_per_step": 4 * n,
                    "d2h_bytes_per_step": 4 * n, "steps": k_e2e, "ms_per_step": round(ms_e2e / k_e2e, 4),
                    "rel_l2_vs_fp64": check},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": 2 * args.steps,
            "details": {**details, **setup},
        }
        print(json.dumps(line), flush=True)
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sigma", type=int, default=14)
    ap.add_argument("--block", type=int, default=1024)
    ap.add_argument("--e2e-steps", type=int, default=400)
    ap.add_argument("--cpu-budget", type=float, default=8.0, help="seconds of CPU-baseline timing")
    ap.add_argument("--quick", action="store_true", help="skip companion numbers and CPU baseline")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="use --sigma/--block instead of the autotuner")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
