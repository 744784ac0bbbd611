"""Benchmark of the batched solver hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the hot path over one batch: plain LU with partial
pivoting plus the solve (gesv: A <- L\\U, B <- X, pivots, info) in float64 on
(65,536 x 64 x 64) general matrices with 4 right-hand sides, kappa log-uniform
in [1e1, 1e8] and 5% of the matrices with one zeroed column (the n=64 case of
the plain-LU benchmark configuration). Inputs are synthetic, built on the
device with the reference's generator construction, and larger than L2.

The ours arm prints one JSON line: device-resident throughput (value), the
end-to-end throughput of the host-pointer C-ABI call with pinned host buffers
(e2e), the roofline of the kernel, the CPU baseline (the reference library
compiled from its sources, all host threads, a bounded sample) and the SM
clocks sampled during the timed region. ``--impl reference`` times only the
reference's own CPU implementation on the same workload.
"""
import argparse
import ctypes as C
import importlib
import json
import os
import pathlib
import re
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
PKG_NAME = "tinysolverdx-batched-small-matrix-cholesky-lu-with-numerical_b200"
METRIC = "batched solves/s at n=32/64: bf16+IR vs plain fp64 at equal backward error"

WORKLOADS = {
    # name: (kind, n, batch, nrhs, dtype, kappa_lo, kappa_hi, zero_col_frac)
    "gesv_f64_n64": ("gesv", 64, 65536, 4, "f64", 1e1, 1e8, 0.05),
    "gesv_f64_n32": ("gesv", 32, 262144, 4, "f64", 1e1, 1e8, 0.05),
    "gesv_f32_n64": ("gesv", 64, 65536, 4, "f32", 1e1, 1e8, 0.05),
    "gesv_f32_n32": ("gesv", 32, 262144, 4, "f32", 1e1, 1e8, 0.05),
    "posv_f64_n16": ("posv", 16, 65536, 1, "f64", 1e1, 1e6, 0.0),
}


def describe(name):
    kind, n, batch, nrhs, dt, klo, khi, zf = WORKLOADS[name]
    what = "LU with partial pivoting + solve (gesv)" if kind == "gesv" else "Cholesky + solve (posv)"
    return {"workload": f"{what}, {dt}, n={n}, batch {batch}, {nrhs} RHS, kappa log-uniform [{klo:g},{khi:g}]"
                        + (f", {zf:.0%} with one zeroed column" if zf else ""),
            "kind": kind, "n": n, "batch_per_gpu": batch, "nrhs": nrhs,
            "l2": "inputs larger than L2 (each step factors a fresh copy of the input stack)"}


def algorithmic_bytes(kind, n, nrhs, s):
    """Bytes one solve must move: read A, write the factor, read B, write X, piv, info."""
    b = 2 * n * n * s + 2 * n * nrhs * s + 4
    return b + (4 * n if kind == "gesv" else 0)


def flops(kind, n, nrhs):
    f = (2 * n ** 3 / 3) if kind == "gesv" else (n ** 3 / 3)
    return f + 2 * n * n * nrhs


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(name):
    """dram bytes per launch recorded from an ncu capture in profiles/ (or None)."""
    p = ROOT / "profiles" / f"{name}_ncu.md"
    if not p.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


# ---------------------------------------------------------------- clocks (NVML)
class ClockSampler:
    """Samples SM clock and throttle reasons every few ms while the timed region runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle"}

    def __init__(self, index):
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max = None
        self.samples, self.reasons = [], set()
        self._stop = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, nm in self.REASONS.items():
                    if r & bit and nm != "gpu_idle":
                        self.reasons.add(nm)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        med = float(np.median(self.samples)) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max, "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- CPU reference
def cpu_reference(kind, n, nrhs, dt, seed, budget_s=12.0):
    """Times the reference library (compiled from its sources) on a bounded sample
    of the workload with all host threads. Returns (solves/s, threads, sample)."""
    from oracle.oracle import Oracle, ref_available, PORT_LIB
    kindlib = "reference" if ref_available() else "port"
    O = Oracle(kindlib)
    threads = os.cpu_count() or 1
    try:
        threads = len(os.sched_getaffinity(0))
    except Exception:
        pass
    O.set_num_threads(threads)
    M = importlib.import_module(PKG_NAME + ".matrices")
    rng = np.random.default_rng(seed)
    dtype = np.float64 if dt == "f64" else np.float32
    sample = 2048
    gen = M.general if kind == "gesv" else M.spd
    A0 = gen(rng, sample, n, M.log_uniform(rng, sample, 1e1, 1e8)).astype(dtype)
    B0 = rng.standard_normal((sample, n, nrhs)).astype(dtype)
    lib = O.lib
    s = "d" if dt == "f64" else "f"
    best, total, reps = 0.0, 0.0, 0
    piv = np.zeros((sample, n), np.int32)
    info = np.zeros(sample, np.int32)
    while total < budget_s and reps < 50:
        A, B = A0.copy(), B0.copy()
        t0 = time.perf_counter()
        if kindlib == "reference":
            if kind == "gesv":
                fn = getattr(lib, f"ref_gesv_batched_{s}")
                fn(A.ctypes.data_as(C.c_void_p), n, sample, B.ctypes.data_as(C.c_void_p), nrhs,
                   piv.ctypes.data_as(C.c_void_p), info.ctypes.data_as(C.c_void_p), 0)
            else:
                fn = getattr(lib, f"ref_posv_batched_{s}")
                fn(A.ctypes.data_as(C.c_void_p), n, sample, B.ctypes.data_as(C.c_void_p), nrhs,
                   info.ctypes.data_as(C.c_void_p), 0)
        else:
            (O.gesv if kind == "gesv" else O.posv)(A, B)
        dt_ = time.perf_counter() - t0
        total += dt_
        reps += 1
        best = max(best, sample / dt_)
        if dt_ < 0.25 and sample * 4 <= (1 << 15):
            # grow the sample until one call is long enough to time
            sample *= 4
            A0 = np.concatenate([A0] * 4)
            B0 = np.concatenate([B0] * 4)
            piv = np.zeros((sample, n), np.int32)
            info = np.zeros(sample, np.int32)
    return best, threads, kindlib, f"{sample} matrices per call, best of {reps} calls (Backend::Auto)"


# ---------------------------------------------------------------- GPU arm
def make_inputs(torch, kind, n, batch, nrhs, dtype, klo, khi, zf, seed, device):
    M = importlib.import_module(PKG_NAME + ".matrices")
    A = M.torch_stack("general" if kind == "gesv" else "spd", n, batch, klo, khi, seed, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 1)
    if zf > 0:
        pick = torch.rand(batch, generator=g, device=device) < zf
        cols = torch.randint(0, n, (batch,), generator=g, device=device)
        idx = torch.nonzero(pick).flatten()
        A[idx, :, cols[idx]] = 0.0
    B = torch.randn(batch, n, nrhs, generator=g, device=device, dtype=torch.float64)
    return A.to(dtype).contiguous(), B.to(dtype).contiguous()


def run_ours(a):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)
    capi = importlib.import_module(PKG_NAME + ".capi")
    kind, n, batch, nrhs, dt, klo, khi, zf = WORKLOADS[a.workload]
    if a.batch:
        batch = a.batch
    dtype = torch.float64 if dt == "f64" else torch.float32
    s = 8 if dt == "f64" else 4
    A0, B0 = make_inputs(torch, kind, n, batch, nrhs, dtype, klo, khi, zf, 1234 + rank, device)
    pool = max(2, min(a.steps + a.warmup, int(a.pool)))
    As = [A0.clone() for _ in range(pool)]
    Bs = [B0.clone() for _ in range(pool)]
    piv = torch.zeros(batch, n, dtype=torch.int32, device=device)
    info = torch.zeros(batch, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream()

    def step(i):
        j = i % pool
        if kind == "gesv":
            capi.gesv(As[j], Bs[j], piv, info, stream=stream)
        else:
            capi.posv(As[j], Bs[j], info, stream=stream)

    for i in range(a.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for i in range(a.steps):
            step(a.warmup + i)
        ev1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches = capi.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / a.steps
    value = world * batch / (ms_step * 1e-3)

    # --- end to end through the host-pointer C-ABI call (pinned host buffers) ---
    e2e = None
    if not a.skip_e2e:
        hA = torch.empty(A0.shape, dtype=dtype, pin_memory=True)
        hB = torch.empty(B0.shape, dtype=dtype, pin_memory=True)
        hP = torch.empty((batch, n), dtype=torch.int32, pin_memory=True)
        hI = torch.empty((batch,), dtype=torch.int32, pin_memory=True)
        A0h, B0h = A0.cpu(), B0.cpu()
        lib = capi.lib()
        sfx = "f64" if dt == "f64" else "f32"
        tot, reps = 0.0, max(3, min(a.steps, 10))
        for i in range(1 + reps):
            hA.copy_(A0h)
            hB.copy_(B0h)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if kind == "gesv":
                rc = getattr(lib, f"tsdx_cuda_gesv_batched_host_{sfx}")(capi.ptr(hA), n, batch, capi.ptr(hB), nrhs,
                                                                       capi.ptr(hP), capi.ptr(hI))
            else:
                rc = getattr(lib, f"tsdx_cuda_posv_batched_host_{sfx}")(capi.ptr(hA), n, batch, capi.ptr(hB), nrhs,
                                                                       capi.ptr(hI))
            capi.check(rc, "host call")
            e1.record()
            torch.cuda.synchronize()
            if i > 0:  # the first call allocates the device workspace
                tot += e0.elapsed_time(e1)
        e2e_ms = tot / reps
        if world > 1:
            t = torch.tensor([e2e_ms], device=device, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        h2d = batch * (n * n + n * nrhs) * s
        d2h = batch * (n * n + n * nrhs) * s + batch * 4 + (batch * n * 4 if kind == "gesv" else 0)
        e2e = {"value": world * batch / (e2e_ms * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
               "api": f"tsdx_cuda_{kind}_batched_host_{sfx} (include/tsdx_cuda.h), pinned host buffers"}

    peak, src = peaks()
    per_launch = batch * algorithmic_bytes(kind, n, nrhs, s)
    achieved = per_launch / (ms_step * 1e-3) / 1e9
    traffic = traffic_from_profiles(a.workload)
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": src,
            "algorithmic_bytes_per_launch": per_launch,
            "kernel": ("lu_blk_kernel" if kind == "gesv" else "chol_team_kernel") + f"<{dt},NP={n}>",
            "gflops": round(batch * flops(kind, n, nrhs) / (ms_step * 1e-3) / 1e9, 1)}

    cpu = None
    if rank == 0 and world == 1 and not a.skip_cpu:
        v, thr, kindlib, sample = cpu_reference(kind, n, nrhs, dt, 99)
        cpu = {"value": round(v, 1), "unit": "solves/s", "cores": thr, "kind": kindlib, "sample": sample}

    if rank == 0:
        cfg = describe(a.workload)
        cfg["batch_per_gpu"] = batch
        cfg["global_batch"] = world * batch
        cfg["parallelism"] = f"batch sharded over {world} GPU(s), no collective"
        out = {"metric": METRIC, "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": dt, "data": "synthetic", "config": cfg, "roofline": roof,
               "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "gpu_launches": int(launches)}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    kind, n, batch, nrhs, dt, *_ = WORKLOADS[a.workload]
    vals = []
    budget = max(2.0, 150.0 / max(1, a.steps + a.warmup))
    for i in range(a.warmup + a.steps):
        v, thr, kindlib, sample = cpu_reference(kind, n, nrhs, dt, 7 + i, budget_s=budget)
        if i >= a.warmup:
            vals.append(v)
    value = float(np.median(vals))
    cfg = describe(a.workload)
    cfg["global_batch"] = batch
    out = {"metric": METRIC, "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": round(batch / value * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": dt, "data": "synthetic", "config": cfg,
           "impl": "reference",
           "cpu_baseline": {"value": round(value, 1), "unit": "solves/s", "cores": thr, "kind": kindlib,
                            "sample": sample},
           "e2e": {"value": round(value, 1), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gesv_f64_n64", choices=sorted(WORKLOADS))
    ap.add_argument("--batch", type=int, default=0, help="override the workload's batch (profiling runs)")
    ap.add_argument("--pool", type=int, default=12, help="distinct input copies cycled through the steps")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    a = ap.parse_args(argv)
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
