"""Benchmark of the batched solver hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the hot path over one batch. The default workload is
plain LU with partial pivoting plus the solve (gesv: A <- L\\U, B <- X, pivots,
info) in float64 on (65,536 x 64 x 64) general matrices with 4 right-hand sides,
kappa log-uniform in [1e1, 1e8] and 5% of the matrices with one zeroed column
(the n=64 case of the plain-LU benchmark configuration). Other workloads
(--workload): the n=32 / float32 variants and Cholesky n=16; ``ir_n64``, the
mixed-precision solve with per-matrix tiers from the learned selector and fp64
refinement (131,072 matrices, half SPD, kappa up to 1e12), next to plain fp64 on
the same inputs; ``stream_f32``, the uneven stream (1,048,576 matrices of mixed
order, kind and right-hand-side count in one graph-captured launch sequence); and
``selector``, the selector's evaluation set (1,048,576 matrices, n 8..64, kappa up
to 1e14) against fixed-tier policies and plain fp64. Inputs are synthetic, built
on the device with the reference's generator construction, and larger than L2.

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
SPECIAL = {
    "ir_n64": "mixed precision (selector-chosen fp16/bf16/fp32/fp64 tier per matrix) + fp64 iterative "
              "refinement with fp64 fallback, n=64, batch 131,072 (half SPD Cholesky, half general LU), "
              "1 RHS, kappa log-uniform [1e1,1e12]",
    "stream_f32": "uneven stream, fp32, 1,048,576 matrices, n uniform {2..64}, 50% SPD Cholesky / 50% LU, "
                  "kappa log-uniform [1e1,1e8], RHS count uniform {1,2,4,8}, one graph-captured launch sequence",
    "selector": "learned tier selector evaluation: 1,048,576 matrices, n uniform {8..64}, half SPD / half LU, "
                "kappa log-uniform [1e0,1e14], 1 RHS, selector tiers + fp64 refinement + fp64 fallback",
    "ir_fp32_n64": "fixed tier (--ir-tier, default fp32) factorization + fp64 refinement (tolerance 1e-15, at most 3 "
                   "corrections, fp64 fallback), n=64 general LU, batch 65,536, 1 RHS, kappa log-uniform [1e1,1e3]",
}


def describe(name, batch, world):
    """The config record of a dense workload; both arms print the same one."""
    kind, n, _, nrhs, dt, klo, khi, zf = WORKLOADS[name]
    what = "LU with partial pivoting + solve (gesv)" if kind == "gesv" else "Cholesky + solve (posv)"
    return {"workload": f"{what}, {dt}, n={n}, batch {batch}, {nrhs} RHS, kappa log-uniform [{klo:g},{khi:g}]"
                        + (f", {zf:.0%} with one zeroed column" if zf else ""),
            "kind": kind, "n": n, "batch_per_gpu": batch, "nrhs": nrhs, "global_batch": world * batch,
            "parallelism": f"batch sharded over {world} GPU(s), no collective",
            "l2": "inputs larger than L2; every warm-up and timed step works on its own untouched copy of the inputs"}


def _matrices():
    """The package's matrices.py (numpy only) loaded by path, so that the reference
    arm never imports the package, whose __init__ loads the GPU library."""
    mod = sys.modules.get("tsdx_bench_matrices")
    if mod is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("tsdx_bench_matrices", ROOT / PKG_NAME / "matrices.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules["tsdx_bench_matrices"] = mod
    return mod


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


def traffic_from_profiles(name, kernel):
    """dram bytes per launch of `kernel` on workload `name`, from the ncu summary
    profiles/<kernel>__<name>.md (or None when that kernel has no capture)."""
    p = ROOT / "profiles" / f"{kernel}__{name}.md"
    if p.exists():
        m = re.search(r"traffic_bytes_per_launch[^:]*:\s*([0-9.eE+]+)", p.read_text())
        if m:
            return float(m.group(1))
    return None


def dense_kernel(kind, n, dt):
    """(file stem, description) of the kernel the library launches for a dense
    workload: the routing of csrc/launch.cuh (TSDX_LU_KERNEL=smem or tc forces one
    LU kernel family)."""
    fam = os.environ.get("TSDX_LU_KERNEL", "")
    np_ = next(p for p in (4, 8, 16, 24, 32, 40, 48, 56, 64) if n <= p)
    if kind == "gesv" and dt == "f64" and np_ >= 32 and (fam == "tc" or (fam != "smem" and (np_ <= 48 or n % 2 == 0))):
        return "tc_kernel", f"tc_kernel<NP={np_}> (float64 LU, trailing update on the FP64 tensor cores)"
    if kind == "gesv" and dt == "f64" and np_ == 64:
        return "blk3_kernel", f"blk3_kernel<{dt},NP=64,LU> (two warps per matrix, look-ahead)"
    if kind == "gesv" and dt == "f64" and np_ >= 48:
        return "blk2_kernel", f"blk2_kernel<{dt},NP={np_},LU> (two warps per matrix)"
    return "blk_kernel", f"blk_kernel<{dt},NP={np_},{'LU' if kind == 'gesv' else 'Cholesky'}>"


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
def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def host_inputs(name, batch, seed, distinct=8192):
    """Host stacks of the workload's distribution for the CPU arms: `distinct` seeded
    matrices (kappa drawn per matrix, zeroed columns as configured) tiled up to the
    batch, and N(0,1) right-hand sides."""
    kind, n, _, nrhs, dt, klo, khi, zf = WORKLOADS[name]
    M = _matrices()
    rng = np.random.default_rng(seed)
    d = min(batch, distinct)
    A = (M.general if kind == "gesv" else M.spd)(rng, d, n, M.log_uniform(rng, d, klo, khi))
    if zf > 0:
        M.zero_one_column(rng, A, zf)
    dtype = np.float64 if dt == "f64" else np.float32
    A = np.ascontiguousarray(np.tile(A, (-(-batch // d), 1, 1))[:batch], dtype=dtype)
    B = rng.standard_normal((batch, n, nrhs)).astype(dtype)
    return A, B


class CpuReference:
    """posv/gesv of the reference library compiled from its sources (oracle/_ref),
    with every host thread, on a whole host stack per call; the C restatement in
    oracle/ stands in only where the reference library was not built."""

    def __init__(self):
        from oracle.oracle import Oracle, ref_available
        self.kind = "reference" if ref_available() else "port"
        self.O = Oracle(self.kind)
        self.threads = host_threads() if self.kind == "reference" else 1
        self.O.set_num_threads(self.threads)

    def seconds(self, kind, A0, B0):
        """Time of one call on fresh copies of A0, B0 (the copies are not timed)."""
        A, B = A0.copy(), B0.copy()
        batch, n, nrhs = B.shape
        piv = np.zeros((batch, n), np.int32)
        info = np.zeros(batch, np.int32)
        s = "d" if A.dtype == np.float64 else "f"
        t0 = time.perf_counter()
        if self.kind == "reference":
            if kind == "gesv":
                getattr(self.O.lib, f"ref_gesv_batched_{s}")(A.ctypes.data_as(C.c_void_p), n, batch,
                                                             B.ctypes.data_as(C.c_void_p), nrhs,
                                                             piv.ctypes.data_as(C.c_void_p),
                                                             info.ctypes.data_as(C.c_void_p), 0)
            else:
                getattr(self.O.lib, f"ref_posv_batched_{s}")(A.ctypes.data_as(C.c_void_p), n, batch,
                                                             B.ctypes.data_as(C.c_void_p), nrhs,
                                                             info.ctypes.data_as(C.c_void_p), 0)
        else:
            (self.O.gesv if kind == "gesv" else self.O.posv)(A, B)
        return time.perf_counter() - t0


def cpu_reference(name, batch, calls=4):
    """cpu_baseline record: the reference library on the whole configured batch,
    one untimed call, then the mean of `calls` timed calls."""
    kind = WORKLOADS[name][0]
    ref = CpuReference()
    if ref.kind != "reference":
        batch = min(batch, 4096)  # the single-threaded C restatement on a bounded sample
    A0, B0 = host_inputs(name, batch, 99)
    ref.seconds(kind, A0, B0)
    t = [ref.seconds(kind, A0, B0) for _ in range(calls)]
    v = batch / (sum(t) / len(t))
    what = "reference library compiled from its sources" if ref.kind == "reference" else "C restatement"
    return {"value": round(v, 1), "unit": "solves/s", "cores": ref.threads, "kind": ref.kind,
            "sample": f"{what}, Backend::Auto, the whole batch of {batch} matrices per call "
                      f"(8192 distinct inputs tiled), mean of {calls} calls after one untimed"}


# ---------------------------------------------------------------- GPU arm
def make_inputs(torch, kind, n, batch, nrhs, dtype, klo, khi, zf, seed, device):
    M = _matrices()
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
    cfg = describe(a.workload, batch, world)
    A0, B0 = make_inputs(torch, kind, n, batch, nrhs, dtype, klo, khi, zf, 1234 + rank, device)
    # every warm-up and timed step factors its own untouched copy of the inputs, as far
    # as device memory holds them (the stack of one step is larger than L2)
    want = a.warmup + a.steps
    per_copy = A0.numel() * A0.element_size() + B0.numel() * B0.element_size()
    free, _ = torch.cuda.mem_get_info(device)
    pool = max(2, min(want, int(0.8 * free) // per_copy, a.pool or want))
    As = [A0.clone() for _ in range(pool)]
    Bs = [B0.clone() for _ in range(pool)]
    if pool < want:
        cfg["l2"] = (f"inputs larger than L2 ({per_copy / 1e9:.2f} GB per step); {pool} copies cycled, so the steps "
                     f"after the first {pool} re-factor an already factored stack")
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
    del As, Bs
    torch.cuda.empty_cache()

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
            hA.copy_(A0h)  # fresh inputs every call, restored outside the timed region
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
    stem, kname = dense_kernel(kind, n, dt)
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic_from_profiles(a.workload, stem),
            "peak_source": src, "algorithmic_bytes_per_launch": per_launch, "kernel": kname,
            "gflops": round(batch * flops(kind, n, nrhs) / (ms_step * 1e-3) / 1e9, 1)}

    # the metric's own comparison (bf16+IR against plain fp64 at equal backward error) on
    # the mixed-precision configuration, at n = 64 and n = 32
    ir = None
    if a.workload == "gesv_f64_n64" and not a.skip_ir:
        ir = ir_comparison(torch, device, rank)

    cpu = None
    if rank == 0 and world == 1 and not a.skip_cpu:
        cpu = cpu_reference(a.workload, batch)

    if rank == 0:
        out = {"metric": METRIC, "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": dt, "data": "synthetic", "config": cfg, "roofline": roof,
               "cpu_baseline": cpu, "e2e": _link(e2e), "clocks": clk.summary(), "gpu_launches": int(launches)}
        if ir is not None:
            out["ir"] = ir
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


IR_CONFIG = ("mixed precision + fp64 iterative refinement (normwise backward error <= 1e-15 within 3 corrections, "
             "else the plain fp64 kernel), half SPD Cholesky / half general LU, 1 RHS, kappa log-uniform [1e1,1e12]; "
             "n=64: 131,072 matrices, n=32: 262,144")


def ir_comparison(torch, device, rank, reps=3):
    """The metric's comparison on the mixed-precision configuration: bf16+IR, fp16+IR,
    fp32+IR, the learned selector's tiers and plain fp64, all on the same inputs, at
    n = 64 and n = 32. Solves/s: CUDA events around each pass (A stays on the device,
    x holds b on entry), mean of `reps` passes after one untimed pass per policy, each
    pass on its own fresh copy of b; the timed passes go round the policies in turn, so
    a drift of the clocks over the run falls on every policy alike. Backward error:
    ||b - A x|| / (||A||_F ||x|| + ||b||) of every returned x, in double-double on the
    device."""
    M, dev = _pkg("matrices"), _pkg("device")
    try:
        sel = _selector(device)
    except RuntimeError:
        sel = None
    out = {"config": IR_CONFIG, "timing": f"mean of {reps} passes after one untimed pass, CUDA events"}
    for n, batch in ((64, 131072), (32, 262144)):
        half = batch // 2
        parts = []
        for spd, cnt, seed in ((True, half, 4321 + rank + n), (False, batch - half, 8765 + rank + n)):
            A = M.torch_stack("spd" if spd else "general", n, cnt, 1e1, 1e12, seed, device=device).contiguous()
            g = torch.Generator(device=device)
            g.manual_seed(seed + 1)
            parts.append((spd, A, torch.randn(cnt, n, generator=g, device=device, dtype=torch.float64)))
        policies = [("plain_fp64", 3), ("bf16_ir", 1), ("fp16_ir", 0), ("fp32_ir", 2)]
        if sel is not None:
            policies.append(("selector", None))
        xs = {name: [[b.clone() for _ in range(reps + 1)] for _, _, b in parts] for name, _ in policies}
        res = {name: {} for name, _ in policies}

        def run(name, tier, r):
            for pi, (spd, A, _) in enumerate(parts):
                if tier is None:
                    res[name][pi] = sel.solve(A, xs[name][pi][r], spd)
                else:
                    res[name][pi] = dev.ir(A, xs[name][pi][r], spd, default_tier=tier)
        for name, tier in policies:
            _once(lambda: run(name, tier, 0))
        total = {name: 0.0 for name, _ in policies}
        for r in range(1, reps + 1):
            for name, tier in policies:
                total[name] += _once(lambda: run(name, tier, r))
        pol = {}
        for name, tier in policies:
            ms = total[name] / reps
            bwd = torch.cat([dev.solve_backward_error(A, xs[name][pi][reps], b) for pi, (_, A, b) in enumerate(parts)])
            status = torch.cat([res[name][pi][1] for pi in range(len(parts))])
            rec = {"solves_per_s": round(batch / (ms * 1e-3), 1), "ms": round(ms, 3), "bwd": _stats(bwd)}
            if tier is None:
                t = torch.cat([res[name][pi][3] for pi in range(len(parts))]).long()
                rec["tiers"] = dict(zip(("fp16", "bf16", "fp32", "fp64"), torch.bincount(t, minlength=4).tolist()))
                rec["fp64_fallbacks"] = int(((t < 3) & (status < 0)).sum().item())
            elif tier < 3:
                rec["fp64_fallbacks"] = int((status < 0).sum().item())
            pol[name] = rec
        del xs, res
        base = pol["plain_fp64"]
        out[f"n{n}"] = {
            "batch": batch, "policies": pol,
            "speedup_vs_plain_fp64": {k: round(v["solves_per_s"] / base["solves_per_s"], 3)
                                      for k, v in pol.items() if k != "plain_fp64"},
            "bwd_max_vs_plain_fp64": {k: round(v["bwd"]["max"] / base["bwd"]["max"], 3)
                                      for k, v in pol.items() if k != "plain_fp64"}}
        del parts
        torch.cuda.empty_cache()
    return out


def run_reference(a):
    """The reference library (compiled from its sources, all host threads) on the
    same workload: each step is one call on the whole configured batch, on fresh
    copies of the inputs made outside the timed region."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    kind, n, batch, nrhs, dt, *_ = WORKLOADS[a.workload]
    if a.batch:
        batch = a.batch
    ref = CpuReference()
    if ref.kind != "reference":
        batch = min(batch, 4096)  # the single-threaded C restatement on a bounded sample
    cfg = describe(a.workload, batch, world)
    A0, B0 = host_inputs(a.workload, batch, 7)
    for _ in range(a.warmup):
        ref.seconds(kind, A0, B0)
    secs = sum(ref.seconds(kind, A0, B0) for _ in range(a.steps))
    value = batch * a.steps / secs
    what = "reference library compiled from its sources" if ref.kind == "reference" else "C restatement"
    out = {"metric": METRIC, "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": round(secs / a.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": dt, "data": "synthetic", "config": cfg,
           "impl": "reference",
           "cpu_baseline": {"value": round(value, 1), "unit": "solves/s", "cores": ref.threads, "kind": ref.kind,
                            "sample": f"{what}, Backend::Auto, one call per step on the whole batch of {batch} "
                                      f"matrices (8192 distinct inputs tiled)"},
           "e2e": {"value": round(value, 1), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------- mixed precision, stream, selector
def _pkg(sub):
    return importlib.import_module(PKG_NAME + "." + sub)


def _dist_setup():
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
    return world, rank, local, device, dist


def _max_over_ranks(ms, world, device, dist):
    import torch
    if world > 1:
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def _timed(step, a, world, local, device, dist):
    """W untimed steps, then K steps between barriers + syncs, CUDA events on the
    launching stream; returns (ms per step (max over ranks), clocks, launches)."""
    import torch
    capi = _pkg("capi")
    for i in range(a.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    l0 = capi.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(st)
        for i in range(a.steps):
            step(a.warmup + i)
        e1.record(st)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1) / a.steps, world, device, dist)
    return ms, clk.summary(), capi.launch_count() - l0


def _once(fn):
    """Device time of one call (ms), synchronized on both sides."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _bwd(A, x, b):
    """Normwise backward error ||b - A x||_2 / (||A||_F ||x||_2 + ||b||_2) per matrix, fp64 on the device."""
    import torch
    r = b - torch.bmm(A, x.unsqueeze(-1))[..., 0]
    return r.norm(dim=1) / (A.flatten(1).norm(dim=1) * x.norm(dim=1) + b.norm(dim=1))


def _stats(v):
    import torch
    v = v.double()
    return {"median": float(v.median().item()), "max": float(v.max().item())}


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _cpu_solves(groups, budget_s=12.0):
    """Reference CPU (compiled from its sources, else the C restatement), all host
    threads, on host samples: groups = [(kind, A (b,n,n), B (b,n,r))]. Returns
    (solves/s, threads, kind)."""
    from oracle.oracle import Oracle, ref_available
    kindlib = "reference" if ref_available() else "port"
    O = Oracle(kindlib)
    thr = _threads()
    O.set_num_threads(thr)
    best, total, reps = 0.0, 0.0, 0
    count = sum(g[1].shape[0] for g in groups)
    while total < budget_s and reps < 20:
        work = [(k, A.copy(), B.copy()) for k, A, B in groups]
        t0 = time.perf_counter()
        for k, A, B in work:
            b, n, r = B.shape
            s = "d" if A.dtype == np.float64 else "f"
            info = np.zeros(b, np.int32)
            if kindlib == "reference":
                if k == "gesv":
                    piv = np.zeros((b, n), np.int32)
                    getattr(O.lib, f"ref_gesv_batched_{s}")(A.ctypes.data_as(C.c_void_p), n, b,
                                                            B.ctypes.data_as(C.c_void_p), r,
                                                            piv.ctypes.data_as(C.c_void_p),
                                                            info.ctypes.data_as(C.c_void_p), 0)
                else:
                    getattr(O.lib, f"ref_posv_batched_{s}")(A.ctypes.data_as(C.c_void_p), n, b,
                                                            B.ctypes.data_as(C.c_void_p), r,
                                                            info.ctypes.data_as(C.c_void_p), 0)
            else:
                (O.gesv if k == "gesv" else O.posv)(A, B)
        dt = time.perf_counter() - t0
        total += dt
        reps += 1
        best = max(best, count / dt)
    return best, thr, kindlib


def _emit(a, world, value, ms, dt, cfg, roof, cpu, e2e, clk, launches, extra=None, impl=None):
    out = {"metric": METRIC, "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": dt, "data": "synthetic", "config": cfg}
    if impl:
        out["impl"] = impl
    if roof is not None:
        out["roofline"] = roof
    out["cpu_baseline"] = cpu
    out["e2e"] = e2e if impl else _link(e2e)
    if clk is not None:
        out["clocks"] = clk
    if launches is not None:
        out["gpu_launches"] = int(launches)
    if extra:
        out.update(extra)
    print(json.dumps(out), flush=True)


def link_ceiling_ms(h2d_bytes, d2h_bytes, up_gbs, down_gbs, both_gbs):
    """Least time (ms) to move h2d_bytes in and d2h_bytes out with the two directions
    overlapped: the smaller byte count at the two-way rate (GB/s per direction), the
    rest of the larger direction at its one-way rate."""
    h, d = float(h2d_bytes), float(d2h_bytes)
    rest = (h - d) / up_gbs if h >= d else (d - h) / down_gbs
    return (min(h, d) / both_gbs + rest) / 1e6


def _link(e2e):
    """Attach the host link's ceiling to an e2e record. Pinned host<->device copies
    of 1 GiB are timed host->device alone, device->host alone and both ways at once.
    The ceiling of a step that moves h bytes in and d bytes out, copies overlapped,
    is min(h, d) at the two-way rate plus the rest of the larger direction at its
    one-way rate; frac = that time over the step's time."""
    if not e2e or not e2e.get("ms_per_step"):
        return e2e
    import torch
    nbytes = 1 << 30
    h_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_in = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    cur = torch.cuda.current_stream()

    def rate(up, down):
        best = float("inf")
        for r in range(4):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cur)
            s1.wait_event(e0)
            s2.wait_event(e0)
            if up:
                with torch.cuda.stream(s1):
                    d_in.copy_(h_in, non_blocking=True)
            if down:
                with torch.cuda.stream(s2):
                    h_out.copy_(d_out, non_blocking=True)
            cur.wait_stream(s1)
            cur.wait_stream(s2)
            e1.record(cur)
            e1.synchronize()
            if r:
                best = min(best, e0.elapsed_time(e1))
        return nbytes / (best * 1e-3) / 1e9

    r_up, r_down, r_both = rate(True, False), rate(False, True), rate(True, True)
    h, d = e2e["h2d_bytes_per_step"], e2e["d2h_bytes_per_step"]
    ceil_s = link_ceiling_ms(h, d, r_up, r_down, r_both) * 1e-3
    ach = max(h, d) / (e2e["ms_per_step"] * 1e-3) / 1e9
    e2e["link"] = {"bound": "pcie", "achieved": round(ach, 1), "unit": "GB/s (larger direction)",
                   "h2d_alone": round(r_up, 1), "d2h_alone": round(r_down, 1), "both_ways": round(r_both, 1),
                   "ceiling_ms": round(ceil_s * 1e3, 3), "frac": round(ceil_s * 1e3 / e2e["ms_per_step"], 3),
                   "how": "pinned host<->device copies of 1 GiB: host->device alone, device->host alone, both "
                          "ways at once (GB/s per direction), best of 3, CUDA events"}
    return e2e


def _roof(bytes_per_step, ms, kernel, flops_per_step=None, traffic=None):
    peak, src = peaks()
    ach = bytes_per_step / (ms * 1e-3) / 1e9
    r = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
         "traffic": traffic, "peak_source": src, "algorithmic_bytes_per_launch": int(bytes_per_step),
         "kernel": kernel}
    if flops_per_step:
        r["gflops"] = round(flops_per_step / (ms * 1e-3) / 1e9, 1)
    return r


def _selector(device):
    sel = _pkg("selector")
    w = ROOT / PKG_NAME / "selector_weights.npz"
    if not w.exists():
        raise RuntimeError(f"{w} is missing: train it with {PKG_NAME}/selector_train.py")
    return sel.Selector.load(str(w), device=device)


E2E_SELECTOR_API = ("Selector.solve_host (features + tier + tsdx_cuda_*_ir_f64 per 96 MB chunk on 3 streams), "
                    "pinned host; x, info, status and tier back")


def _e2e_selector(s, parts, world, device, dist):
    """Mean time (ms, max over ranks) of Selector.solve_host over device-resident
    parts [(A, b, spd)] staged once into pinned host memory; b is restored between
    steps outside the timed region."""
    import torch
    hp = [(A.cpu().pin_memory(), b.cpu().pin_memory(), spd) for A, b, spd in parts]
    work = [(hA, torch.empty_like(hb).pin_memory(), spd) for hA, hb, spd in hp]
    ts = []
    for r in range(4):  # the first call warms the caching allocator
        for (_, hb, _), (_, wb, _) in zip(hp, work):
            wb.copy_(hb)
        t = _once(lambda: s.solve_host(work))
        if r:
            ts.append(t)
    return _max_over_ranks(sum(ts) / len(ts), world, device, dist)


def _ir_workload(a, world, rank, local, device, dist):
    import torch
    M, sel, dev = _pkg("matrices"), _pkg("selector"), _pkg("device")
    n = 64
    batch = a.batch or 131072
    half = batch // 2
    parts = []
    for spd, cnt, seed in ((True, half, 4321 + rank), (False, batch - half, 8765 + rank)):
        A = M.torch_stack("spd" if spd else "general", n, cnt, 1e1, 1e12, seed, device=device).contiguous()
        g = torch.Generator(device=device)
        g.manual_seed(seed + 1)
        parts.append((spd, A, torch.randn(cnt, n, generator=g, device=device, dtype=torch.float64)))
    s = _selector(device)
    pool = max(2, min(a.steps + a.warmup, 24))
    xs = [[b.clone() for _ in range(pool)] for _, _, b in parts]

    def step(i):
        for (spd, A, _), bp in zip(parts, xs):
            s.solve(A, bp[i % pool], spd)

    ms, clk, launches = _timed(step, a, world, local, device, dist)
    value = world * batch / (ms * 1e-3)
    # the same inputs through plain fp64 (x only, A untouched) and fixed-tier policies, one pass each
    extra, tiers, bw = {}, {}, {}
    for name, tier in (("plain_fp64", 3), ("fixed_fp32", 2), ("fixed_bf16", 1), ("fixed_fp16", 0)):
        t = 0.0
        fall = 0
        for spd, A, b in parts:
            x = b.clone()
            res = {}

            def run():
                res["st"] = dev.ir(A, x, spd, default_tier=tier)[1]
            t += _once(run)
            if tier < 3:
                fall += int((res["st"] < 0).sum().item())
            if name == "plain_fp64":
                bw.setdefault("plain_fp64", []).append(_bwd(A, x, b))
        extra[name] = {"solves_per_s": round(batch / (t * 1e-3), 1), "ms": round(t, 4)}
        if tier < 3:
            extra[name]["fp64_fallbacks"] = fall
    for spd, A, b in parts:
        x = b.clone()
        info, status, bwd, tier = s.solve(A, x, spd)
        be = _bwd(A, x, b)
        bw.setdefault("selector", []).append(be)
        for t in range(4):
            sel_t = (tier == t)
            tiers[sel.TIERS[t]] = tiers.get(sel.TIERS[t], 0) + int(sel_t.sum().item())
            ok = sel_t & (status >= 0)
            if ok.any():
                bw.setdefault(f"refined_{sel.TIERS[t]}", []).append(be[ok])
        tiers["fp64_fallbacks"] = tiers.get("fp64_fallbacks", 0) + int(((tier < 3) & (status < 0)).sum().item())
    errs = {k: _stats(torch.cat(v)) for k, v in bw.items()}
    extra["selector_tiers"] = tiers
    extra["backward_error"] = errs
    extra["bwd_max_ratio_vs_plain_fp64"] = round(errs["selector"]["max"] / errs["plain_fp64"]["max"], 3)
    extra["speedup_vs_plain_fp64"] = round(value / world / extra["plain_fp64"]["solves_per_s"], 3)
    bytes_step = batch * (8 * (n * n + 2 * n) + 4)
    all_fp64 = tiers.get("fp64") == batch
    routed = ("every matrix routed to fp64 by the calibrated policy: tc_kernel (LU) and blk_kernel (Cholesky), "
              "x only") if all_fp64 else "ir_kernel<64> + features + mlp_forward + fp64 fallback"
    roof = _roof(bytes_step, ms, routed, traffic=None if all_fp64 else traffic_from_profiles("ir_n64", "ir_kernel"))
    # end to end: pinned host A and b in, x and info out, every step
    e2e = None
    if not a.skip_e2e:
        t = _e2e_selector(s, [(A, b, spd) for spd, A, b in parts], world, device, dist)
        e2e = {"value": round(world * batch / (t * 1e-3), 1), "unit": "solves/s",
               "h2d_bytes_per_step": batch * (n * n + n) * 8, "d2h_bytes_per_step": batch * (n * 8 + 9),
               "ms_per_step": round(t, 3), "api": E2E_SELECTOR_API}
    cpu = None
    if rank == 0 and world == 1 and not a.skip_cpu:
        rng = np.random.default_rng(5)
        smp = 2048
        kap = M.log_uniform(rng, smp, 1e1, 1e12)
        groups = [("posv", M.spd(rng, smp, n, kap), rng.standard_normal((smp, n, 1))),
                  ("gesv", M.general(rng, smp, n, kap), rng.standard_normal((smp, n, 1)))]
        v, thr, kl = _cpu_solves(groups)
        cpu = {"value": round(v, 1), "unit": "solves/s", "cores": thr, "kind": kl,
               "sample": f"{2 * smp} n=64 fp64 solves (half posv, half gesv), 1 RHS, per call best of repeated calls"}
    cfg = {"workload": SPECIAL["ir_n64"], "global_batch": world * batch, "batch_per_gpu": batch,
           "parallelism": f"batch sharded over {world} GPU(s), no collective",
           "l2": "inputs larger than L2 (4.3 GB of A per step)",
           "selector": f"{PKG_NAME}/selector_weights.npz"}
    return value, ms, "f64 (tiers fp16/bf16/fp32 factor, fp64 residual)", cfg, roof, cpu, e2e, clk, launches, extra


def stream_inputs(count, rank, device):
    """The uneven stream of the benchmark: n uniform over 2..64, Cholesky (SPD) and LU
    (general) half each, kappa log-uniform [1e1, 1e8] per matrix, 1, 2, 4 or 8
    right-hand sides; packed float32 A and B on the device. Returns
    (n, nrhs, kind, A, B) with n, nrhs, kind as numpy arrays."""
    import torch
    M, stream = _pkg("matrices"), _pkg("stream")
    g = np.random.default_rng(1000 + rank)
    n = g.integers(2, 65, count).astype(np.int32)
    kind = g.integers(0, 2, count).astype(np.int8)
    nrhs = g.choice([1, 2, 4, 8], count).astype(np.int32)
    aoff, boff, poff, na, nb, npv = stream.layout(n, nrhs)
    A0 = torch.empty(na, dtype=torch.float32, device=device)
    key = kind.astype(np.int64) * 100 + n
    order = np.argsort(key, kind="stable")
    ks, starts = np.unique(key[order], return_index=True)
    starts = list(starts) + [count]
    aoff_d = aoff.to(device)
    for gi, k in enumerate(ks):
        idx = order[starts[gi]:starts[gi + 1]]
        nn, kk = int(k % 100), int(k // 100)
        X = M.torch_stack("spd" if kk == 0 else "general", nn, len(idx), 1e1, 1e8, 2000 + gi + 97 * rank,
                          device=device).float()
        dst = aoff_d[torch.from_numpy(idx).to(device)][:, None] + torch.arange(nn * nn, device=device)[None, :]
        A0[dst.reshape(-1)] = X.reshape(-1)
        del X, dst
    gB = torch.Generator(device=device)
    gB.manual_seed(3000 + rank)
    B0 = torch.randn(nb, generator=gB, dtype=torch.float32, device=device)
    return n, nrhs, kind, A0, B0


def _stream_workload(a, world, rank, local, device, dist):
    import torch
    stream = _pkg("stream")
    count = a.batch or 1048576
    n, nrhs, kind, A0, B0 = stream_inputs(count, rank, device)
    aoff, boff, poff, na, nb, npv = stream.layout(n, nrhs)
    plan = stream.StreamPlan(n, nrhs, kind, torch.float32, device=device)
    plan.tune(A0, B0, reps=2)
    pool = max(2, min(a.steps + a.warmup, 11))
    As = [A0.clone() for _ in range(pool)]
    Bs = [B0.clone() for _ in range(pool)]
    graphs = []
    for j in range(pool):
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr):
            stream.solve(As[j], plan.aoff, Bs[j], plan.boff, plan.piv, plan.poff, plan.info, plan.n, plan.nrhs,
                         plan.kind, True, plan.sched, plan.scratch)
        graphs.append(gr)
    # reset the pool after the captures' side effects (capture does not run kernels, but be explicit)
    for j in range(pool):
        As[j].copy_(A0)
        Bs[j].copy_(B0)
    capi = _pkg("capi")
    ms, clk, _ = _timed(lambda i: graphs[i % pool].replay(), a, world, local, device, dist)
    launches = 10 * a.steps  # histogram, scan, scatter and seven drains per replay (counted at capture)
    value = world * count / (ms * 1e-3)
    n64 = n.astype(np.int64)
    bytes_step = int((4 * (2 * n64 * n64 + 2 * n64 * nrhs) + 4 + np.where(kind == 1, 4 * n64, 0)).sum())
    flops_step = float((np.where(kind == 1, 2 * n64 ** 3 / 3, n64 ** 3 / 3) + 2 * n64 * n64 * nrhs).sum())
    roof = _roof(bytes_step, ms, "stream_kernel<float> x7 drains (+ histogram, scan, scatter)", flops_step,
                 traffic_from_profiles("stream_f32", "stream_kernel"))
    extra = {"schedule": {"sched_bits": plan.sched, "tuned_ms": {str(k): round(v, 3) for k, v in plan.timings.items()}}}
    e2e = None
    if not a.skip_e2e:
        # the host-memory stream call on pinned buffers: the set crosses PCIe in 96 MB chunks
        # with the copies overlapping the solves; inputs are restored between steps, untimed
        hA, hB = A0.cpu().pin_memory(), B0.cpu().pin_memory()
        wA, wB = torch.empty_like(hA).pin_memory(), torch.empty_like(hB).pin_memory()
        oP = torch.empty(max(npv, 1), dtype=torch.int32).pin_memory()
        oI = torch.empty(count, dtype=torch.int32).pin_memory()
        nt, rt, kt = torch.from_numpy(n), torch.from_numpy(nrhs), torch.from_numpy(kind)

        def e2e_step():
            stream.solve_host(wA, wB, oP, oI, nt, rt, kt, True, plan.sched)
        ts = []
        for r in range(4):  # the first call sizes the library's device workspace
            wA.copy_(hA)
            wB.copy_(hB)
            t = _once(e2e_step)
            if r:
                ts.append(t)
        t = _max_over_ranks(sum(ts) / len(ts), world, device, dist)
        e2e = {"value": round(world * count / (t * 1e-3), 1), "unit": "solves/s",
               "h2d_bytes_per_step": (na + nb + npv) * 4 + count * 33,
               "d2h_bytes_per_step": (na + nb + npv + count) * 4,
               "ms_per_step": round(t, 3),
               "api": "stream.solve_host (tsdx_cuda_solve_stream_host_f32), pinned host, copies overlapped in 96 MB chunks"}
    cpu = None
    if rank == 0 and world == 1 and not a.skip_cpu:
        smp = 16384
        groups = {}
        A_h = A0[:int(aoff[smp])].cpu().numpy() if smp < count else A0.cpu().numpy()
        B_h = B0[:int(boff[smp])].cpu().numpy() if smp < count else B0.cpu().numpy()
        for i in range(min(smp, count)):
            ni, ri = int(n[i]), int(nrhs[i])
            groups.setdefault((int(kind[i]), ni, ri), []).append(i)
        cg = []
        for (k, ni, ri), idx in groups.items():
            As_ = np.stack([A_h[int(aoff[i]):int(aoff[i]) + ni * ni].reshape(ni, ni) for i in idx])
            Bs_ = np.stack([B_h[int(boff[i]):int(boff[i]) + ni * ri].reshape(ni, ri) for i in idx])
            cg.append(("gesv" if k else "posv", As_, Bs_))
        v, thr, kl = _cpu_solves(cg)
        cpu = {"value": round(v, 1), "unit": "solves/s", "cores": thr, "kind": kl,
               "sample": f"first {min(smp, count)} matrices of the stream, one reference call per (kind, n, nrhs) "
                         f"group ({len(cg)} groups), summed"}
    cfg = {"workload": SPECIAL["stream_f32"], "global_batch": world * count, "batch_per_gpu": count,
           "parallelism": f"stream sharded over {world} GPU(s), no collective",
           "l2": f"inputs larger than L2 ({na * 4 / 1e9:.1f} GB of A), {pool} input copies cycled"}
    return value, ms, "f32", cfg, roof, cpu, e2e, clk, launches, extra


def _selector_workload(a, world, rank, local, device, dist):
    import torch
    sel, dev, M = _pkg("selector"), _pkg("device"), _pkg("matrices")
    train = importlib.import_module(PKG_NAME + ".selector_train")
    count = a.batch or 1048576
    X, y, groups = train.dataset(count, 77 + rank, device=device, keep=True)
    s = _selector(device)
    pred = s.predict(X)
    acc = float((pred == y).float().mean().item())
    confusion = torch.zeros(4, 4, dtype=torch.int64)
    for t in range(4):
        for p_ in range(4):
            confusion[t, p_] = int(((y == t) & (pred == p_)).sum().item())
    pool = 2

    def step(i):
        for gr in groups:
            s.solve(gr["A"], gr["xs"][i % pool], gr["spd"])

    for gr in groups:
        gr["xs"] = [gr["b"].clone() for _ in range(pool)]
    ms, clk, launches = _timed(step, a, world, local, device, dist)
    value = world * count / (ms * 1e-3)
    extra = {"label_accuracy": round(acc, 4), "confusion_true_by_pred": confusion.tolist(),
             "label_counts": dict(zip(sel.TIERS, torch.bincount(y.long(), minlength=4).cpu().tolist()))}
    # policies without the network, and a perfect selector (the labels), one pass each
    policies = {"plain_fp64": 3, "fixed_fp32": 2, "fixed_fp16": 0, "oracle_labels": None}
    bw = {}
    off = 0
    for name, tier in policies.items():
        t, fall = 0.0, 0
        for gr in groups:
            x = gr["b"].clone()
            res = {}
            tt = None if tier is not None else s.policy(gr["y"], gr["n"], gr["spd"]).to(torch.int8).contiguous()

            def run():
                res["st"] = dev.ir(gr["A"], x, gr["spd"], tier=tt, default_tier=3 if tier is None else tier)[1]
            t += _once(run)
            if tier != 3:
                fall += int(((res["st"] < 0) & ((tt < 3) if tier is None else True)).sum().item())
            if name == "plain_fp64":
                bw.setdefault("plain_fp64", []).append(_bwd(gr["A"], x, gr["b"]))
        extra[name] = {"solves_per_s": round(count / (t * 1e-3), 1), "ms": round(t, 3)}
        if tier != 3:
            extra[name]["fp64_fallbacks"] = fall
    fall = nfp64 = 0
    for gr in groups:
        x = gr["b"].clone()
        _, status, _, tier = s.solve(gr["A"], x, gr["spd"])
        bw.setdefault("selector", []).append(_bwd(gr["A"], x, gr["b"]))
        fall += int(((tier < 3) & (status < 0)).sum().item())
        nfp64 += int((tier == 3).sum().item())
    extra["selector_fp64_fallbacks"] = fall
    errs = {k: _stats(torch.cat(v)) for k, v in bw.items()}
    extra["backward_error"] = errs
    extra["speedup_vs_plain_fp64"] = round(value / world / extra["plain_fp64"]["solves_per_s"], 3)
    extra["speedup_vs_fixed_fp16"] = round(value / world / extra["fixed_fp16"]["solves_per_s"], 3)
    extra["speedup_vs_fixed_fp32"] = round(value / world / extra["fixed_fp32"]["solves_per_s"], 3)
    nsum = sum(gr["count"] * (8 * (gr["n"] ** 2 + 2 * gr["n"]) + 4) for gr in groups)
    routed = ("every matrix routed to fp64 by the calibrated policy: the plain fp64 kernels of each order, x only"
              if nfp64 == count else "ir_kernel (+ features, mlp_forward, fp64 fallback)")
    roof = _roof(nsum, ms, routed, traffic=None)
    cfg = {"workload": SPECIAL["selector"], "global_batch": world * count, "batch_per_gpu": count,
           "parallelism": f"evaluation set sharded over {world} GPU(s), no collective",
           "l2": "inputs larger than L2 (13 GB of A per step)", "selector": f"{PKG_NAME}/selector_weights.npz"}
    e2e = None
    if not a.skip_e2e:
        t = _e2e_selector(s, [(gr["A"], gr["b"], gr["spd"]) for gr in groups], world, device, dist)
        e2e = {"value": round(world * count / (t * 1e-3), 1), "unit": "solves/s",
               "h2d_bytes_per_step": sum(gr["count"] * (gr["n"] ** 2 + gr["n"]) * 8 for gr in groups),
               "d2h_bytes_per_step": sum(gr["count"] * (gr["n"] * 8 + 9) for gr in groups),
               "ms_per_step": round(t, 3), "api": E2E_SELECTOR_API}
    return value, ms, "f64 (tiers fp16/bf16/fp32 factor, fp64 residual)", cfg, roof, None, e2e, clk, launches, extra


def _ir_fixed_workload(a, world, rank, local, device, dist):
    import torch
    M, dev = _pkg("matrices"), _pkg("device")
    n, batch = 64, a.batch or 65536
    A = M.torch_stack("general", n, batch, 1e1, 1e3, 5150 + rank, device=device).contiguous()
    g = torch.Generator(device=device)
    g.manual_seed(5151 + rank)
    b = torch.randn(batch, n, generator=g, device=device, dtype=torch.float64)
    pool = max(2, min(a.steps + a.warmup, 24))
    xs = [b.clone() for _ in range(pool)]
    tier = {"fp16": 0, "bf16": 1, "fp32": 2}[a.ir_tier]
    ms, clk, launches = _timed(lambda i: dev.ir(A, xs[i % pool], False, default_tier=tier), a, world, local, device,
                               dist)
    value = world * batch / (ms * 1e-3)
    x = b.clone()
    _, status, _ = dev.ir(A, x, False, default_tier=tier)
    xp = b.clone()
    tp = _once(lambda: dev.ir(A, xp, False, default_tier=3))
    refined = status[status >= 0]
    extra = {"tier": a.ir_tier, "refined_without_fallback": float((status >= 0).float().mean().item()),
             "corrections_median": float(refined.float().median().item()) if refined.numel() else None,
             "plain_fp64": {"solves_per_s": round(batch / (tp * 1e-3), 1), "ms": round(tp, 4)},
             "speedup_vs_plain_fp64": round(value / world / (batch / (tp * 1e-3)), 3),
             "backward_error": {f"ir_{a.ir_tier}": _stats(dev.solve_backward_error(A, x, b)),
                                "plain_fp64": _stats(dev.solve_backward_error(A, xp, b))}}
    roof = _roof(batch * (8 * (n * n + 2 * n) + 4), ms, f"ir_kernel<64,LU> ({a.ir_tier} tier)",
                 traffic=traffic_from_profiles(f"ir_{a.ir_tier}_n64", "ir_kernel"))
    cpu = None
    if rank == 0 and world == 1 and not a.skip_cpu:
        rng = np.random.default_rng(6)
        v, thr, kl = _cpu_solves([("gesv", M.general(rng, 4096, n, M.log_uniform(rng, 4096, 1e1, 1e3)),
                                   rng.standard_normal((4096, n, 1)))])
        cpu = {"value": round(v, 1), "unit": "solves/s", "cores": thr, "kind": kl,
               "sample": "4096 n=64 fp64 gesv, 1 RHS (the reference has no mixed-precision path)"}
    cfg = {"workload": SPECIAL["ir_fp32_n64"], "global_batch": world * batch, "batch_per_gpu": batch,
           "parallelism": f"batch sharded over {world} GPU(s), no collective",
           "l2": "inputs larger than L2 (2.1 GB of A per step)"}
    return value, ms, f"f64 ({a.ir_tier} factor, fp64 residual)", cfg, roof, cpu, None, clk, launches, extra


def run_ours_special(a):
    world, rank, local, device, dist = _dist_setup()
    fn = {"ir_n64": _ir_workload, "stream_f32": _stream_workload, "selector": _selector_workload,
          "ir_fp32_n64": _ir_fixed_workload}[a.workload]
    value, ms, dt, cfg, roof, cpu, e2e, clk, launches, extra = fn(a, world, rank, local, device, dist)
    if rank == 0:
        _emit(a, world, value, ms, dt, cfg, roof, cpu, e2e, clk, launches, extra)
    if world > 1:
        dist.destroy_process_group()


def run_reference_special(a):
    """The reference's own CPU implementation on a bounded sample of the workload:
    plain fp64 posv/gesv for the mixed-precision workloads (the reference has no
    mixed-precision path), per-(kind, n, nrhs) group calls for the stream."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    M = _matrices()
    vals = []
    budget = max(2.0, 150.0 / max(1, a.steps + a.warmup))
    rng = np.random.default_rng(9)
    if a.workload == "stream_f32":
        groups = []
        for kk in (0, 1):
            for ni in range(2, 65):
                for r in (1, 2, 4, 8):
                    kap = M.log_uniform(rng, 16, 1e1, 1e8)
                    A = (M.spd if kk == 0 else M.general)(rng, 16, ni, kap).astype(np.float32)
                    groups.append(("posv" if kk == 0 else "gesv", A,
                                   rng.standard_normal((16, ni, r)).astype(np.float32)))
        sample = "16 fp32 matrices per (kind, n, nrhs) for every n in 2..64, both kinds, nrhs in {1,2,4,8} (8064)"
    else:
        sizes = (64,) if a.workload in ("ir_n64", "ir_fp32_n64") else (8, 24, 40, 56, 64)
        khi = {"ir_n64": 1e12, "ir_fp32_n64": 1e3}.get(a.workload, 1e14)
        groups = []
        for ni in sizes:
            for kk in ("posv", "gesv"):
                kap = M.log_uniform(rng, 1024, 1e1, khi)
                A = (M.spd if kk == "posv" else M.general)(rng, 1024, ni, kap)
                groups.append((kk, A, rng.standard_normal((1024, ni, 1))))
        sample = f"1024 fp64 matrices per (kind, n) for n in {sizes}, 1 RHS, plain posv/gesv"
    thr, kl = 1, "port"
    for i in range(a.warmup + a.steps):
        v, thr, kl = _cpu_solves(groups, budget_s=budget)
        if i >= a.warmup:
            vals.append(v)
    value = float(np.median(vals))
    cfg = {"workload": SPECIAL[a.workload]}
    per_step = {"ir_n64": 131072, "stream_f32": 1048576, "selector": 1048576, "ir_fp32_n64": 65536}[a.workload]
    cfg["global_batch"] = per_step
    _emit(a, world, value, per_step / value * 1e3, "f32" if a.workload == "stream_f32" else "f64", cfg, None,
          {"value": round(value, 1), "unit": "solves/s", "cores": thr, "kind": kl, "sample": sample},
          {"value": round(value, 1), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
          None, None, impl="reference")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gesv_f64_n64", choices=sorted(WORKLOADS) + sorted(SPECIAL))
    ap.add_argument("--batch", type=int, default=0, help="override the workload's batch (profiling runs)")
    ap.add_argument("--pool", type=int, default=0,
                    help="at most this many input copies (default: one per warm-up and timed step)")
    ap.add_argument("--skip-ir", action="store_true", help="leave out the mixed-precision comparison block")
    ap.add_argument("--ir-tier", default="fp32", choices=["fp16", "bf16", "fp32"],
                    help="factorization tier of the ir_fp32_n64 workload")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    a = ap.parse_args(argv)
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        (run_reference_special if a.workload in SPECIAL else run_reference)(a)
    else:
        (run_ours_special if a.workload in SPECIAL else run_ours)(a)


if __name__ == "__main__":
    main()
