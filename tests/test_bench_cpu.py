"""Host-side arithmetic of bench.py (no GPU): the e2e link-ceiling model."""
import importlib.util

import pytest

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_link_ceiling_model():
    f = _bench().link_ceiling_ms
    # equal traffic both ways: all of it at the two-way rate
    assert f(44.3e9, 44.3e9, 55.0, 52.0, 44.3) == pytest.approx(1000.0)
    # one way only: the one-way rate
    assert f(55.6e9, 0, 55.6, 52.0, 44.3) == pytest.approx(1000.0)
    assert f(0, 52.0e9, 55.6, 52.0, 44.3) == pytest.approx(1000.0)
    # mixed: 1 GB both ways at 40 GB/s (25 ms), the other 2 GB in at 60 GB/s (33.3 ms)
    assert f(3e9, 1e9, 60.0, 50.0, 40.0) == pytest.approx(25.0 + 2e9 / 60e6)
    # mixed, larger outbound: 1 GB both ways (25 ms), 1 GB more out at 50 GB/s (20 ms)
    assert f(1e9, 2e9, 60.0, 50.0, 40.0) == pytest.approx(45.0)


def test_reference_arm_contract():
    """bench.py --impl reference runs the reference library (compiled from its sources
    into oracle/_ref) on the host and prints one JSON line with the fields the
    comparison needs; it needs no GPU."""
    import json
    import subprocess
    import sys
    if not (ROOT / "oracle" / "_ref" / "libtsdx_ref.so").exists():
        pytest.skip("oracle/_ref not built")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "posv_f64_n16",
                          "--steps", "1", "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_under_torchrun_two_ranks():
    """Launched like the multi-GPU runs (torchrun, 2 ranks): rank 0 alone runs the
    reference and prints one line; the other rank exits 0 without work."""
    import json
    import socket
    import subprocess
    import sys
    if not (ROOT / "oracle" / "_ref" / "libtsdx_ref.so").exists():
        pytest.skip("oracle/_ref not built")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
           "--workload", "posv_f64_n16", "--steps", "1", "--warmup", "3"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0


def test_reference_arm_loads_only_the_reference_library():
    """The reference arm's process maps oracle/_ref/libtsdx_ref.so and none of the
    package's native libraries (it never imports the package)."""
    import subprocess
    import sys
    if not (ROOT / "oracle" / "_ref" / "libtsdx_ref.so").exists():
        pytest.skip("oracle/_ref not built")
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'posv_f64_n16', "
            "'--steps', '1', '--warmup', '3', '--batch', '4096']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPS', int('libtsdx_ref.so' in maps), int('libtsdx_cuda.so' in maps), int('_core.' in maps), "
            "int(any('b200' in m for m in sys.modules)))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("MAPS")][0]
    assert line.split()[1:] == ["1", "0", "0", "0"], line


def test_both_arms_describe_the_same_config():
    b = _bench()
    for name in b.WORKLOADS:
        batch = b.WORKLOADS[name][2]
        c = b.describe(name, batch, 1)
        assert c["global_batch"] == batch and c["batch_per_gpu"] == batch and c["parallelism"]


def test_dense_kernel_follows_the_launch_routing(monkeypatch):
    """bench.py names the kernel that csrc/launch.cuh launches: float64 LU on the
    tensor-core kernel from padded order 32 (even orders up to 64, every order up to
    48), the two-warp kernels for odd orders above 48, blk_kernel otherwise."""
    b = _bench()
    monkeypatch.delenv("TSDX_LU_KERNEL", raising=False)
    for n in (25, 32, 33, 41, 47, 48, 50, 56, 58, 64):
        assert b.dense_kernel("gesv", n, "f64")[0] == "tc_kernel", n
    for n in (49, 51, 55):
        assert b.dense_kernel("gesv", n, "f64")[0] == "blk2_kernel", n
    for n in (57, 61, 63):
        assert b.dense_kernel("gesv", n, "f64")[0] == "blk3_kernel", n
    for kind, n, dt in (("gesv", 24, "f64"), ("gesv", 64, "f32"), ("gesv", 32, "f32"), ("posv", 16, "f64"),
                        ("posv", 64, "f64")):
        assert b.dense_kernel(kind, n, dt)[0] == "blk_kernel", (kind, n, dt)
    monkeypatch.setenv("TSDX_LU_KERNEL", "smem")
    assert b.dense_kernel("gesv", 64, "f64")[0] == "blk3_kernel"
    monkeypatch.setenv("TSDX_LU_KERNEL", "tc")
    assert b.dense_kernel("gesv", 63, "f64")[0] == "tc_kernel"


def test_roofline_traffic_comes_from_the_routed_kernels_profile(monkeypatch):
    """A dense line's roofline traffic is read from profiles/<kernel>__<workload>.md of
    the kernel that runs; the default workload has one."""
    b = _bench()
    monkeypatch.delenv("TSDX_LU_KERNEL", raising=False)
    prof = ROOT / "profiles"
    for name, (kind, n, _b, _r, dt, *_rest) in b.WORKLOADS.items():
        stem, _ = b.dense_kernel(kind, n, dt)
        cited = b.traffic_from_profiles(name, stem)
        others = [p.name for p in prof.glob(f"*__{name}.md") if not p.name.startswith(stem + "__")]
        assert not others, f"{name}: profiles of kernels that do not run: {others}"
        if (prof / f"{stem}__{name}.md").exists():
            assert cited is not None and cited > 0, name
    assert b.traffic_from_profiles("gesv_f64_n64", "tc_kernel") > 0
