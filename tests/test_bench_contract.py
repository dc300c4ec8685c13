"""bench.py's reference arm runs on the host alone: it times the reference's own
stock driver (oracle/_ref) on the O(3) workload and prints one JSON line with
the fields the measurement contract asks of it."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    from oracle.oracle import have_reference

    if not have_reference():
        pytest.skip("reference harness (oracle/_ref) not built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--L", "16",
                        "--steps", "3", "--warmup", "1"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "site-updates/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 3 and d["warmup"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"] and d["config"]["L"] == 16


@pytest.mark.gpu
@pytest.mark.parametrize("workload,L", [("userxy", 256), ("usero3", 32), ("usero3csr", 32), ("userwolff", 128),
                                        ("useru1", 8), ("useru1tables", 8)])
def test_user_model_bench_lines_keep_the_contract(workload, L):
    """The user-model workloads (generic device kernels of include/umc/device.cuh)
    print one JSON line with the contract's fields, a roofline of their own
    kernel and a positive end-to-end figure."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", workload, "--L", str(L),
                        "--steps", "5", "--warmup", "3", "--no-cpu-baseline"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["value"] > 0 and d["steps"] == 5 and d["warmup"] == 3 and d["unit"] in ("site-updates/s", "link-updates/s")
    assert d["roofline"]["kernel"] in ("metropolis_sweeps", "wolff_flips") and d["roofline"]["achieved"] > 0
    assert d["gpu_launches"] >= 5 and d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0
    assert d["config"]["L"] == L and "clocks" in d
