"""The reference arm of bench.py (the reference's own CPU code, timed on this
host's cores) prints one JSON line with the fields the benchmark contract
names; it needs no GPU, so it runs here."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_contract_line(oracle_built):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--workload", "water"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["unit"] == "solves/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"].startswith("water box") and d["config"]["atoms"] == 98304
    assert "water" in d["metric"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_bench_defaults_to_the_largest_single_gpu_workload():
    """With no flags both arms run the 1,048,576-charge triclinic solve."""
    sys.path.insert(0, ROOT)
    import bench

    assert bench.DEFAULT_WORKLOAD == "triclinic"
    c = bench.load_workload(bench.DEFAULT_WORKLOAD)
    assert c.n == 1048576 and c.K == (256, 256, 256) and c.order == 6 and c.beta == 3.5
    assert "1,048,576" in bench.WORKLOADS[bench.DEFAULT_WORKLOAD][0]
