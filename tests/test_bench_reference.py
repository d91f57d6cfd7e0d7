"""bench.py's reference arm (the oracle on the host cores) prints one JSON
line with the keys the measurement contract names, on the GPU arm's
workload, without loading the library under test (no GPU: the arm runs on
the CPU).  A small grid stands in for the 600 x 600 x 120 workload here."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_contract_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--grid", "48,40,30"], capture_output=True, text=True, timeout=600,
                       cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 1 and d["warmup"] == 3
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    # same workload description as the GPU arm (bench.workload_desc), whole grid
    sys.path.insert(0, str(ROOT))
    import bench
    bench.WORKLOAD.update(ip=48, jp=40, kp=30)
    try:
        assert d["config"]["workload"] == bench.workload_desc(48, 40, 30)
    finally:
        bench.WORKLOAD.update(ip=600, jp=600, kp=120)
    assert d["config"]["grid"] == [48, 40, 30]
    # the case is built by the oracle alone: only oracle libraries are mapped
    assert d["native_libs"] and all(x.startswith("oracle/") for x in d["native_libs"]), d["native_libs"]
