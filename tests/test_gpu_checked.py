"""The bounds-checked build (liblesb200_checked.so, LES_CHECKED): every box
index of every kernel that addresses the state through IX() is checked
against its allocation.  The same workload (tests/checked_workload.py: time
steps over ragged shapes in both sum modes, the context's halo entries, both
FP64 refinements, the step adjoint with a drag scale, an ensemble) runs on
both libraries in child processes; the checked one must see no index out of
range, and its results must be bit-identical to the plain library's (the
step adjoint, whose atomic sums are order-dependent, to 1e-5 relative).
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _run(checked: bool) -> dict:
    env = dict(os.environ)
    env.pop("LES_B200_CHECKED", None)
    if checked:
        env["LES_B200_CHECKED"] = "1"
    out = subprocess.run([sys.executable, "-m", "tests.checked_workload"], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_checked_build_sees_no_out_of_range_index(require_gpu):
    chk = _run(True)
    assert chk["lib"] == "liblesb200_checked.so"
    assert chk["status"] == 0
    assert chk["violations"] == 0, f"first out-of-range (i, j, k): {chk['first']}"
    plain = _run(False)
    assert plain["lib"] == "liblesb200.so"
    assert plain["status"] != 0  # the plain build has no bounds record
    for part in ("steps", "refine", "ensemble"):
        assert chk[part] == plain[part], part
    for k, v in plain["adjoint"].items():
        assert abs(chk["adjoint"][k] - v) <= 1e-5 * abs(v), (k, chk["adjoint"][k], v)
