"""NVTX ranges around the library's host entry points: a test-only NVTX tool
(tests/nvtx_record.c, built here with gcc) is injected through
NVTX_INJECTION64_PATH into a child process that calls the C ABI, and the
ranges it records are checked (names, nesting, every push popped)."""
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent


def _tool(tmp_path) -> Path:
    so = tmp_path / "libnvtx_record.so"
    subprocess.run(["gcc", "-O1", "-shared", "-fPIC", "-I/usr/local/cuda/include", "-o", str(so),
                    str(HERE / "nvtx_record.c")], check=True)
    return so


def _record(tmp_path, body: str):
    log = tmp_path / "ranges.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(_tool(tmp_path)), LES_NVTX_LOG=str(log))
    script = "import sys\nsys.path.insert(0, %r)\n" % str(ROOT) + textwrap.dedent(body)
    subprocess.run([sys.executable, "-c", script], check=True, env=env, cwd=str(ROOT), timeout=600)
    lines = log.read_text().splitlines() if log.exists() else []
    depth, names = 0, []
    for ln in lines:
        if ln.startswith("+"):
            depth += 1
            names.append((depth, ln[1:]))
        else:
            assert ln == "-", ln
            depth -= 1
            assert depth >= 0, "pop without push"
    assert depth == 0, "range left open"
    return names


def test_entry_points_open_and_close_ranges_without_a_gpu(tmp_path):
    names = _record(tmp_path, """
        import ctypes as C
        from les_halo_b200 import abi
        L = abi.lib()
        p = abi.LesParams()
        abi.check(L.les_params_default(C.byref(p), 16, 12, 40))
        ctx = C.c_void_p()
        assert L.les_ctx_create(C.byref(p), C.byref(ctx)) == abi.LES_ERR_DIMS  # early error return
        assert L.les_step(None, 1, 1) == abi.LES_ERR_BAD_ARG
    """)
    assert names == [(1, "les_params_default"), (1, "les_ctx_create"), (1, "les_step")], names


@pytest.mark.gpu
def test_step_ranges_on_the_gpu(tmp_path, require_gpu):
    names = _record(tmp_path, """
        import les_halo_b200 as lh
        g = lh.GpuLes(lh.synthetic_case(48, 40, 80, seed=3, dt=0.05, nmaxp=50))
        g.step(1, 3)
        g.sync()
        g.close()
    """)
    top = [n for d, n in names if d == 1]
    for want in ("les_ctx_create", "les_ctx_upload", "les_step", "les_ctx_sync", "les_ctx_destroy"):
        assert want in top, (want, top)
    inner = [n for d, n in names if d == 2]
    assert inner.count("step") == 3, inner
    assert (3, "step_graph_capture") in names and (3, "sor_autotune") in names, names
