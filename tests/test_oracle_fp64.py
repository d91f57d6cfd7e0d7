"""The FP32 step against the same algorithm in double precision (no GPU).

The FP32 oracle is bit-identical to the CUDA path (tests/test_gpu_step.py),
so this bounds the CUDA path's distance to the FP64 oracle: within the
stated 1e-5 relative L2 on u, v, w, p, for the plain press and for the
FP64-refined press with the spectral inner solve."""
import pytest

from oracle import fp64_error_table as T

TOL_REL_L2 = 1e-5


@pytest.mark.parametrize("refine", [None, (1, 0, 0.0)])
def test_fp32_step_within_tolerance_of_fp64(refine):
    e = T.errors(48, 40, 30, 12, refine=refine)
    for n in ("u", "v", "w", "p"):
        assert e[n] <= TOL_REL_L2, (n, e[n])
    assert max(e.values()) <= 1e-4, e
