"""press with a fixed SOR iteration count is linear (no GPU).

The adjoint entry les_press_b_ transposes press.f95:49-146 as a linear map
of (rhs, u, v, w, f, g, h, p); this checks that premise on the FP64 oracle:
F(a x1 + b x2) = a F(x1) + b F(x2) on every output element, up to FP64
rounding, and F(0) = 0."""
import numpy as np
import pytest

import oracle
from les_halo_b200 import synthetic_case
from tests.test_gpu_adjoint import IN, OUT, IP, JP, KP, press64, rand_fields


@pytest.mark.parametrize("niter", [0, 3])
def test_press_is_linear_with_a_fixed_iteration_count(niter):
    case = synthetic_case(IP, JP, KP, seed=21, masks_and_poisson=oracle.masks_and_poisson)
    x1, x2 = rand_fields(IN, 1), rand_fields(IN, 2)
    a, b = 0.75, -1.25
    x3 = {n: np.asfortranarray(a * x1[n].astype(np.float64) + b * x2[n].astype(np.float64)) for n in IN}
    f1, f2, f3 = press64(case, x1, niter), press64(case, x2, niter), press64(case, x3, niter)
    for n in OUT:
        want = a * f1[n] + b * f2[n]
        assert np.max(np.abs(f3[n] - want)) <= 1e-11 * max(1.0, float(np.max(np.abs(want)))), n
    z = press64(case, {n: 0.0 * x1[n] for n in IN}, niter)
    assert all(not np.any(z[n]) for n in OUT)
