"""les_ctx_field_sums, the reference's WV_DEBUG array sums
(src/Fortran/velnw.f95:61-68, feedbf.f95:30-36 and 68-83): every state
array's sum over its Fortran bounds equals the correctly rounded sum of the
downloaded array (math.fsum), rhs included as the download returns it."""
import math

import numpy as np
import pytest

from les_halo_b200 import GpuLes, abi, fields as FL, synthetic_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(40, 36, 30), (33, 19, 12)])
def test_field_sums_match_the_downloaded_arrays(require_gpu, dims):
    g = GpuLes(synthetic_case(*dims, seed=7, dt=0.05, nmaxp=50))
    try:
        g.step(1, 2)
        g.sync()
        sums = g.field_sums()
        got = g.download(FL.STATE + FL.MASKS)
        for n in FL.STATE + FL.MASKS:
            want = math.fsum(got[n].astype(np.float64).ravel())
            # the device sums exactly (terms truncated below 2^-64) and rounds once
            assert sums[n] == pytest.approx(want, rel=1e-13, abs=got[n].size * 2.0 ** -60), n
    finally:
        g.close()
