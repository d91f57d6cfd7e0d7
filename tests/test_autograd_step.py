"""The step adjoint behind torch.autograd (no GPU): a TKE objective written
in torch over StepFunction steps, loss.backward(), against the reference
gradients of oracle/adjoint64.tke_gradient (same FP64 adjoint, composed by
hand with checkpoints)."""
import numpy as np
import torch

import oracle
from oracle import adjoint64
from les_halo_b200 import synthetic_case
from tests.autograd_step import StepFunction, tke_torch
from tests.test_adjoint64 import IP, JP, KP, rnd

NAMES = ["dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s",
         "cn3l", "cn3s", "cn4l", "cn4s"]


def test_autograd_gradients_equal_the_reference_adjoint():
    case = synthetic_case(IP, JP, KP, seed=10, masks_and_poisson=oracle.masks_and_poisson)
    pr = case.params
    prm = {k: float(np.float32(getattr(pr, k))) for k in ("dt", "ro", "vn", "alpha", "beta", "omega")}
    co = {nm: case.arrays[nm] for nm in NAMES}
    x = {nm: rnd(nm, 900 + s) for s, nm in enumerate(adjoint64.STATE)}
    wp0 = rnd("wind_profile", 950)
    drag0 = 1.0 + 0.2 * np.random.default_rng(11).standard_normal((IP, JP))
    box, nt = ((3, 8), (2, 7), (1, 3)), 3

    step = adjoint64.Step64(IP, JP, KP, co, prm, 3)
    wp = torch.tensor(wp0, requires_grad=True)
    drag = torch.tensor(drag0, requires_grad=True)
    state = [torch.tensor(np.ascontiguousarray(x[k]), requires_grad=True) for k in adjoint64.STATE]
    cur, loss = state, 0.0
    for t in range(nt):
        cur = StepFunction.apply(step, 2 + t, wp, drag, *cur)
        loss = loss + tke_torch(IP, JP, KP, dict(zip(adjoint64.STATE, cur)), box) / nt
    loss.backward()

    ref = adjoint64.Step64(IP, JP, KP, co, prm, 3, drag=drag0)
    J, grads, bar = adjoint64.tke_gradient(ref, 2, nt, x, wp0, box, ckpt=2)
    assert abs(loss.item() - J) <= 1e-13 * abs(J)
    assert np.allclose(wp.grad.numpy(), grads["wp"], rtol=1e-10, atol=1e-14)
    assert np.allclose(drag.grad.numpy(), grads["drag"], rtol=1e-10, atol=1e-14)
    for k, t in zip(adjoint64.STATE, state):
        assert np.allclose(t.grad.numpy(), bar[k], rtol=1e-10, atol=1e-14), k
