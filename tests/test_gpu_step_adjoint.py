"""The device adjoint of whole time steps (les_adj_*) against the FP64
reference adjoint (oracle/adjoint64.py, itself checked against central
differences of the FP64 oracle) and against central differences of the CUDA
forward itself.

The step adjoint runs in FP32 (its parameter gradients accumulate in FP64),
so it is compared with the FP64 reference to a relative tolerance, not bit
for bit: TOL on the norm of the difference over all arrays, relative to the
norm of the reference.
"""
import numpy as np
import pytest

import oracle
from oracle import adjoint64
from les_halo_b200 import GpuAdjoint, GpuLes, fields as FL, set_drag, synthetic_case, tke_gradient

pytestmark = pytest.mark.gpu
IP, JP, KP = 24, 20, 12
NITER = 3
TOL = 1e-4
NAMES = ["dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s",
         "cn3l", "cn3s", "cn4l", "cn4s"]


def rnd(name, seed, ip=IP, jp=JP, kp=KP, scale=1.0):
    a = FL.alloc(name, ip, jp, kp)
    a[...] = scale * np.random.default_rng(seed).standard_normal(a.shape)
    return a


def _setup(seed, drag=None):
    case = synthetic_case(IP, JP, KP, seed=seed, masks_and_poisson=oracle.masks_and_poisson)
    case.params.nmaxp = NITER
    case.params.pjuge = -1.0  # every step runs NITER iterations
    x = {n: rnd(n, 1000 + seed * 50 + s) for s, n in enumerate(FL.STATE)}
    wp = rnd("wind_profile", 999 + seed)
    for n in FL.STATE:
        case.arrays[n] = x[n]
    case.arrays["wind_profile"] = wp
    pr = case.params
    prm = {k: float(np.float32(getattr(pr, k))) for k in ("dt", "ro", "vn", "alpha", "beta", "omega")}
    co = {nm: case.arrays[nm] for nm in NAMES}
    step = adjoint64.Step64(IP, JP, KP, co, prm, NITER, drag=drag)
    gpu = GpuLes(case)
    if drag is not None:
        set_drag(gpu, drag)
    return case, gpu, step, x, wp


def _close(got, want, names):
    num = sum(float(np.sum((got[n].astype(np.float64) - want[n]) ** 2)) for n in names)
    den = sum(float(np.sum(np.asarray(want[n], dtype=np.float64) ** 2)) for n in names)
    return np.sqrt(num / den)


@pytest.mark.parametrize("n", [1, 5])
@pytest.mark.parametrize("with_drag", [False, True])
def test_step_adjoint_against_fp64_reference(require_gpu, n, with_drag):
    drag = (1.0 + 0.3 * np.random.default_rng(4).standard_normal((IP, JP))).astype(np.float32) if with_drag else None
    case, gpu, step, x, wp = _setup(3 + n, drag)
    y = {nm: rnd(nm, 2000 + s) for s, nm in enumerate(FL.STATE)}
    x64 = {k: v.astype(np.float64) for k, v in x.items()}
    _, tape = step.forward(n, x64, wp.astype(np.float64))
    ref, grads = step.adjoint(n, tape, wp.astype(np.float64), {k: v.astype(np.float64) for k, v in y.items()})
    adj = GpuAdjoint(gpu, 1, NITER)
    adj.save(0)
    adj.write(y)
    adj.step_b(n, 0)
    got = adj.read(state=True)
    err = _close(got["state"], ref, FL.STATE)
    assert err <= TOL, err
    # every array on its own, against the whole adjoint's scale
    scale = np.sqrt(sum(float(np.sum(np.asarray(ref[k]) ** 2)) for k in FL.STATE))
    for k in FL.STATE:
        d = np.linalg.norm(got["state"][k].astype(np.float64) - ref[k])
        assert d <= TOL * scale, (k, d / scale)
    assert np.linalg.norm(got["wp"] - grads["wp"]) <= TOL * np.linalg.norm(grads["wp"])
    if with_drag:
        assert np.linalg.norm(got["drag"] - grads["drag"]) <= TOL * np.linalg.norm(grads["drag"])
    adj.close()
    gpu.close()


def test_checkpointed_tke_gradient_against_fp64_reference(require_gpu):
    # J = mean over 5 steps of the box's resolved TKE, checkpoints every 2
    # steps with recomputation, with a drag scale: gradients for the inflow
    # profile, the drag scale and the initial state
    drag = (1.0 + 0.2 * np.random.default_rng(7).standard_normal((IP, JP))).astype(np.float32)
    case, gpu, step, x, wp = _setup(11, drag)
    box, nt, ckpt = ((3, 8), (2, 7), (1, 3)), 5, 2
    adj = GpuAdjoint(gpu, 3 + ckpt, NITER)
    J, g = tke_gradient(gpu, adj, 1, nt, box, ckpt)
    J64, grads, bar = adjoint64.tke_gradient(step, 1, nt, {k: v.astype(np.float64) for k, v in x.items()},
                                             wp.astype(np.float64), box, ckpt=2)
    assert abs(J - J64) <= 1e-5 * abs(J64), (J, J64)
    assert np.linalg.norm(g["wp"] - grads["wp"]) <= TOL * np.linalg.norm(grads["wp"])
    assert np.linalg.norm(g["drag"] - grads["drag"]) <= TOL * np.linalg.norm(grads["drag"])
    assert _close(g["state"], bar, FL.STATE) <= TOL
    adj.close()
    gpu.close()


def test_checkpoint_spacing_does_not_change_the_gradient(require_gpu):
    # the recomputed segments give the forward values the first pass saw
    # (the forward is deterministic): spacings 1, 2 and 5 agree closely (the
    # atomic adds of the adjoint make the last bits order-dependent)
    res = []
    for ckpt in (1, 2, 5):
        case, gpu, step, x, wp = _setup(12)
        adj = GpuAdjoint(gpu, 5 + ckpt, NITER)
        J, g = tke_gradient(gpu, adj, 2, 5, ((3, 8), (2, 7), (1, 3)), ckpt)
        res.append((J, g["wp"]))
        adj.close()
        gpu.close()
    for J, wpb in res[1:]:
        assert J == res[0][0]
        assert np.linalg.norm(wpb - res[0][1]) <= 1e-5 * np.linalg.norm(res[0][1])


def test_gradient_against_fp64_central_differences(require_gpu):
    # The config-3 structure on a small grid: terrain, 6 steps from the
    # initial state with checkpoints every 3, J = time-mean resolved TKE of
    # a box.  The CUDA gradient (FP32 adjoint) against central differences
    # (h = 1e-3) of the FP64 oracle's steps in 16 seeded directions, moving
    # the inflow profile and the drag scale by a relative h.
    drag0 = np.ones((IP, JP), np.float32)
    case, gpu, step, x, wp0 = _setup(14, drag0)
    box, nt, ckpt = ((5, 12), (4, 11), (1, 4)), 6, 3
    adj = GpuAdjoint(gpu, 2 + ckpt, NITER)
    J, g = tke_gradient(gpu, adj, 1, nt, box, ckpt)
    x64 = {k: v.astype(np.float64) for k, v in x.items()}

    def J64(wp, drag):
        st = adjoint64.Step64(step.ip, step.jp, step.kp, step.co, step.prm, NITER, drag=drag)
        s, acc = x64, 0.0
        for t in range(nt):
            s, _ = st.forward(1 + t, s, wp)
            acc += adjoint64.tke(IP, JP, KP, s, box) / nt
        return acc

    assert abs(J - J64(wp0.astype(np.float64), drag0.astype(np.float64))) <= 1e-5 * abs(J)
    rng = np.random.default_rng(77)
    h = 1e-3
    errs = []
    for d in range(16):
        dwp = rng.standard_normal(wp0.shape) * np.abs(wp0)
        ddrag = rng.standard_normal((IP, JP))
        fd = (J64(wp0 + h * dwp, drag0 + h * ddrag) - J64(wp0 - h * dwp, drag0 - h * ddrag)) / (2 * h)
        ad = float(np.sum(g["wp"] * dwp)) + float(np.sum(g["drag"] * ddrag))
        errs.append(abs(fd - ad) / abs(fd))
    print("adjoint vs FP64 central differences, relative errors:", " ".join(f"{e:.1e}" for e in errs))
    assert max(errs) <= 1e-4, errs
    adj.close()
    gpu.close()


@pytest.mark.slow
def test_config3_gradient_against_central_differences(require_gpu):
    # The adjoint configuration: the 150 x 150 x 90 benchmark terrain from
    # its warm-up, 100 steps with a checkpoint every 10, J = time mean of the
    # resolved TKE of a 20 x 20 x 5-cell pedestrian box (cell centres below
    # 10 m); gradients with respect to the 90-value inflow profile (every
    # column of wind_profile(j, k) moved together) and the 150 x 150 drag
    # scale, against central differences of the CUDA forward (h = 1e-3, the
    # profile and the drag scale moved by a relative h) in 16 seeded
    # directions.  Here the differences are the less exact side: the FP32
    # forward's rounding, carried through 100 steps of the flow, is a part in
    # 1e6 to 1e7 of J, against a change of J of about a part in 1e3, so a
    # direction whose derivative is small can show a relative error of a few
    # 1e-4 while the typical one agrees to about 1e-5.
    ip, jp, kp, nt, ckpt = 150, 150, 90, 100, 10
    box = ((66, 85), (66, 85), (1, 5))
    case = synthetic_case(ip, jp, kp, seed=1, masks_and_poisson=oracle.masks_and_poisson)
    case.params.pjuge = -1.0  # all 50 SOR iterations in every step, as differentiated
    wp0 = case.a("wind_profile").copy(order="F")
    prof = wp0.mean(axis=0)
    gpu = GpuLes(case)
    gpu.warmup(1)
    ones = np.ones((ip, jp), np.float32)
    set_drag(gpu, ones)
    adj = GpuAdjoint(gpu, -(-nt // ckpt) + ckpt + 1, 50)
    adj.save(adj.nslots - 1)  # the warmed-up initial state
    J, g = tke_gradient(gpu, adj, 1, nt, box, ckpt)
    gprof = g["wp"].sum(axis=0)  # the profile moves every j of a level together

    def J_of(wp, drag):
        adj.load(adj.nslots - 1)
        gpu.set_wind_profile(np.asfortranarray(wp, dtype=np.float32))
        set_drag(gpu, drag)
        acc = 0.0
        for t in range(nt):
            gpu.step(1 + t, 1)
            acc += adj.tke(-1, box) / nt
        return acc

    assert abs(J_of(wp0, ones) - J) <= 1e-12 * abs(J)
    rng = np.random.default_rng(2024)
    h = 1e-3
    errs = []
    for d in range(16):
        dprof = rng.standard_normal(kp) * prof
        ddrag = rng.standard_normal((ip, jp))
        wpp = wp0 + h * dprof[np.newaxis, :]
        wpm = wp0 - h * dprof[np.newaxis, :]
        fd = (J_of(wpp, ones + h * ddrag) - J_of(wpm, ones - h * ddrag)) / (2 * h)
        ad = float(np.dot(gprof, dprof)) + float(np.sum(g["drag"] * ddrag))
        errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
    print("config-3 adjoint vs central differences of the FP32 forward, relative errors:",
          " ".join(f"{e:.1e}" for e in errs))
    assert max(errs) <= 1e-3, errs
    assert float(np.median(errs)) <= 1e-4, errs
    adj.close()
    gpu.close()


def test_autograd_function_over_the_c_abi(require_gpu):
    # loss.backward() through tests/autograd_step.TkeObjective (CUDA forward
    # and device adjoint behind the C ABI) gives the FP64 reference gradients
    import torch
    from tests.autograd_step import TkeObjective
    drag0 = (1.0 + 0.2 * np.random.default_rng(9).standard_normal((IP, JP))).astype(np.float32)
    case, gpu, step, x, wp0 = _setup(13, drag0)
    box, nt, ckpt = ((4, 9), (3, 8), (2, 4)), 4, 2
    adj = GpuAdjoint(gpu, 2 + ckpt + 1, NITER)
    init = adj.nslots - 1
    adj.save(init)
    wp = torch.tensor(wp0.astype(np.float64), requires_grad=True)
    drag = torch.tensor(drag0.astype(np.float64), requires_grad=True)
    loss = TkeObjective.apply(wp, drag, gpu, adj, init, 1, nt, box, ckpt)
    loss.backward()
    J64, grads, _ = adjoint64.tke_gradient(step, 1, nt, {k: v.astype(np.float64) for k, v in x.items()},
                                           wp0.astype(np.float64), box, ckpt=2)
    assert abs(loss.item() - J64) <= 1e-5 * abs(J64)
    assert np.linalg.norm(wp.grad.numpy() - grads["wp"]) <= TOL * np.linalg.norm(grads["wp"])
    assert np.linalg.norm(drag.grad.numpy() - grads["drag"]) <= TOL * np.linalg.norm(grads["drag"])
    adj.close()
    gpu.close()
