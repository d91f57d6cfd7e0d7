"""Host-side mirror of the reference's LES driver for the B200 library.

``LesCase`` holds the model arrays in the reference's Fortran layout (what
main_ocl.f95 allocates); ``synthetic_case`` builds one from the seeded
generators of les_synth.h; ``GpuLes`` is the accelerator driver, mirroring
``initialise_LES_kernel`` / ``run_LES_kernel``
(src/OpenCL/module_LES_combined_ocl_TEMPL_V2.f95:18-30, 219-231) on top of
the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import fields as FL


@dataclass
class LesCase:
    ip: int
    jp: int
    kp: int
    params: abi.LesParams
    arrays: dict = field(default_factory=dict)
    built_fraction: float = 0.0

    def a(self, name):
        return self.arrays[name]

    def copy(self) -> "LesCase":
        return LesCase(self.ip, self.jp, self.kp, _copy_params(self.params),
                       {k: v.copy(order="F") for k, v in self.arrays.items()}, self.built_fraction)

    def host_fields(self) -> abi.LesHostFields:
        hf = abi.LesHostFields()
        for n in abi.HOST_FIELD_NAMES:
            arr = self.arrays.get(n)
            setattr(hf, n, FL.ptr(arr) if arr is not None else None)
        return hf


def _copy_params(p: abi.LesParams) -> abi.LesParams:
    q = abi.LesParams()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(p))
    return q


def default_params(ip, jp, kp, dt=0.05, inflow="external", nmaxp=50) -> abi.LesParams:
    p = abi.LesParams()
    abi.check(abi.lib().les_params_default(C.byref(p), ip, jp, kp))
    p.dt = dt
    p.nmaxp = nmaxp
    p.inflow_mode = abi.LES_INFLOW_EXTERNAL if inflow == "external" else abi.LES_INFLOW_POWER_LAW
    return p


def synth_cfg(ip, jp, kp, seed=1, **over) -> abi.LesSynthCfg:
    cfg = abi.LesSynthCfg()
    abi.lib().les_synth_default(C.byref(cfg), ip, jp, kp, seed)
    for k, v in over.items():
        setattr(cfg, k, v)
    return cfg


def synthetic_case(ip, jp, kp, seed=1, dt=0.05, inflow="external", nmaxp=50,
                   masks_and_poisson=None, **cfg_over) -> LesCase:
    """Grid, terrain and inflow from the seeded generators; state zeroed as
    init.f95:46-69 leaves it.  Masks and Poisson coefficients are filled by
    `masks_and_poisson(case, zbm)` if given, else on the device with
    les_building_masks / les_poisson_coeffs."""
    L = abi.lib()
    cfg = synth_cfg(ip, jp, kp, seed, **cfg_over)
    case = LesCase(ip, jp, kp, default_params(ip, jp, kp, dt=dt, inflow=inflow, nmaxp=nmaxp))
    A = case.arrays
    for n in FL.METRICS:
        A[n] = FL.alloc(n, ip, jp, kp)
    abi.check(L.les_synth_grid(C.byref(cfg), *[FL.ptr(A[n]) for n in
                                               ("dx1", "dxl", "dy1", "dyl", "z2", "dzn", "dzs",
                                                "dxs", "dys")]))
    zbm = FL.alloc("zbm", ip, jp, kp)
    case.built_fraction = float(L.les_synth_terrain(C.byref(cfg), FL.ptr(zbm)))
    A["zbm"] = zbm
    A["wind_profile"] = FL.alloc("wind_profile", ip, jp, kp)
    abi.check(L.les_synth_inflow(C.byref(cfg), FL.ptr(A["z2"]), FL.ptr(A["dzn"]),
                                 FL.ptr(A["wind_profile"])))
    if inflow != "external":
        del A["wind_profile"]
    for n in FL.STATE + FL.MASKS + FL.POISSON + ["delx1"]:
        A[n] = FL.alloc(n, ip, jp, kp)
    if masks_and_poisson is not None:
        masks_and_poisson(case, zbm)
    else:
        abi.check(L.les_building_masks(ip, jp, kp, FL.ptr(zbm), FL.ptr(A["z2"]), FL.ptr(A["dzn"]),
                                       *[FL.ptr(A[n]) for n in FL.MASKS]))
        abi.check(L.les_poisson_coeffs(ip, jp, kp, FL.ptr(A["dxs"]), FL.ptr(A["dys"]),
                                       FL.ptr(A["dzs"]), *[FL.ptr(A[n]) for n in FL.POISSON]))
    return case


class GpuLes:
    """Device-resident LES state; the B200 twin of run_LES_kernel."""

    def __init__(self, case: LesCase):
        self.case = case
        self.ctx = C.c_void_p()
        abi.check(abi.lib().les_ctx_create(C.byref(case.params), C.byref(self.ctx)))
        self._hf = case.host_fields()
        abi.check(abi.lib().les_ctx_upload(self.ctx, C.byref(self._hf)))

    def close(self):
        if self.ctx:
            abi.lib().les_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def warmup(self, n=1):
        abi.check(abi.lib().les_ctx_warmup(self.ctx, n))

    def step(self, n0, nsteps=1):
        abi.check(abi.lib().les_step(self.ctx, n0, nsteps))

    def sync(self):
        abi.check(abi.lib().les_ctx_sync(self.ctx))

    def set_wind_profile(self, wp: np.ndarray):
        abi.check(abi.lib().les_set_wind_profile(self.ctx, FL.ptr(wp)))

    def metrics(self) -> dict:
        m = abi.LesMetrics()
        abi.check(abi.lib().les_last_metrics(self.ctx, C.byref(m)))
        return {n: getattr(m, n) for n, _ in m._fields_}

    def field_sums(self) -> dict:
        """The reference's WV_DEBUG sums (sum(u), sum(v), ... over each array's
        bounds, velnw.f95:61-68): exact on the device, rounded to FP64."""
        out = (C.c_double * len(abi.FIELD_IDS))()
        abi.check(abi.lib().les_ctx_field_sums(self.ctx, out))
        return {n: out[i] for i, n in enumerate(abi.FIELD_IDS)}

    def download(self, names=None) -> dict:
        """Fortran-layout copies of the state arrays."""
        names = names or FL.STATE + FL.MASKS
        out = {n: FL.alloc(n, self.case.ip, self.case.jp, self.case.kp) for n in names}
        hf = abi.LesHostFields()
        for n in names:
            setattr(hf, n, FL.ptr(out[n]))
        abi.check(abi.lib().les_ctx_download(self.ctx, C.byref(hf)))
        return out

    # -- time statistics and restart files (aveflow.f95, press.f95:191-201,
    # adam.f95:22-31, ifdata.f95:227-247) --
    def aveflow(self, n, n1, nmax, time=0.0, data10=None, data11=None):
        enc = lambda x: None if x is None else str(x).encode()
        abi.check(abi.lib().les_aveflow(self.ctx, n, n1, nmax, time, enc(data10), enc(data11)))

    def _ave_fields(self, stats: dict) -> abi.LesAveflowFields:
        s = abi.LesAveflowFields()
        for n, a in stats.items():
            assert a.dtype == np.float32 and a.flags["F_CONTIGUOUS"]
            setattr(s, n, a.ctypes.data)
        return s

    def aveflow_download(self) -> dict:
        ip, jp, kp = self.case.ip, self.case.jp, self.case.kp
        out = {n: np.zeros((ip, jp, kp), np.float32, order="F") for n in abi.AVEFLOW_CELL}
        out.update({n: np.zeros((ip, kp), np.float32, order="F") for n in abi.AVEFLOW_COL})
        abi.check(abi.lib().les_aveflow_download(self.ctx, C.byref(self._ave_fields(out))))
        return out

    def aveflow_upload(self, stats: dict):
        abi.check(abi.lib().les_aveflow_upload(self.ctx, C.byref(self._ave_fields(stats))))

    def write_restart(self, data20, data21, fghold=None):
        abi.check(abi.lib().les_write_restart(self.ctx, str(data20).encode() if data20 else None,
                                              str(data21).encode() if data21 else None,
                                              None if fghold is None else FL.ptr(fghold)))

    def read_restart(self, data30, data31, fghold=None):
        """Returns (n, time) of the data30 header."""
        n, t = C.c_int(), C.c_float()
        abi.check(abi.lib().les_read_restart(self.ctx, str(data30).encode(), str(data31).encode(),
                                             C.byref(n), C.byref(t),
                                             None if fghold is None else FL.ptr(fghold)))
        return n.value, t.value

    def set_reduction_mode(self, mode: int):
        """Order of the step's global sums: abi.LES_RED_CANONICAL (exact) or
        LES_RED_F_* bits for the reference's serial FP32 loops (parity runs)."""
        abi.check(abi.lib().les_ctx_set_reduction_mode(self.ctx, mode))

    def press_refine_fp64(self, outer, inner, rel_tol=0.0):
        abi.check(abi.lib().les_press_refine_fp64(self.ctx, outer, inner, rel_tol))

    def refine_metrics(self) -> dict:
        m = abi.LesRefineMetrics()
        abi.check(abi.lib().les_last_refine_metrics(self.ctx, C.byref(m)))
        return {n: getattr(m, n) for n, _ in m._fields_}

    def launches(self) -> int:
        return int(abi.lib().les_ctx_launch_count(self.ctx))

    def stream(self) -> int:
        return int(abi.lib().les_ctx_stream(self.ctx) or 0)

    def field(self, name):
        """(device pointer, ox, si, sj, sk) of a state field's box."""
        d = C.c_void_p()
        ox, si, sj, sk = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        abi.check(abi.lib().les_ctx_field(self.ctx, abi.FIELD_IDS.index(name), C.byref(d),
                                          C.byref(ox), C.byref(si), C.byref(sj), C.byref(sk)))
        return d.value, ox.value, si.value, sj.value, sk.value


class GpuAdjoint:
    """Adjoint of whole time steps of a GpuLes (les_adj_* of les_abi.h):
    state slots for checkpoints and recomputation, the step adjoint, the
    resolved-TKE objective and its seed, and the accumulated gradients."""

    def __init__(self, gpu: GpuLes, nslots: int, niter: int):
        self.gpu = gpu
        self.h = C.c_void_p()
        abi.check(abi.lib().les_adj_create(gpu.ctx, nslots, niter, C.byref(self.h)))
        self.nslots = nslots

    def close(self):
        if self.h:
            abi.lib().les_adj_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def save(self, slot):
        abi.check(abi.lib().les_adj_save(self.h, slot))

    def load(self, slot):
        abi.check(abi.lib().les_adj_load(self.h, slot))

    def zero(self):
        abi.check(abi.lib().les_adj_zero(self.h))

    @staticmethod
    def _box(box):
        (i0, i1), (j0, j1), (k0, k1) = box
        return (C.c_int * 6)(i0, i1, j0, j1, k0, k1)

    def tke(self, slot, box) -> float:
        J = C.c_double()
        abi.check(abi.lib().les_adj_tke(self.h, slot, self._box(box), C.byref(J)))
        return J.value

    def seed_tke(self, slot, box, scale):
        abi.check(abi.lib().les_adj_seed_tke(self.h, slot, self._box(box), scale))

    def step_b(self, n, slot):
        abi.check(abi.lib().les_adj_step_b(self.h, n, slot))

    def read(self, state=False):
        c = self.gpu.case
        wp = np.zeros((c.jp, c.kp), np.float64, order="F")
        drag = np.zeros((c.ip, c.jp), np.float64, order="F")
        out = {}
        hf = None
        if state:
            out = {n: FL.alloc(n, c.ip, c.jp, c.kp) for n in FL.STATE}
            hf = abi.LesHostFields()
            for n in FL.STATE:
                setattr(hf, n, FL.ptr(out[n]))
        abi.check(abi.lib().les_adj_read(self.h, wp.ctypes.data, drag.ctypes.data,
                                         C.byref(hf) if hf is not None else None))
        return {"wp": wp, "drag": drag, "state": out}

    def write(self, state_b: dict):
        hf = abi.LesHostFields()
        keep = {n: np.asfortranarray(state_b[n], dtype=np.float32) for n in FL.STATE if n in state_b}
        for n, a in keep.items():
            setattr(hf, n, FL.ptr(a))
        abi.check(abi.lib().les_adj_write(self.h, C.byref(hf)))


def set_drag(gpu: GpuLes, drag):
    """Per-column scale s(i, j) of feedbf's force (f += s fx) for the next
    steps; None restores the reference's s = 1."""
    d = None if drag is None else np.asfortranarray(drag, dtype=np.float32)
    abi.check(abi.lib().les_ctx_set_drag(gpu.ctx, FL.ptr(d) if d is not None else None))


def tke_forward(gpu: GpuLes, adj: GpuAdjoint, n0: int, nt: int, box, ckpt: int, keep_last: bool = False) -> float:
    """J = (1/nt) sum over steps n0 .. n0+nt-1 of the resolved TKE of box
    after the step, from the context's current state, keeping a checkpoint
    every ckpt steps in slots 0, 1, .. (slot 0: the initial state).  With
    keep_last, the inputs of the last segment's steps also go to the slots
    tke_reverse recomputes them into (ceil(nt/ckpt) ...), so that it need not
    recompute that segment."""
    nck = -(-nt // ckpt)
    tl = (nck - 1) * ckpt  # first step of the last segment
    adj.save(0)
    J = 0.0
    for t in range(nt):
        if keep_last and t >= tl:
            adj.save(nck + t - tl)
        gpu.step(n0 + t, 1)
        J += adj.tke(-1, box) / nt
        if (t + 1) % ckpt == 0 and t + 1 < nt:
            adj.save((t + 1) // ckpt)
    return J


def tke_reverse(gpu: GpuLes, adj: GpuAdjoint, n0: int, nt: int, box, ckpt: int, last_kept: bool = False) -> dict:
    """The gradient of tke_forward's J (same arguments, run just before):
    the step adjoint backwards over the checkpoints, each segment's step
    inputs recomputed from its checkpoint into slots ceil(nt/ckpt) ... (the
    last segment's taken as tke_forward left them when it ran with
    keep_last and last_kept is set).  The context is left at the end of the
    first segment.  Returns the FP64 gradients of the inflow profile ("wp",
    jp x kp) and the drag scale ("drag", ip x jp; zero unless set) and the
    adjoint of the initial state."""
    nck = -(-nt // ckpt)
    assert adj.nslots >= nck + ckpt, "too few slots"
    adj.zero()
    for seg in reversed(range(nck)):
        t0, t1 = seg * ckpt, min(seg * ckpt + ckpt, nt)
        if not (last_kept and seg == nck - 1):  # else the context still holds the state after step t1-1
            adj.load(seg)
            for t in range(t0, t1):
                adj.save(nck + t - t0)
                gpu.step(n0 + t, 1)
        for t in reversed(range(t0, t1)):
            adj.seed_tke(-1 if t == t1 - 1 else nck + t + 1 - t0, box, 1.0 / nt)
            adj.step_b(n0 + t, nck + t - t0)
    return adj.read(state=True)


def tke_gradient(gpu: GpuLes, adj: GpuAdjoint, n0: int, nt: int, box, ckpt: int):
    """tke_forward then tke_reverse: (J, gradients), the last segment's step
    inputs kept from the forward run instead of recomputed.  Needs
    ceil(nt/ckpt) + ckpt slots."""
    J = tke_forward(gpu, adj, n0, nt, box, ckpt, keep_last=True)
    return J, tke_reverse(gpu, adj, n0, nt, box, ckpt, last_kept=True)


class Ensemble:
    """Independent domains (GpuLes members) advanced by one graph launch per step."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.ctx.value for m in self.members])
        self.h = C.c_void_p()
        abi.check(abi.lib().les_ensemble_create(len(self.members), arr, C.byref(self.h)))

    def step(self, n0, nsteps=1):
        abi.check(abi.lib().les_ensemble_step(self.h, n0, nsteps))

    def sync(self):
        abi.check(abi.lib().les_ensemble_sync(self.h))

    def stream(self) -> int:
        return int(abi.lib().les_ensemble_stream(self.h) or 0)

    def launches(self) -> int:
        return int(abi.lib().les_ensemble_launch_count(self.h))

    def tune_info(self) -> dict:
        """The ensemble autotuner's candidates (ms per four tuning passes of
        every member) and the one chosen."""
        ms = (C.c_float * 16)()
        n, ch = C.c_int(), C.c_int()
        abi.check(abi.lib().les_ensemble_tune_info(self.h, ms, 16, C.byref(n), C.byref(ch)))
        names = ["own", "1,28,1", "1,28,2", "1,24,1", "1,20,1", "1,12,1", "1,28,1,2", "1,28,2,2", "1,20,1,2",
                 "1,12,1,2"]
        return {"candidates": {names[i] if i < len(names) else str(i): round(ms[i], 3) for i in range(n.value)},
                "chosen": names[ch.value] if 0 <= ch.value < len(names) else None}

    def close(self):
        if self.h:
            abi.lib().les_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
