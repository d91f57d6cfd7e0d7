"""Python binding of the CPU oracle (liblesoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, always as the checker or the
timed CPU baseline -- never by the les_halo_b200 product path.

The oracle restates the reference's Fortran CPU time step
(src/Fortran/*.f95) in C++ with the reference's array bounds and argument
order; see les_oracle.h.  Physics fields are parity-unpinned (the reference
ships no stored outputs and cannot be compiled here: no Fortran compiler);
the halo pack/unpack restatement is pinned to the reference's own C test
programs (src/OpenCL/test_halo_*.c, built by `make -C oracle ref`).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liblesoracle.so"
REF_DIR = HERE / "_ref"

# Reduction modes (les_oracle.h): a bit mask of the sums taken in the
# reference's sequential FP32 order; 0 = the exact canonical sums.
RED_CANONICAL, RED_F_RHSAV, RED_F_SOR, RED_F_PAV, RED_FAITHFUL = 0, 1, 2, 4, 7

_lib = None
_P = C.c_void_p


class OracleParams(C.Structure):
    _fields_ = [("ip", C.c_int), ("jp", C.c_int), ("kp", C.c_int), ("dt", C.c_float),
                ("ro", C.c_float), ("vn", C.c_float), ("alpha", C.c_float), ("beta", C.c_float),
                ("nmaxp", C.c_int), ("pjuge", C.c_float), ("omega", C.c_float)]


FIELD_NAMES = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold", "hold",
               "rhs", "sm", "amask1", "bmask1", "cmask1", "dmask1", "cn1", "cn2l", "cn2s", "cn3l",
               "cn3s", "cn4l", "cn4s", "dx1", "dy1", "dzn", "dzs", "dxs", "dys", "z2", "delx1",
               "wind_profile"]


class OracleFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in FIELD_NAMES]


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.oracle_run_steps.argtypes = [C.POINTER(OracleParams), C.POINTER(OracleFields), C.c_int,
                                       C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.oracle_ifdata.argtypes = [C.POINTER(OracleParams), C.POINTER(OracleFields), C.c_int]
        L.oracle_set_reduction_mode.argtypes = [C.c_int]
        L.oracle_canonical_sum.argtypes = [C.c_int, C.c_int, C.c_int, _P]
        L.oracle_canonical_sum.restype = C.c_double
        L.oracle_last_uout.restype = C.c_float
        L.oracle_halo_buffer_floats.restype = C.c_size_t
        L.oracle_halo_buffer_floats.argtypes = [C.c_uint] * 5 + [C.c_int]
        for n in ("oracle_halo_pack", "oracle_halo_unpack"):
            getattr(L, n).argtypes = [_P, _P] + [C.c_uint] * 5 + [C.c_size_t, C.c_size_t, C.c_int]
        L.oracle_constants.argtypes = [_P] * 4
        for n in ("oracle_grid_reference", "oracle_grid_metrics"):
            getattr(L, n).argtypes = [C.c_int] * 3 + [_P] * 9
        L.oracle_init.argtypes = [C.c_int] * 3 + [_P] * 21
        L.oracle_feedbfm.argtypes = [C.c_int] * 3 + [_P] * 7
        L.oracle_press_ex.argtypes = [C.c_int] * 3 + [_P] * 10 + [C.c_float] + [_P] * 8 + \
            [C.c_int, C.c_float, C.c_float] + [_P] * 3
        L.oracle_press_ex.restype = C.c_int
        L.oracle_aveflow.argtypes = [C.c_int] * 5 + [_P] * 22 + [C.c_int, _P]
        L.oracle_set_press_refine.argtypes = [C.c_int, C.c_int, C.c_double]
        L.oracle_last_refine.argtypes = [C.POINTER(C.c_double)]
        L.oracle_last_refine.restype = C.c_int
        L.oracle_synth_default.restype = None
        L.oracle_synth_default.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_uint64]
        L.oracle_synth_grid.restype = None
        L.oracle_synth_grid.argtypes = [_P] * 10
        L.oracle_synth_terrain.restype = C.c_float
        L.oracle_synth_terrain.argtypes = [_P, _P]
        L.oracle_synth_inflow.restype = None
        L.oracle_synth_inflow.argtypes = [_P] * 4
        _lib = L
    return _lib


def ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["F_CONTIGUOUS"]
    return a.ctypes.data


def params_of(case) -> OracleParams:
    p = case.params
    return OracleParams(case.ip, case.jp, case.kp, p.dt, p.ro, p.vn, p.alpha, p.beta, p.nmaxp,
                        p.pjuge, p.omega)


def fields_of(arrays: dict) -> OracleFields:
    of = OracleFields()
    for n in FIELD_NAMES:
        a = arrays.get(n)
        setattr(of, n, ptr(a) if a is not None else None)
    return of


def set_reduction_mode(mode: int):
    lib().oracle_set_reduction_mode(mode)


def ifdata(case, n=1):
    """ifdata.f95:250-284 on the case's arrays (in place)."""
    lib().oracle_ifdata(C.byref(params_of(case)), C.byref(fields_of(case.arrays)), n)


def run_steps(case, n0, nsteps, nmax=None):
    """main_ocl.f95:233-299 for nsteps steps (in place); returns SOR iteration counts."""
    iters = (C.c_int * max(nsteps, 1))()
    lib().oracle_run_steps(C.byref(params_of(case)), C.byref(fields_of(case.arrays)), n0, nsteps,
                           nmax if nmax is not None else n0 + nsteps - 1, iters)
    return list(iters)[:nsteps]


def masks_and_poisson(case, zbm):
    """init.f95:82-107 + feedbfm.f95:21-63 into case.arrays (CPU)."""
    from les_halo_b200 import fields as FL
    A = case.arrays
    ip, jp, kp = case.ip, case.jp, case.kp
    tmp = {n: FL.alloc(n, ip, jp, kp) for n in ("u", "v", "w", "p")}
    lib().oracle_init(kp, jp, ip, ptr(tmp["u"]), ptr(tmp["v"]), ptr(tmp["w"]), ptr(tmp["p"]),
                      ptr(A["cn2s"]), ptr(A["dxs"]), ptr(A["cn2l"]), ptr(A["cn3s"]), ptr(A["dys"]),
                      ptr(A["cn3l"]), ptr(A["dzs"]), ptr(A["cn4s"]), ptr(A["cn4l"]), ptr(A["cn1"]),
                      ptr(A["amask1"]), ptr(A["bmask1"]), ptr(A["cmask1"]), ptr(A["dmask1"]),
                      ptr(zbm), ptr(A["z2"]), ptr(A["dzn"]))


def halo_pack(array, buffer, im, jm, km, hw, vdim, soa=False, inner=False):
    es, vs = (1, im * jm * km) if soa else (vdim, 1)
    lib().oracle_halo_pack(array.ctypes.data, buffer.ctypes.data, im, jm, km, hw, vdim, es, vs,
                           int(inner))


def halo_unpack(array, buffer, im, jm, km, hw, vdim, soa=False, inner=False):
    es, vs = (1, im * jm * km) if soa else (vdim, 1)
    lib().oracle_halo_unpack(array.ctypes.data, buffer.ctypes.data, im, jm, km, hw, vdim, es, vs,
                             int(inner))


def halo_buffer_floats(im, jm, km, hw, vdim, inner=False):
    return int(lib().oracle_halo_buffer_floats(im, jm, km, hw, vdim, int(inner)))


AVE_CELL = ["aveu", "avev", "avew", "avep", "avel", "aveuu", "avevv", "aveww", "avesm", "avesmsm",
            "uwfx"]
AVE_COL = ["avesu", "avesv", "avesw", "avesuu", "avesvv", "avesww", "uwfxs"]


def ave_alloc(ip, jp, kp):
    """Zeroed aveflow arrays: (ip,jp,kp) and (ip,kp), Fortran order."""
    out = {n: np.zeros((ip, jp, kp), np.float32, order="F") for n in AVE_CELL}
    out.update({n: np.zeros((ip, kp), np.float32, order="F") for n in AVE_COL})
    return out


def aveflow(case, stats: dict, n, n1, nmax):
    """aveflow.f95:42-157 on the case's u, v, w, p, sm into stats (in place)."""
    A = case.arrays
    c = [ptr(stats[k]) for k in AVE_CELL]
    col = [ptr(stats[k]) for k in AVE_COL]
    lib().oracle_aveflow(n, n1, case.kp, case.jp, case.ip, *c, *col[:6], ptr(A["u"]), ptr(A["v"]),
                         ptr(A["w"]), ptr(A["p"]), ptr(A["sm"]), nmax, col[6])


def set_press_refine(outer, inner, tol):
    """FP64-refined press for the following oracle steps (outer = 0: plain)."""
    lib().oracle_set_press_refine(outer, inner, tol)


def last_refine():
    out = (C.c_double * 4)()
    n = lib().oracle_last_refine(out)
    return {"rhsav": out[0], "pav": out[1], "rel_initial": out[2], "rel_final": out[3], "outer": n}


def constants():
    """set.f95:78-82 as the Fortran computes them: ro, vn, alpha, beta."""
    v = [C.c_float() for _ in range(4)]
    lib().oracle_constants(*[C.addressof(x) for x in v])
    return tuple(x.value for x in v)


def synthetic_case(ip, jp, kp, seed=1, dt=0.05, inflow="external", nmaxp=50, **cfg_over):
    """The seeded synthetic case of les_synth.h built on the CPU alone: the
    same generator source (les_halo_b200/csrc/les_synth_gen.h, compiled
    into this library), the oracle's grid metrics (grid.f95:55-82), masks
    and Poisson coefficients (init.f95:82-107, feedbfm.f95:21-63).  Gives
    the arrays of les_halo_b200.synthetic_case bit for bit, without loading
    liblesb200.so; state zeroed as init.f95:46-69 leaves it."""
    from les_halo_b200 import abi as A, fields as FL
    from les_halo_b200.model import LesCase
    L = lib()
    cfg = A.LesSynthCfg()
    L.oracle_synth_default(C.addressof(cfg), ip, jp, kp, seed)
    for k, v in cfg_over.items():
        setattr(cfg, k, v)
    p = A.LesParams()
    p.ip, p.jp, p.kp = ip, jp, kp
    p.dt = dt
    p.ro, p.vn, p.alpha, p.beta = constants()
    p.cs0, p.nmaxp, p.pjuge, p.omega = 0.1, nmaxp, 0.0001, 1.0
    p.inflow_mode = A.LES_INFLOW_EXTERNAL if inflow == "external" else A.LES_INFLOW_POWER_LAW
    p.ical = 0
    case = LesCase(ip, jp, kp, p)
    arr = case.arrays
    for n in FL.METRICS:
        arr[n] = FL.alloc(n, ip, jp, kp)
    L.oracle_synth_grid(C.addressof(cfg), *[ptr(arr[n]) for n in
                                            ("dx1", "dxl", "dy1", "dyl", "z2", "dzn", "dzs", "dxs", "dys")])
    zbm = FL.alloc("zbm", ip, jp, kp)
    case.built_fraction = float(L.oracle_synth_terrain(C.addressof(cfg), ptr(zbm)))
    arr["zbm"] = zbm
    if inflow == "external":
        arr["wind_profile"] = FL.alloc("wind_profile", ip, jp, kp)
        L.oracle_synth_inflow(C.addressof(cfg), ptr(arr["z2"]), ptr(arr["dzn"]), ptr(arr["wind_profile"]))
    for n in FL.STATE + FL.MASKS + FL.POISSON + ["delx1"]:
        arr[n] = FL.alloc(n, ip, jp, kp)
    masks_and_poisson(case, zbm)
    return case
