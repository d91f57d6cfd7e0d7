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

RED_CANONICAL, RED_FAITHFUL = 0, 1

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
