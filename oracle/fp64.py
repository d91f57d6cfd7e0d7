"""The oracle instantiated in double precision (liblesoracle64.so).

TEST INFRASTRUCTURE ONLY, like the rest of oracle/: the FP64 reference
against which the FP32 time step's error is stated.  The library is the
same C++ restatement of the Fortran step compiled with every `float` made
`double` and every float literal made a double literal (oracle/Makefile),
run with plain sequential FP64 sums (the faithful reduction mode).

An FP64 case is built from an FP32 case's inputs: the grid metrics, the
terrain heights and the inflow profile are converted exactly to double;
the Poisson coefficients, masks and the initial state are recomputed in
double by the restated init.f95 / feedbfm.f95.
"""
from __future__ import annotations

import ctypes as C
import subprocess

import numpy as np

from . import FIELD_NAMES, HERE, RED_FAITHFUL

LIB_PATH = HERE / "liblesoracle64.so"
_lib = None
_P = C.c_void_p


class OracleParams64(C.Structure):
    _fields_ = [("ip", C.c_int), ("jp", C.c_int), ("kp", C.c_int), ("dt", C.c_double),
                ("ro", C.c_double), ("vn", C.c_double), ("alpha", C.c_double), ("beta", C.c_double),
                ("nmaxp", C.c_int), ("pjuge", C.c_double), ("omega", C.c_double)]


class OracleFields64(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in FIELD_NAMES]


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
        L = C.CDLL(str(LIB_PATH))
        L.oracle_run_steps.argtypes = [C.POINTER(OracleParams64), C.POINTER(OracleFields64), C.c_int,
                                       C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.oracle_ifdata.argtypes = [C.POINTER(OracleParams64), C.POINTER(OracleFields64), C.c_int]
        L.oracle_set_reduction_mode.argtypes = [C.c_int]
        L.oracle_init.argtypes = [C.c_int] * 3 + [_P] * 21
        L.oracle_set_reduction_mode(RED_FAITHFUL)
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
    return a.ctypes.data


class Case64:
    """Float64 arrays with the Fortran bounds of an FP32 case."""

    def __init__(self, case32):
        from les_halo_b200 import fields as FL
        self.ip, self.jp, self.kp = case32.ip, case32.jp, case32.kp
        ip, jp, kp = self.ip, self.jp, self.kp
        p = case32.params
        self.params = OracleParams64(ip, jp, kp, float(np.float32(p.dt)), float(np.float32(p.ro)),
                                     float(np.float32(p.vn)), float(np.float32(p.alpha)),
                                     float(np.float32(p.beta)), int(p.nmaxp), float(np.float32(p.pjuge)),
                                     float(np.float32(p.omega)))
        A32 = case32.arrays
        self.arrays = {n: np.asfortranarray(a.astype(np.float64)) for n, a in A32.items()}
        A = self.arrays
        tmp = {n: np.asfortranarray(FL.alloc(n, ip, jp, kp).astype(np.float64)) for n in ("u", "v", "w", "p")}
        lib().oracle_init(kp, jp, ip, _ptr(tmp["u"]), _ptr(tmp["v"]), _ptr(tmp["w"]), _ptr(tmp["p"]),
                          _ptr(A["cn2s"]), _ptr(A["dxs"]), _ptr(A["cn2l"]), _ptr(A["cn3s"]), _ptr(A["dys"]),
                          _ptr(A["cn3l"]), _ptr(A["dzs"]), _ptr(A["cn4s"]), _ptr(A["cn4l"]), _ptr(A["cn1"]),
                          _ptr(A["amask1"]), _ptr(A["bmask1"]), _ptr(A["cmask1"]), _ptr(A["dmask1"]),
                          _ptr(A["zbm"]), _ptr(A["z2"]), _ptr(A["dzn"]))

    def a(self, name):
        return self.arrays[name]

    def _fields(self):
        of = OracleFields64()
        for n in FIELD_NAMES:
            setattr(of, n, _ptr(self.arrays.get(n)))
        return of

    def ifdata(self, n=1):
        lib().oracle_ifdata(C.byref(self.params), C.byref(self._fields()), n)

    def run_steps(self, n0, nsteps):
        iters = (C.c_int * max(nsteps, 1))()
        lib().oracle_run_steps(C.byref(self.params), C.byref(self._fields()), n0, nsteps, n0 + nsteps - 1,
                               iters)
        return list(iters)[:nsteps]
