"""Fortran-layout arrays of the LES model and their bounds.

Bounds follow the reference's declarations (src/Fortran/main_ocl.f95:41-167)
with ip=im, jp=jm, kp=km.  Arrays are numpy float32 in Fortran (column-major)
order, so ``a.ctypes.data`` is exactly what the reference's Fortran host
passes by reference.
"""
from __future__ import annotations

import numpy as np

# name -> (lower, upper) per dimension; ip/jp/kp substituted at allocation.
_BOUNDS = {
    "u": ("0:ip+1", "-1:jp+1", "0:kp+1"),
    "v": ("0:ip+1", "-1:jp+1", "0:kp+1"),
    "w": ("0:ip+1", "-1:jp+1", "-1:kp+1"),
    "p": ("0:ip+2", "0:jp+2", "0:kp+1"),
    "usum": ("0:ip", "0:jp", "0:kp"),
    "vsum": ("0:ip", "0:jp", "0:kp"),
    "wsum": ("0:ip", "0:jp", "0:kp"),
    "f": ("0:ip", "0:jp", "0:kp"),
    "g": ("0:ip", "0:jp", "0:kp"),
    "h": ("0:ip", "0:jp", "0:kp"),
    "fx": ("0:ip", "0:jp", "0:kp"),
    "fy": ("0:ip", "0:jp", "0:kp"),
    "fz": ("0:ip", "0:jp", "0:kp"),
    "fold": ("1:ip", "1:jp", "1:kp"),
    "gold": ("1:ip", "1:jp", "1:kp"),
    "hold": ("1:ip", "1:jp", "1:kp"),
    "cn1": ("1:ip", "1:jp", "1:kp"),
    "rhs": ("0:ip+1", "0:jp+1", "0:kp+1"),
    "sm": ("-1:ip+1", "-1:jp+1", "0:kp+1"),
    "amask1": ("0:ip+1", "0:jp+1", "0:kp+1"),
    "dmask1": ("0:ip+1", "0:jp+1", "0:kp+1"),
    "bmask1": ("-1:ip+1", "0:jp+1", "0:kp+1"),
    "cmask1": ("0:ip+1", "-1:jp+1", "0:kp+1"),
    "dfu1": ("0:ip", "1:jp", "1:kp"),
    "dfv1": ("1:ip", "0:jp", "1:kp"),
    "dfw1": ("1:ip", "1:jp", "1:kp"),
    "cn2l": ("1:ip",), "cn2s": ("1:ip",),
    "cn3l": ("1:jp",), "cn3s": ("1:jp",),
    "cn4l": ("1:kp",), "cn4s": ("1:kp",),
    "dx1": ("-1:ip+1",), "dxl": ("0:ip",), "dxs": ("0:ip",),
    "dy1": ("0:jp+1",), "dyl": ("0:jp",), "dys": ("0:jp",),
    "dzn": ("-1:kp+2",), "dzs": ("-1:kp+2",),
    "z2": ("1:kp+2",), "delx1": ("1:kp",),
    "zbm": ("-1:ip+1", "-1:jp+1"),
    "wind_profile": ("1:jp", "1:kp"),
}
for _n in range(1, 10):
    wide = ("-1:ip+2", "0:jp+2", "0:kp+2") if _n in (1, 5) else ("0:ip+2", "0:jp+2", "0:kp+2")
    _BOUNDS[f"diu{_n}"] = wide
    _BOUNDS[f"cov{_n}"] = wide
    _BOUNDS[f"nou{_n}"] = wide

STATE = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold", "hold",
         "rhs", "sm"]
MASKS = ["amask1", "bmask1", "cmask1", "dmask1"]
POISSON = ["cn1", "cn2l", "cn2s", "cn3l", "cn3s", "cn4l", "cn4s"]
METRICS = ["dx1", "dxl", "dy1", "dyl", "dzn", "dzs", "dxs", "dys", "z2"]


def _ev(expr: str, ip: int, jp: int, kp: int) -> int:
    return int(eval(expr, {"__builtins__": {}}, {"ip": ip, "jp": jp, "kp": kp}))


def bounds(name: str, ip: int, jp: int, kp: int):
    """[(lower, upper), ...] of array `name`."""
    out = []
    for d in _BOUNDS[name]:
        lo, hi = d.split(":")
        out.append((_ev(lo, ip, jp, kp), _ev(hi, ip, jp, kp)))
    return out


def alloc(name: str, ip: int, jp: int, kp: int, fill: float = 0.0) -> np.ndarray:
    shape = [hi - lo + 1 for lo, hi in bounds(name, ip, jp, kp)]
    a = np.empty(shape, dtype=np.float32, order="F")
    a[...] = fill
    return a


def index(name: str, ip: int, jp: int, kp: int, *idx):
    """numpy index of Fortran element idx (ints or slices with Fortran ends)."""
    out = []
    for (lo, hi), x in zip(bounds(name, ip, jp, kp), idx):
        if isinstance(x, slice):
            a = lo if x.start is None else x.start
            b = hi if x.stop is None else x.stop
            out.append(slice(a - lo, b - lo + 1))
        else:
            out.append(x - lo)
    return tuple(out)


def interior(name: str, arr: np.ndarray, ip: int, jp: int, kp: int) -> np.ndarray:
    """View of (1:ip, 1:jp, 1:kp) of a 3-D field."""
    return arr[index(name, ip, jp, kp, slice(1, ip), slice(1, jp), slice(1, kp))]


def ptr(a):
    """Address of the first element (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["F_CONTIGUOUS"], "need Fortran-ordered float32"
    return a.ctypes.data


def set_interior(name: str, arr: np.ndarray, values: np.ndarray, ip: int, jp: int, kp: int):
    """arr(1:ip, 1:jp, 1:kp) = values (ghosts untouched)."""
    arr[index(name, ip, jp, kp, slice(1, ip), slice(1, jp), slice(1, kp))] = values
