"""Comparison helpers for the parity tests."""
import numpy as np

from les_halo_b200 import fields as FL


def first_mismatch(name, a, b, ip, jp, kp):
    bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
    if len(bad) == 0:
        return None
    idx = bad[0]
    lows = [lo for lo, _ in FL.bounds(name, ip, jp, kp)]
    ftn = tuple(int(i) + lo for i, lo in zip(idx, lows))
    return f"{name}{ftn}: got {a[tuple(idx)]!r} want {b[tuple(idx)]!r} ({len(bad)} differ)"


def assert_bitexact(got: dict, want: dict, ip, jp, kp, names=None):
    names = names or sorted(got)
    msgs = []
    for n in names:
        m = first_mismatch(n, got[n], want[n], ip, jp, kp)
        if m:
            msgs.append(m)
    assert not msgs, "; ".join(msgs)


def rel_l2(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
