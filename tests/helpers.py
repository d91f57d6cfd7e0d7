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


# gfortran sequential unformatted records, big-endian (the reference's
# -fconvert=big-endian build): 4-byte count, data, 4-byte count.
def read_fortran_records(path):
    data = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(data):
        n = int.from_bytes(data[pos:pos + 4], "big")
        body = data[pos + 4:pos + 4 + n]
        assert int.from_bytes(data[pos + 4 + n:pos + 8 + n], "big") == n, "bad end marker"
        out.append(body)
        pos += 8 + n
    return out


def write_fortran_records(path, records):
    with open(path, "wb") as f:
        for r in records:
            b = r if isinstance(r, bytes) else np.ascontiguousarray(r).tobytes()
            f.write(len(b).to_bytes(4, "big") + b + len(b).to_bytes(4, "big"))


def be_floats(arr):
    """Interior array as the reference writes it: i fastest, big-endian."""
    return np.asarray(arr, np.float32).ravel(order="F").astype(">f4").tobytes()
