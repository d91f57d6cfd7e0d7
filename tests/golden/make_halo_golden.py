"""Generate tests/golden/halo_kat.json from the reference's own halo tests.

Runs the four C programs of the reference (src/OpenCL/test_halo_read.c,
test_halo_write.c, test_halo_read_correct.c, test_halo_write_correct.c),
compiled unmodified from their sources by `make -C oracle ref` into
oracle/_ref/, and records every number they print, in order.  The programs
print but do not assert; the recorded output is the known answer.

Usage: python tests/golden/make_halo_golden.py   (needs the reference tree)
"""
import json
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
REF = ROOT / "oracle" / "_ref"
NUM = re.compile(r"-?\d+(?:\.\d+)?(?:e[-+]?\d+)?")

# Parameters as written in each program's main().
PROGRAMS = {
    "test_halo_read": dict(im=20, jm=20, km=2, h_w=3, v_dim=2),
    "test_halo_write": dict(im=30, jm=40, km=2, h_w=3, v_dim=2),
    "test_halo_read_correct": dict(im=20, jm=20, km=2, h_w=1, v_dim=2),
    "test_halo_write_correct": dict(im=20, jm=20, km=2, h_w=3, v_dim=2),
}


def main():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref"], check=True)
    out = {}
    for prog, prm in PROGRAMS.items():
        txt = subprocess.run([str(REF / prog)], capture_output=True, text=True, check=True).stdout
        nums = [float(x) for x in NUM.findall(txt)]
        out[prog] = dict(params=prm, printed=nums,
                         source=f"src/OpenCL/{prog}.c (reference), stdout numbers in order")
    dst = Path(__file__).resolve().parent / "halo_kat.json"
    dst.write_text(json.dumps(out))
    print(dst, {k: len(v["printed"]) for k, v in out.items()})


if __name__ == "__main__":
    main()
