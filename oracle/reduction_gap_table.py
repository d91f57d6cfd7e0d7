"""Effect of the order of the global sums on the fields (test infrastructure).

Runs the oracle with the exact canonical sums and with each of the
reference's serial FP32 loops (press.f95:66-75 rhsav, 87-99 the SOR
residual, 123-133 pav) made faithful on its own and all together, on the
les_synth.h benchmark case, and prints the relative L2 distance of u, v, w,
p to the all-faithful run after 10, 100 and the given number of steps.

    python oracle/reduction_gap_table.py [ip jp kp steps]   (default 150 150 90 200)
"""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import oracle  # noqa: E402

MODES = {"all faithful": oracle.RED_FAITHFUL, "exact (library default)": oracle.RED_CANONICAL,
         "rhsav faithful": oracle.RED_F_RHSAV, "SOR residual faithful": oracle.RED_F_SOR,
         "pav faithful": oracle.RED_F_PAV}


def run(mode, ip, jp, kp, steps, marks):
    oracle.set_reduction_mode(mode)
    try:
        case = oracle.synthetic_case(ip, jp, kp, seed=1)
        oracle.ifdata(case, 1)
        out, n = {}, 1
        for m in marks:
            oracle.run_steps(case, n, m - n + 1)
            n = m + 1
            out[m] = {f: case.a(f).astype(np.float64) for f in ("u", "v", "w", "p")}
        return out
    finally:
        oracle.set_reduction_mode(oracle.RED_CANONICAL)


def main():
    ip, jp, kp, steps = (int(x) for x in sys.argv[1:5]) if len(sys.argv) >= 5 else (150, 150, 90, 200)
    marks = sorted({min(10, steps), min(100, steps), steps})
    res = {name: run(mode, ip, jp, kp, steps, marks) for name, mode in MODES.items()}
    ref = res["all faithful"]
    print(f"{ip}x{jp}x{kp}, relative L2 to the all-faithful run")
    print("| sums | step | u | v | w | p |\n|---|---|---|---|---|---|")
    for name in list(MODES)[1:]:
        for m in marks:
            r = [np.linalg.norm(res[name][m][f] - ref[m][f]) / np.linalg.norm(ref[m][f]) for f in "uvwp"]
            print(f"| {name} | {m} | " + " | ".join(f"{x:.1e}" for x in r) + " |")


if __name__ == "__main__":
    main()
