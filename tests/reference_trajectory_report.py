"""Writes the 200-step trajectory comparison of the CUDA step with the
reference's own step code as a markdown report (a study driver, not a test;
tests/test_reference_trajectory.py asserts the same runs).

    python tests/reference_trajectory_report.py [--out report.md] [--no-gpu]

Cases: the plain-step world as configured (32^3, 3 channels, 9 kernels of
radius 8, seed 0) and the same world with asymptotic growth (seeds 0, 3).
Each row: the GPU against the reference build (float FFT stand-in), then the
reference build with a float64 FFT against the same build (tests/trajectory.py
describes the three runs and the columns).  With --no-gpu the GPU columns are
left out.
"""
from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from lenia_b200 import params as P  # noqa: E402
from trajectory import asymptotic_variant, run_trajectories  # noqa: E402

SHOW = (1, 2, 3, 4, 5, 10, 20, 30, 50, 75, 100, 125, 150, 175, 200)


def table(rows, rows64, steps):
    out = ["| step | GPU: flips | A L∞ | A L2 | U L∞ | F L∞ | F L2 | mass | ref64: flips | A L∞ | A L2 | mass |",
           "|---|---|---|---|---|---|---|---|---|---|---|---|"]
    for i in range(steps):
        q = rows64[i]
        if q["step"] not in SHOW:
            continue
        if rows:
            r = rows[i]
            g = (f"{r['flips']} | {r['A_inf']:.2e} | {r['A_l2']:.2e} | {r['U_inf']:.2e} | {r['F_inf']:.2e} | "
                 f"{r['F_l2']:.2e} | {r['mass_rel']:.2e}")
        else:
            g = " | ".join(["-"] * 7)
        out.append(f"| {q['step']} | {g} | {q['flips']} | {q['A_inf']:.2e} | {q['A_l2']:.2e} | {q['mass_rel']:.2e} |")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--no-gpu", action="store_true")
    args = ap.parse_args()
    lines = ["# 200 steps of the plain-step world: CUDA step vs the reference's own step code", ""]
    cases = [("as configured (seed 0)", P.config0(seed=0)),
             ("asymptotic growth, seed 0", asymptotic_variant(P.config0(seed=0))),
             ("asymptotic growth, seed 3", asymptotic_variant(P.config0(seed=3)))]
    for name, wl in cases:
        rows, rows64 = run_trajectories(wl, args.steps, with_gpu=not args.no_gpu)
        ff = next((r["step"] for r in rows if r["flips"]), None) if rows else None
        ff64 = next((r["step"] for r in rows64 if r["flips"]), None)
        lines += [f"## {name}", "",
                  f"First growth-table bin flip: GPU step {ff}, float64-FFT reference build step {ff64}.  "
                  f"Mass at the last step: {rows64[-1]['mass']:.1f} (reference build).", ""]
        lines += table(rows, rows64, args.steps)
        lines.append("")
        print(f"{name}: done", file=sys.stderr)
    text = "\n".join(lines) + "\n"
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)
    print(text)


if __name__ == "__main__":
    main()
