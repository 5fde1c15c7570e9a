"""Precision of the convolution modes against the float64 oracle.

Runs the plain-step configuration (3 channels, 9 kernels drawn as in the
32^3 plain step, central differences, RT reintegration with sigma 0.65,
periodic borders) on a width^3 grid with kernels of the given radius, from
the plain step's seeded U(0,1) cube scaled to half the side, in each
convolution mode of the library (FFT in FP32, direct BF16, direct BF16x3),
next to oracle/fp64.py on the same GPU in float64.  Per step and per mode:

  U     max |u - u64| and ||u - u64|| / ||u64|| over all kernels' u_k
  F     the same for the flow field F (3 x C x N)
  mass  max over channels of |sum A - sum A64| / sum A64

Regimes: "trajectory" (every path runs its own steps from the same start;
errors include divergence of the dynamics), "one-step" (before each step
every world is reset to the oracle's state, so the errors are those of one
step's arithmetic) and "one-step-exact" (the same against the oracle with
the exact bell in place of the growth table: the table's quantisation then
counts as error).

  python tests/precision_study.py --width 256 --radius 20 --steps 100 \
      --json out.json --md summary.md [--exact-bell]

--exact-bell runs worlds and oracle with the exact-bell growth option (no
growth table), so that no growth-table bin flips mask the arithmetic.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

MODES = ("FFT", "DIRECT_BF16", "DIRECT_BF16X3")


def workload(width: int, radius: int, seed: int, exact_bell: bool = False):
    from lenia_b200 import params as P
    wl = P.config2(seed=seed, width=width, radius=radius)
    wl.desc.exact_bell = exact_bell
    return wl.desc, wl.kernels, wl.A0


def _err(x, ref):
    import torch
    d = (x.double() - ref).abs()
    return float(d.max()), float(torch.linalg.vector_norm(x.double() - ref) / torch.linalg.vector_norm(ref))


def run(width=256, radius=20, steps=100, seed=2, regime="trajectory", modes=MODES, log=None, exact_bell=False):
    import torch
    from lenia_b200.world import World
    from oracle import fp64
    dev = torch.device("cuda")
    desc, ks, A0 = workload(width, radius, seed, exact_bell)
    C, K, N = desc.channels, len(ks), desc.cells
    ref = fp64.Fp64Step(desc, ks, fp64.Xp(dev), exact_bell=exact_bell or regime == "one-step-exact")
    ref.set_state(A0)
    worlds = {}
    for m in modes:
        w = World(desc, ks)
        w.set_conv_mode(m)
        w.set_debug(True)
        w.set_state(A0.ravel())
        worlds[m] = w
    bufU = torch.empty(K * N, dtype=torch.float32, device=dev)
    bufF = torch.empty(3 * C * N, dtype=torch.float32, device=dev)
    bufA = torch.empty(C * N, dtype=torch.float32, device=dev)
    rows = []
    for s in range(steps):
        if regime.startswith("one-step"):
            st = ref.state
            for w in worlds.values():
                for name, v in (("A", st.A), ("V", st.V), ("GA", st.GA), ("SUM", st.SUM)):
                    w.set(name, v.float().reshape(-1).contiguous())
        t0 = time.time()
        ref.step()
        torch.cuda.synchronize()
        t_ref = time.time() - t0
        u64 = torch.stack([u.reshape(-1) for u in ref.U]).reshape(-1)
        F64 = torch.stack([torch.stack([f.reshape(-1) for f in row]) for row in ref.F]).reshape(-1)
        m64 = np.array(ref.mass())
        row = {"step": s + 1, "ref_s": round(t_ref, 3)}
        for m, w in worlds.items():
            w.step(1)
            w.sync()
            w.get("U", out=bufU)
            w.get("F", out=bufF)
            w.get("A", out=bufA)
            mass = bufA.double().reshape(C, -1).sum(dim=1).cpu().numpy()
            row[m] = {"U": _err(bufU, u64), "F": _err(bufF, F64),
                      "mass": float(np.max(np.abs(mass - m64) / np.abs(m64)))}
        rows.append(row)
        if log:
            print(json.dumps(row), file=log, flush=True)
    for w in worlds.values():
        w.close()
    return rows


def summary_md(results: dict, width: int, radius: int, steps: int) -> str:
    out = [f"# Convolution precision against the float64 oracle, {width}^3, radius {radius}, {steps} steps", ""]
    for regime, rows in results.items():
        out.append(f"## {regime}")
        out.append("")
        out.append("| mode | step | U L-inf | U rel L2 | F L-inf | F rel L2 | mass rel |")
        out.append("|---|---|---|---|---|---|---|")
        picks = sorted({1, min(10, steps), steps})
        for m in MODES:
            if m not in rows[0]:
                continue
            for s in picks:
                r = rows[s - 1][m]
                out.append(f"| {m} | {s} | {r['U'][0]:.2e} | {r['U'][1]:.2e} | {r['F'][0]:.2e} | {r['F'][1]:.2e} | "
                           f"{r['mass']:.2e} |")
            worst = {k: max(rows[i][m][k][0] if k != 'mass' else rows[i][m][k] for i in range(steps))
                     for k in ("U", "F", "mass")}
            out.append(f"| {m} | max over steps | {worst['U']:.2e} | | {worst['F']:.2e} | | {worst['mass']:.2e} |")
        out.append("")
    return "\n".join(out) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--radius", type=int, default=20)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--regimes", default="one-step,trajectory")
    ap.add_argument("--json", default=None)
    ap.add_argument("--md", default=None)
    ap.add_argument("--exact-bell", action="store_true",
                    help="worlds and oracle with the exact-bell growth option (no growth table)")
    a = ap.parse_args()
    results = {}
    for regime in a.regimes.split(","):
        results[regime] = run(a.width, a.radius, a.steps, a.seed, regime, log=sys.stdout, exact_bell=a.exact_bell)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(results, f)
    md = summary_md(results, a.width, a.radius, a.steps)
    if a.exact_bell:
        md = md.replace("float64 oracle,", "float64 oracle (exact-bell growth in worlds and oracle),", 1)
    if a.md:
        with open(a.md, "w") as f:
            f.write(md)
    print(md)


if __name__ == "__main__":
    main()
