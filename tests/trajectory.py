"""Long trajectories of the CUDA step beside the reference's own code.

Three runs of one world advance together, step by step:

* `gpu`   — the CUDA library (lenia_b200.World);
* `ref`   — the reference's own step code (lenia.cpp, reintegration.cpp,
  transposition.cpp, mesh.cpp compiled unmodified, oracle/_ref), with the
  project's float FFT standing in for FFTW;
* `ref64` — the same reference code linked with a float64 FFT stand-in
  (oracle/refshim/fftw_shim64.c): a second, equally valid build of the
  reference, whose distance from `ref` measures how far two correct FFTs let
  the reference's own step drift apart.

The growth table is indexed with (int)(u * 255) (lenia.h:79-84), a
truncation: any two FFTs whose u differ in the last bits disagree on the
table entry for the few cells whose u * 255 sits next to an integer (a "bin
flip"), after which the two trajectories follow different paths.  Until the
first flip, H, F, MU and A of the CUDA step equal the reference's bit for
bit; u itself differs at FFT rounding level from the first step on.

Per step and per field the rows hold the relative L-infinity distance
max|a - b| / max|b| and the relative L2 distance ||a - b|| / ||b|| of A, U
and F, the relative difference of the total mass, and the number of (kernel,
cell) pairs whose table index differs from the reference's.
"""
from __future__ import annotations

import numpy as np

F255 = np.float32(255.0)


def rel_inf(a: np.ndarray, b: np.ndarray) -> float:
    den = float(np.abs(b).max())
    return float(np.abs(a.astype(np.float64) - b).max()) / den if den > 0 else float(np.abs(a).max())


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    b64 = b.astype(np.float64)
    den = float(np.linalg.norm(b64))
    num = float(np.linalg.norm(a.astype(np.float64) - b64))
    return num / den if den > 0 else num


def lut_flips(u: np.ndarray, u_ref: np.ndarray) -> int:
    """(kernel, cell) pairs whose growth-table index (int)(u * 255) differs."""
    return int(((u * F255).astype(np.int32) != (u_ref * F255).astype(np.int32)).sum())


def compare_row(step: int, got: dict, ref: dict) -> dict:
    row = {"step": step, "flips": lut_flips(got["U"], ref["U"])}
    for name in ("A", "U", "F"):
        row[f"{name}_inf"] = rel_inf(got[name], ref[name])
        row[f"{name}_l2"] = rel_l2(got[name], ref[name])
        row[f"{name}_equal"] = bool(np.array_equal(got[name], ref[name]))
    m, mr = float(got["A"].astype(np.float64).sum()), float(ref["A"].astype(np.float64).sum())
    row["mass_rel"] = abs(m - mr) / mr if mr > 0 else abs(m)
    row["mass"] = m
    return row


def fields(run) -> dict:
    return {name: run.get(name) for name in ("A", "U", "F")}


def asymptotic_variant(wl):
    """The world with asymptotic growth H += h (LUT - A) on channels 0-2
    (mt_fft_step, lenia.cpp:496-594; the ChannelData flag, render.h): its
    mass can fall as well as rise, so the pattern keeps changing instead of
    filling the grid."""
    import dataclasses
    from lenia_b200.params import Workload
    desc = dataclasses.replace(wl.desc, asymptotic=(True, True, True, False))
    return Workload(desc, wl.kernels, wl.A0)


def run_trajectories(wl, steps: int, with_gpu: bool = True):
    """Advances the CUDA world (with_gpu), the reference build and its float64
    FFT twin `steps` steps from wl.A0; returns (rows gpu vs ref, rows ref64 vs
    ref)."""
    from oracle import oracle as O
    p = wl.desc.as_dict()
    ks = [k.as_dict() for k in wl.kernels]
    ref = O.RefOracle(p, ks, lib=O.REF_LIB)
    ref.set_state(A=wl.A0.ravel())
    ref64 = O.RefOracle(p, ks, lib=O.REF_LIB_FFT64)
    ref64.set_state(A=wl.A0.ravel())
    gpu = None
    if with_gpu:
        from lenia_b200.world import World
        gpu = World(wl.desc, wl.kernels)
        gpu.set_debug(True)
        gpu.set_state(wl.A0.ravel())
    rows_gpu, rows_64 = [], []
    try:
        for s in range(1, steps + 1):
            ref.step(1)
            ref64.step(1)
            fr = fields(ref)
            rows_64.append(compare_row(s, fields(ref64), fr))
            if gpu is not None:
                gpu.step(1)
                gpu.sync()
                rows_gpu.append(compare_row(s, fields(gpu), fr))
    finally:
        if gpu is not None:
            gpu.close()
    return rows_gpu, rows_64
