"""Labels for the persistent-pattern search (the caller of the step in the
learned-proposal configuration; the reference has no counterpart).

From the per-channel grid statistics of lenia_world_stats / lenia_batch_stats
(mass; the circular moments sum a cos(2 pi x / W), sum a sin(2 pi x / W) per
axis; max; cells above a fill threshold) this module derives
  - channel mass ratios and the total mass,
  - the torus-aware centroid: per axis the angle of the mass-weighted mean of
    e^(2 pi i x / W), mapped back to [0, W),
  - the mass-weighted spread: per axis the circular standard deviation
    W / (2 pi) sqrt(-2 ln R), R = |sum a e^(i theta)| / sum a (0 for a point
    mass, large for a spread-out field), combined over axes as a root sum of
    squares,
  - the centroid velocity between two observations (torus-wrapped),
and labels a run at its final observation:
  dead        total mass below a quarter of the initial mass, or max below
              0.05;
  exploding   non-finite statistics, more than half of the cells above the
              fill threshold, or a spread above a fifth of the side;
  persistent  otherwise (alive and bounded).
The thresholds are this project's choice (the reference defines no labels).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Sequence

import numpy as np

MASS, CX, SX, CY, SY, CZ, SZ, MAX, FILL = range(9)
LABELS = ("dead", "exploding", "persistent")


def _axis(cos_sum, sin_sum, mass, ext):
    """(centroid in [0, ext), circular standard deviation) of one axis."""
    ang = np.arctan2(sin_sum, cos_sum)
    c = (ang % (2 * np.pi)) * ext / (2 * np.pi)
    with np.errstate(divide="ignore", invalid="ignore"):
        R = np.hypot(cos_sum, sin_sum) / mass
        sd = ext / (2 * np.pi) * np.sqrt(np.maximum(-2.0 * np.log(np.clip(R, 1e-300, 1.0)), 0.0))
    return c, sd


@dataclass
class Summary:
    mass: np.ndarray        # (C,)
    total: float
    ratios: np.ndarray      # (C,)
    centroid: np.ndarray    # (C + 1, 3): per channel, then of all channels
    spread: np.ndarray      # (C + 1,)
    max: np.ndarray         # (C,)
    fill: float             # fraction of cells (over channels) above the threshold


def summarize(stats: np.ndarray, width: int, height: int) -> Summary:
    st = np.asarray(stats, dtype=np.float64)
    C = st.shape[0]
    ext = (width, height, width)
    mass = st[:, MASS]
    total = float(mass.sum())
    with np.errstate(divide="ignore", invalid="ignore"):
        ratios = mass / total
    cent = np.zeros((C + 1, 3))
    sd = np.zeros((C + 1, 3))
    rows = [st[c] for c in range(C)] + [st.sum(axis=0)]
    for r, row in enumerate(rows):
        for a, (ci, si) in enumerate(((CX, SX), (CY, SY), (CZ, SZ))):
            cent[r, a], sd[r, a] = _axis(row[ci], row[si], row[MASS], ext[a])
    cells = width * height * width
    return Summary(mass=mass, total=total, ratios=ratios, centroid=cent, spread=np.sqrt((sd ** 2).sum(axis=1)),
                   max=st[:, MAX], fill=float(st[:, FILL].sum() / (C * cells)))


def torus_delta(a: np.ndarray, b: np.ndarray, ext: Sequence[float]) -> np.ndarray:
    """b - a per axis, wrapped into [-ext/2, ext/2)."""
    e = np.asarray(ext, dtype=np.float64)
    return (np.asarray(b) - np.asarray(a) + e / 2) % e - e / 2


def centroid_speed(s0: Summary, s1: Summary, steps: int, width: int, height: int) -> np.ndarray:
    """Centroid speed (cells per step) per channel and of all channels."""
    d = torus_delta(s0.centroid, s1.centroid, (width, height, width))
    return np.sqrt((d ** 2).sum(axis=1)) / max(steps, 1)


def features(s_prev: Summary, s_obs: Summary, initial_mass: float, steps_between: int, width: int,
             height: int) -> np.ndarray:
    """The 16 early-step statistics for three channels: mass ratios (3), total
    mass over the initial mass (1), spread per channel and overall relative to
    the side (4), centroid speed per channel and overall (4), max per channel
    (3), fill fraction (1)."""
    C = len(s_obs.mass)
    assert C == 3, "the feature vector is defined for three channels"
    sp = centroid_speed(s_prev, s_obs, steps_between, width, height)
    f = np.concatenate([s_obs.ratios, [s_obs.total / initial_mass if initial_mass > 0 else 0.0],
                        s_obs.spread / width, sp, s_obs.max, [s_obs.fill]])
    return np.nan_to_num(f, nan=0.0, posinf=1e6, neginf=-1e6)


def label(s_final: Summary, initial_mass: float, width: int) -> str:
    vals = np.concatenate([s_final.mass, s_final.max, [s_final.total, s_final.fill]])
    if not np.all(np.isfinite(vals)):
        return "exploding"
    if s_final.total < 0.25 * initial_mass or s_final.max.max() < 0.05:
        return "dead"
    if s_final.fill > 0.5 or s_final.spread[-1] > 0.2 * width:
        return "exploding"
    return "persistent"


def run_labels(workloads, steps: int = 1000, observe: int = 50, lanes: int = 0, fill_threshold: float = 0.1
               ) -> Dict[str, np.ndarray]:
    """Steps the worlds as one batch and returns, per world, the features at
    step `observe` (against step observe - 1), the label at step `steps`, and
    the label index.  Every world must have three channels."""
    from .batch import Batch
    b = Batch([wl.desc for wl in workloads], [wl.kernels for wl in workloads], lanes=lanes)
    for i, wl in enumerate(workloads):
        b.set_state(i, wl.A0)
    init = [summarize(s, wl.desc.width, wl.desc.height) for s, wl in zip(b.stats(fill_threshold), workloads)]
    b.step(observe - 1)
    prev = [summarize(s, wl.desc.width, wl.desc.height) for s, wl in zip(b.stats(fill_threshold), workloads)]
    b.step(1)
    obs = [summarize(s, wl.desc.width, wl.desc.height) for s, wl in zip(b.stats(fill_threshold), workloads)]
    b.step(steps - observe)
    fin = [summarize(s, wl.desc.width, wl.desc.height) for s, wl in zip(b.stats(fill_threshold), workloads)]
    b.sync()
    b.close()
    feats = np.stack([features(p, o, i.total, 1, wl.desc.width, wl.desc.height)
                      for p, o, i, wl in zip(prev, obs, init, workloads)])
    labs = [label(f, i.total, wl.desc.width) for f, i, wl in zip(fin, init, workloads)]
    return {"features": feats, "labels": np.array(labs), "label_index": np.array([LABELS.index(x) for x in labs])}
