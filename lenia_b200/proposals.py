"""Learned proposals for the persistent-pattern search, against uniform
sampling.

Candidates are kernel sets drawn as in config 0 (one kernel per channel pair,
1-3 shells, b ~ U(0,1), m ~ U(0.1,0.5), s ~ U(0.01,0.18), h ~ U(0.01,1)) on
cubic worlds with 3 channels and a seeded cube, run as mass-conserving Flow
Lenia (see `candidates`).  A run is a *hit* when its
label at the final step is "persistent" (alive and bounded, lenia_b200.labels).

  uniform  every candidate runs to the final step;
  learned  every candidate runs to the observation step; the network scores
           its 79 inputs (the 63 kernel parameters and the 16 statistics of
           lenia_b200.labels.features); only the top fraction continues to
           the final step, from its saved state.

Both arms are timed on the GPU (CUDA events around the batch steps and the
network); hits per GPU-second compares them.  Every hit of the learned arm is
confirmed by the plain simulation of that candidate to the final step.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Dict, List, Sequence

import numpy as np

from . import labels as L
from . import params as P

N_KERNELS = 9
KERNEL_FEATURES = 7  # b0, b1, b2, m, s, h, r_a


def candidates(n: int, seed: int, width: int = 32, asymptotic: bool = False,
               growth_type: int = P.GROWTH_NOGROWTH, sigma: float = 0.5) -> List[P.Workload]:
    """n candidate worlds, mass-conserving Flow Lenia by default: sigma 0.5
    (the reference's reintegration spreads (2 sigma)^3 / (4 sigma^2) of a
    cell's mass per step with S_NORM 0, exactly 1 only at sigma 0.5; at the
    benchmark's 0.65 every world fills the grid) and no growth (with the
    reference's growth, h bell >= 0, every random kernel set fills the grid;
    asymptotic channels fill most of it)."""
    out = []
    for i in range(n):
        rng = np.random.default_rng((seed, i))
        desc = P.WorldDesc(width=width, height=width, channels=3, timestep=0.2, theta_a=2.0, sigma=sigma, dd=1.0,
                           growth_type=growth_type, mode_type=P.MODE_RT, sobel_border=P.BORDER_TORUS,
                           border=P.BORDER_TORUS, gradient_mode=P.GRADIENT_CENTRAL_DIFF, blur_central_diff=False,
                           mu_vel=False, asymptotic=(asymptotic,) * 4, soft_clip=(False,) * 4)
        ks = P.sample_kernels(rng, 3, radius=max(2, width // 4))
        out.append(P.Workload(desc, ks, P.seed_cube(rng, desc, width // 2)))
    return out


def kernel_features(kernels: Sequence[P.KernelParams]) -> np.ndarray:
    f = np.zeros((N_KERNELS, KERNEL_FEATURES), np.float64)
    for i, k in enumerate(kernels[:N_KERNELS]):
        b = (list(k.b) + [0.0, 0.0, 0.0])[:3]
        f[i] = [b[0], b[1], b[2], k.m, k.s, k.h, k.r_a]
    return f.ravel()


def _timed(fn, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0


@dataclass
class Runs:
    features: np.ndarray   # (n, 79)
    labels: np.ndarray     # (n,) strings
    hits: np.ndarray       # (n,) bool
    t_observe: float       # GPU seconds to reach the observation step (all candidates)
    t_finish: float        # GPU seconds from there to the final step (all candidates)
    states: list           # per candidate (A, V, GA, SUM) at the observation step, when kept
    init_totals: np.ndarray  # (n,) initial total mass


def simulate(wls: List[P.Workload], observe: int, final: int, keep_states: bool = False, lanes: int = 64) -> Runs:
    """All candidates to `final` in one batch, with the statistics at 0,
    observe - 1, observe and final."""
    import torch
    from .batch import Batch
    stream = torch.cuda.current_stream()
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=lanes)
    b.set_stream(stream.cuda_stream)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    W = wls[0].desc.width
    s0 = [L.summarize(s, W, W) for s in b.stats()]
    t1 = _timed(lambda: b.step(observe - 1), stream)
    sp = [L.summarize(s, W, W) for s in b.stats()]
    t2 = _timed(lambda: b.step(1), stream)
    so = [L.summarize(s, W, W) for s in b.stats()]
    states = [tuple(b.get(i, n) for n in ("A", "V", "GA", "SUM")) for i in range(len(wls))] if keep_states else []
    t3 = _timed(lambda: b.step(final - observe), stream)
    sf = [L.summarize(s, W, W) for s in b.stats()]
    b.sync()
    b.close()
    feats = np.stack([np.concatenate([kernel_features(wl.kernels), L.features(p, o, i.total, 1, W, W)])
                      for wl, p, o, i in zip(wls, sp, so, s0)])
    labs = np.array([L.label(f, i.total, W) for f, i in zip(sf, s0)])
    return Runs(feats, labs, labs == "persistent", t1 + t2, t3, states, np.array([i.total for i in s0]))


def continue_runs(wls: List[P.Workload], states, init_totals, observe: int, final: int, lanes: int = 64):
    """The selected candidates from their observation-step state to `final`
    (init_totals: each candidate's initial total mass): (labels, GPU seconds)."""
    import torch
    from .batch import Batch
    stream = torch.cuda.current_stream()
    W = wls[0].desc.width
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=lanes)
    b.set_stream(stream.cuda_stream)
    for i, (wl, st) in enumerate(zip(wls, states)):
        b.set_state(i, *st)
    t = _timed(lambda: b.step(final - observe), stream)
    sf = [L.summarize(s, W, W) for s in b.stats()]
    b.sync()
    b.close()
    return np.array([L.label(f, m0, W) for f, m0 in zip(sf, init_totals)]), t


def train(features: np.ndarray, hits: np.ndarray, epochs: int = 60, batch: int = 256, lr: float = 1e-3,
          seed: int = 0):
    """(network, feature mean, feature scale, GPU seconds) trained on the
    standardised features with class-balanced sampling."""
    import torch
    from .mlp import MLP
    mu = features.mean(axis=0)
    sd = features.std(axis=0) + 1e-6
    x = torch.from_numpy(((features - mu) / sd).astype(np.float32)).cuda()
    y = torch.from_numpy(hits.astype(np.float32)).cuda()
    net = MLP(features.shape[1], 256, seed=seed)
    g = torch.Generator(device="cuda").manual_seed(seed)
    pos = torch.nonzero(y > 0.5).flatten()
    neg = torch.nonzero(y < 0.5).flatten()
    stream = torch.cuda.current_stream()

    def run():
        n = x.shape[0]
        for _ in range(epochs):
            if len(pos) and len(neg):
                half = n // 2
                idx = torch.cat([pos[torch.randint(len(pos), (half,), device="cuda", generator=g)],
                                 neg[torch.randint(len(neg), (n - half,), device="cuda", generator=g)]])
                idx = idx[torch.randperm(n, device="cuda", generator=g)]
            else:
                idx = torch.randperm(n, device="cuda", generator=g)
            for i in range(0, n, batch):
                j = idx[i:i + batch]
                net.train_step(x[j], y[j], lr=lr, wd=1e-4, stream=stream.cuda_stream)

    t = _timed(run, stream)
    return net, mu, sd, t


def score(net, mu, sd, features: np.ndarray):
    import torch
    x = torch.from_numpy(((features - mu) / sd).astype(np.float32)).cuda()
    stream = torch.cuda.current_stream()
    out = {}
    t = _timed(lambda: out.setdefault("z", net.forward(x, stream=stream.cuda_stream)), stream)
    return out["z"].cpu().numpy(), t


def single_statistic_rule(features: np.ndarray, hits: np.ndarray):
    """The non-learned early filter: among the 16 step-50 statistics (the
    columns after the 63 kernel parameters), the one whose ranking (either
    sign) best separates the training hits, by rank AUC.  Returns (column,
    sign, training AUC)."""
    best = (N_KERNELS * KERNEL_FEATURES, 1.0, 0.5)
    if hits.all() or not hits.any():
        return best
    for col in range(N_KERNELS * KERNEL_FEATURES, features.shape[1]):
        a = ranking_auc(features[:, col], hits)
        for sign, auc in ((1.0, a), (-1.0, 1.0 - a)):
            if auc > best[2]:
                best = (col, sign, auc)
    return best


def ranking_auc(score: np.ndarray, hits: np.ndarray):
    """Probability that a random hit scores above a random non-hit (ties
    count half); None without both classes."""
    if hits.all() or not hits.any():
        return None
    order = np.argsort(score, kind="stable")
    ranks = np.empty(len(score))
    ranks[order] = np.arange(len(score))
    # average ranks of ties
    s_sorted = score[order]
    i = 0
    while i < len(s_sorted):
        j = i
        while j + 1 < len(s_sorted) and s_sorted[j + 1] == s_sorted[i]:
            j += 1
        if j > i:
            ranks[order[i:j + 1]] = (i + j) / 2.0
        i = j + 1
    npos, nneg = int(hits.sum()), int((~hits).sum())
    return float((ranks[hits].sum() - npos * (npos - 1) / 2.0) / (npos * nneg))


def study(n_train: int = 4096, n_test: int = 2048, width: int = 32, observe: int = 50, final: int = 400,
          keep: float = 0.2, seed: int = 17) -> Dict:
    """The whole comparison; returns its numbers (GPU seconds, hits, rates).

    Four arms on the same test candidates, each timed on the GPU: uniform
    (every candidate to the final step) and three early filters that run
    every candidate to the observation step and continue the same number of
    them, `keep` of the test set, from their saved states: the network's top
    scores (learned), a uniform random choice (random), and the top of the
    single step-50 statistic that best separates the training hits
    (statistic).  Every continued run is the plain simulation of its
    candidate; a hit of a filtered arm counts only when that run ends
    persistent."""
    t0 = time.time()
    tr = simulate(candidates(n_train, seed, width), observe, final)
    net, mu, sd, t_train = train(tr.features, tr.hits, seed=seed)
    test_wls = candidates(n_test, seed + 1, width)
    te = simulate(test_wls, observe, final, keep_states=True)
    z, t_score = score(net, mu, sd, te.features)
    k = max(1, int(round(keep * n_test)))
    col, sign, stat_auc_train = single_statistic_rule(tr.features, tr.hits)
    rng = np.random.default_rng(seed + 2)
    picks = {
        "learned": np.argsort(-z, kind="stable")[:k],
        "random": np.sort(rng.choice(n_test, size=k, replace=False)),
        "statistic": np.argsort(-sign * te.features[:, col], kind="stable")[:k],
    }
    t_uniform = te.t_observe + te.t_finish
    hits_u = int(te.hits.sum())
    rate_u = hits_u / t_uniform
    arms = {"uniform": {"hits": hits_u, "gpu_s": t_uniform, "hits_per_gpu_hour": 3600 * rate_u}}
    agree = True
    for name, chosen in picks.items():
        labels_cont, t_cont = continue_runs([test_wls[i] for i in chosen], [te.states[i] for i in chosen],
                                            te.init_totals[chosen], observe, final)
        # the continued runs are the plain simulation of each chosen candidate
        confirmed = labels_cont == "persistent"
        agree = agree and bool(np.all(labels_cont == te.labels[chosen]))
        t_arm = te.t_observe + t_cont + (t_score if name == "learned" else 0.0)
        h = int(confirmed.sum())
        arms[name] = {"hits": h, "gpu_s": t_arm, "hits_per_gpu_hour": 3600 * h / t_arm,
                      "ratio_to_uniform": (h / t_arm) / rate_u if rate_u > 0 else None}
    # the learned arm charged with its training: the label simulation and the
    # network's training, spread over this one test set
    t_learn_all = arms["learned"]["gpu_s"] + tr.t_observe + tr.t_finish + t_train
    arms["learned"]["hits_per_gpu_hour_with_training"] = 3600 * arms["learned"]["hits"] / t_learn_all
    return {
        "candidates": {"train": n_train, "test": n_test, "width": width, "observe": observe, "final": final,
                       "keep_fraction": keep},
        "train_hit_rate": float(tr.hits.mean()), "test_hit_rate": float(te.hits.mean()),
        "gpu_s": {"train_simulation": tr.t_observe + tr.t_finish, "train_network": t_train,
                  "uniform": t_uniform, "learned": arms["learned"]["gpu_s"], "score": t_score},
        "hits": {"uniform": hits_u, "learned": arms["learned"]["hits"],
                 "learned_confirmed_equal_uniform_labels": agree},
        "hits_per_gpu_hour": {"uniform": arms["uniform"]["hits_per_gpu_hour"],
                              "learned": arms["learned"]["hits_per_gpu_hour"],
                              "ratio": arms["learned"]["ratio_to_uniform"]},
        "arms": arms,
        "statistic_rule": {"column": int(col), "statistic": int(col - N_KERNELS * KERNEL_FEATURES),
                           "sign": sign, "train_auc": stat_auc_train,
                           "test_auc": ranking_auc(sign * te.features[:, col], te.hits)},
        "ranking_auc": ranking_auc(z, te.hits),
        "wall_s": time.time() - t0,
    }


if __name__ == "__main__":
    import json
    import sys
    args = dict(a.split("=") for a in sys.argv[1:])
    res = study(**{k: (float(v) if k == "keep" else int(v)) for k, v in args.items()})
    print(json.dumps(res))
