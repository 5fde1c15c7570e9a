"""The proposal network: forward and gradients against a numpy float64
restatement with the same bfloat16 rounding of every tensor-core operand
(activations, weights, and dz in the backward products), and training."""
import numpy as np
import pytest
from scipy.special import erf

pytestmark = pytest.mark.gpu

DIMS = [79, 256, 256, 256, 1]


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), as the kernels stage them."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    finite = (u & 0x7F800000) != 0x7F800000
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return np.where(finite, r, u).astype(np.uint32).view(np.float32)


def np_forward_backward(p, x, y):
    from lenia_b200.mlp import split_params
    layers = split_params(p, DIMS)
    acts, zs = [x.astype(np.float32)], []
    for i, (W, b) in enumerate(layers):
        z = bf16(acts[-1]).astype(np.float64) @ bf16(W).astype(np.float64).T + b
        zs.append(z)
        if i + 1 < len(layers):
            acts.append((0.5 * z * (1 + erf(z / np.sqrt(2)))).astype(np.float32))
    zl = zs[-1][:, 0]
    loss = np.mean(np.log1p(np.exp(-np.abs(zl))) + np.maximum(zl, 0) - zl * y)
    dz = ((1 / (1 + np.exp(-zl)) - y) / len(y))[:, None]
    grads = []
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        # dz enters both products rounded to bfloat16 (the tensor cores take
        # bfloat16 operands); the bias gradient sums it in float
        dzb = bf16(dz.astype(np.float32)).astype(np.float64)
        gW = dzb.T @ bf16(acts[i]).astype(np.float64)
        gb = dz.sum(axis=0)
        grads.append((gW, gb))
        if i > 0:
            da = dzb @ bf16(W).astype(np.float64)
            z = zs[i - 1]
            gp = 0.5 * (1 + erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)
            dz = da * gp
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return zs[-1][:, 0], loss, flat


def test_parameter_count_matches_the_specification():
    from lenia_b200.mlp import MLP
    m = MLP(79, 256, seed=1)
    assert m.n_params == 152321
    m.close()


def test_forward_and_gradients_match_float64_restatement():
    import torch
    from lenia_b200.mlp import MLP
    rng = np.random.default_rng(0)
    B = 300
    x = rng.normal(size=(B, 79)).astype(np.float32)
    y = (rng.uniform(size=B) < 0.3).astype(np.float32)
    m = MLP(79, 256, seed=3)
    p = m.params()
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    logits = m.forward(xt).cpu().numpy()
    loss = m.gradients(xt, yt)
    g = m.grads()
    zl, loss_ref, g_ref = np_forward_backward(p, x, y)
    # float32 accumulation vs float64; a value that lands on the other side of
    # a bfloat16 rounding boundary (GPU erff vs numpy) moves one operand by
    # 2^-8 relative, so single outliers of ~1e-3 are expected.  A wrong
    # formula would give errors of order one.
    err = np.abs(logits - zl)
    assert np.median(err) <= 1e-6 and err.max() <= 1e-2 * (1 + np.max(np.abs(zl)))
    assert abs(loss - loss_ref) <= 1e-3 * (1 + abs(loss_ref))
    assert np.linalg.norm(g - g_ref) <= 1e-2 * np.linalg.norm(g_ref)
    cos = float(g @ g_ref / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    assert cos > 0.9999, cos
    m.close()


def test_training_learns_a_separable_rule():
    import torch
    from lenia_b200.mlp import MLP
    rng = np.random.default_rng(1)
    x = rng.normal(size=(4096, 79)).astype(np.float32)
    y = ((x[:, 0] + 0.5 * x[:, 5] - x[:, 40]) > 0.3).astype(np.float32)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    m = MLP(79, 256, seed=2)
    first = m.gradients(xt, yt)
    for epoch in range(30):
        perm = torch.randperm(4096, device="cuda")
        for i in range(0, 4096, 512):
            idx = perm[i:i + 512]
            m.train_step(xt[idx], yt[idx], lr=1e-3)
    last = m.gradients(xt, yt)
    acc = ((m.forward(xt) > 0).float() == yt).float().mean().item()
    assert last < 0.3 * first and acc > 0.95, (first, last, acc)
    m.close()


def test_proposal_study_runs_end_to_end():
    """A small study: both arms timed, every learned hit re-simulated from its
    saved state with the same label as in the uniform run."""
    from lenia_b200.proposals import study
    res = study(n_train=96, n_test=64, width=24, observe=10, final=40, keep=0.25, seed=5)
    assert res["hits"]["learned_confirmed_equal_uniform_labels"]
    assert res["gpu_s"]["learned"] < res["gpu_s"]["uniform"]
    assert 0.0 <= res["test_hit_rate"] <= 1.0
    # the two non-learned early filters continue as many candidates
    for arm in ("random", "statistic"):
        assert arm in res["arms"] and res["arms"][arm]["gpu_s"] < res["gpu_s"]["uniform"]
