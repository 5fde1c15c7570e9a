"""Grid statistics (GPU, FP64, deterministic) and the labels built on them."""
from __future__ import annotations

import numpy as np
import pytest

from lenia_b200 import labels as L
from lenia_b200 import params as P


def np_stats(A: np.ndarray, fill: float = 0.1) -> np.ndarray:
    """The statistics of lenia_world_stats, in numpy float64."""
    A = np.asarray(A, dtype=np.float32)
    C, D, H, W = A.shape
    a = A.astype(np.float64)
    tx = 2 * np.pi * np.arange(W) / W
    ty = 2 * np.pi * np.arange(H) / H
    tz = 2 * np.pi * np.arange(D) / W
    out = np.zeros((C, 9))
    for c in range(C):
        m = a[c]
        out[c, 0] = m.sum()
        out[c, 1] = (m * np.cos(tx)[None, None, :]).sum()
        out[c, 2] = (m * np.sin(tx)[None, None, :]).sum()
        out[c, 3] = (m * np.cos(ty)[None, :, None]).sum()
        out[c, 4] = (m * np.sin(ty)[None, :, None]).sum()
        out[c, 5] = (m * np.cos(tz)[:, None, None]).sum()
        out[c, 6] = (m * np.sin(tz)[:, None, None]).sum()
        out[c, 7] = max(m.max(), 0.0)
        out[c, 8] = float((A[c] > np.float32(fill)).sum())
    return out


def blob(W, centre, sigma=2.0, C=3):
    z, y, x = np.meshgrid(np.arange(W), np.arange(W), np.arange(W), indexing="ij")
    d = [(np.arange(W)[None, None, :] * 0 + g) for g in (x, y, z)]
    r2 = 0.0
    for g, c0 in zip((x, y, z), centre):
        dd = (g - c0 + W / 2) % W - W / 2   # torus distance
        r2 = r2 + dd ** 2
    f = np.exp(-r2 / (2 * sigma ** 2)).astype(np.float32)
    del d
    return np.repeat(f[None], C, axis=0)


def test_centroid_and_spread_of_a_blob():
    W = 32
    for centre in ((5.0, 20.0, 11.0), (0.0, 31.0, 16.0)):   # the second straddles the boundary
        s = L.summarize(np_stats(blob(W, centre)), W, W)
        d = L.torus_delta(np.array(centre), s.centroid[-1], (W, W, W))
        assert np.abs(d).max() < 1e-6, (centre, s.centroid[-1])
        assert 2.5 < s.spread[-1] < 5.0       # sqrt(3) * 2 for sigma 2
        assert np.allclose(s.ratios, 1 / 3)


def test_labels_of_simple_fields():
    W = 24
    init = L.summarize(np_stats(blob(W, (12, 12, 12))), W, W)
    alive = L.summarize(np_stats(blob(W, (3, 12, 20))), W, W)
    assert L.label(alive, init.total, W) == "persistent"
    dead = L.summarize(np_stats(0.001 * blob(W, (3, 12, 20))), W, W)
    assert L.label(dead, init.total, W) == "dead"
    full = L.summarize(np_stats(np.full((3, W, W, W), 0.8, np.float32)), W, W)
    assert L.label(full, init.total, W) == "exploding"
    nan = np_stats(blob(W, (3, 3, 3)))
    nan[0, 0] = np.nan
    assert L.label(L.summarize(nan, W, W), init.total, W) == "exploding"


def test_feature_vector_and_velocity():
    W = 32
    s0 = L.summarize(np_stats(blob(W, (30.0, 8.0, 8.0))), W, W)
    s1 = L.summarize(np_stats(blob(W, (1.0, 8.0, 8.0))), W, W)   # moved +3 across the boundary
    sp = L.centroid_speed(s0, s1, 3, W, W)
    assert np.allclose(sp, 1.0, atol=1e-6)
    f = L.features(s0, s1, s0.total, 3, W, W)
    assert f.shape == (16,) and np.all(np.isfinite(f))


@pytest.mark.gpu
def test_gpu_stats_match_numpy_and_repeat():
    from lenia_b200.world import World
    wl = P.config0(seed=3)
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    w.step(4)
    A = w.get("A").reshape(wl.A0.shape)
    g1, g2 = w.stats(0.1), w.stats(0.1)
    assert np.array_equal(g1.view(np.uint64), g2.view(np.uint64))   # fixed summation order
    ref = np_stats(A, 0.1)
    assert np.array_equal(g1[:, 7], ref[:, 7]) and np.array_equal(g1[:, 8], ref[:, 8])
    scale = np.abs(ref[:, :1]) + 1e-30
    assert np.all(np.abs(g1[:, :7] - ref[:, :7]) <= 1e-12 * scale)
    w.close()


@pytest.mark.gpu
def test_batch_stats_and_labels():
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wls = P.config3(5, seed=21, sizes=(24, 32))
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=2)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    b.step(3)
    bs = b.stats()
    for i, wl in enumerate(wls):
        w = World(wl.desc, wl.kernels)
        w.set_state(wl.A0.ravel())
        w.step(3)
        assert np.array_equal(bs[i].view(np.uint64), w.stats().view(np.uint64)), i
        w.close()
    b.close()
    res = L.run_labels(wls, steps=12, observe=6, lanes=2)
    assert res["features"].shape == (5, 16) and np.all(np.isfinite(res["features"]))
    assert set(res["labels"]) <= set(L.LABELS)
