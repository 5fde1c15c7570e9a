"""Random kernel sets and seeds as the reference draws them.

`generate_random` restates generate_random (lenia.cpp:370-429) and
seed_grid_gaussian (lenia.cpp:305-334): a neighbourhood of 1-8 cells, 1-10
kernels of that radius with 1-2 shells, b = (rand() % 100) / 100,
m = (100 + rand() % 500) / 1000, s = m / 10 + (rand() % 200) / 1000, h = r_a =
1, the first kernel 0 -> 0 and the others between random channels, then five
Gaussian blobs exp(-d^2 / (2 r^2)) added to every channel.  The random
numbers come from `MsvcRand`, the rand() of the reference's platform, so a
seed gives the reference's own draw.  This is the uniform-sampling baseline of
the persistent-pattern search.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .params import KernelParams


class MsvcRand:
    """rand()/srand() of the MSVC C runtime: x = 214013 x + 2531011 mod 2^32,
    returning bits 16..30 (0..32767)."""

    def __init__(self, seed: int = 1):
        self.state = seed & 0xFFFFFFFF

    def rand(self) -> int:
        self.state = (self.state * 214013 + 2531011) & 0xFFFFFFFF
        return (self.state >> 16) & 0x7FFF


def _f32(x) -> np.float32:
    return np.float32(x)


def seed_grid_gaussian(r: MsvcRand, channels: int, width: int, height: int, radius: int) -> np.ndarray:
    """Five blobs at random centres, exp(-d^2 / (2 radius^2)) summed in float
    into every channel (lenia.cpp:305-334); shape (C, D, H, W), D = W."""
    W, H, D = width, height, width
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    grid = np.zeros((D, H, W), dtype=np.float32)
    den = np.float32(2 * radius * radius)
    for _ in range(5):
        cx = r.rand() % W
        cy = r.rand() % H
        cz = r.rand() % W
        dist = ((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2).astype(np.float32)
        arg = (-dist) / den                                  # float division
        # exp of a float argument rounded to float (the reference calls the C
        # runtime's expf, which may differ from the rounded value by an ulp)
        v = np.exp(arg.astype(np.float64)).astype(np.float32)
        grid = (grid + v).astype(np.float32)
    return np.repeat(grid[None], channels, axis=0)


def generate_random(r: MsvcRand, channels: int, width: int, height: int
                    ) -> Tuple[List[KernelParams], np.ndarray, int]:
    """(kernels, seeded grid (C, D, H, W), neighbourhood) of one draw."""
    neighborhood = 1 + r.rand() % 8
    kernel_count = r.rand() % 10 + 1
    ks = []
    for i in range(kernel_count):
        beta = r.rand() % 2 + 1
        b = [float(_f32(r.rand() % 100) / _f32(100)) for _ in range(beta)]
        m = _f32(100 + r.rand() % 500) / _f32(1000)
        s = _f32(m / _f32(10)) + _f32(_f32(r.rand() % 200) / _f32(1000))
        if channels == 1 or i == 0:
            c0 = c1 = 0
        else:
            c0 = r.rand() % channels
            c1 = r.rand() % channels
        ks.append(KernelParams(radius=neighborhood, beta_size=beta, b=b, r_a=1.0, m=float(m), s=float(_f32(s)),
                               h=1.0, c0=c0, c1=c1))
    A0 = seed_grid_gaussian(r, channels, width, height, neighborhood)
    return ks, A0, neighborhood
