"""Parameter set of the 3D Flow Lenia step and the seeded workload generators.

The fields mirror the reference's mutable globals and structs:
scalars and mode enums (main.cpp:27-56, main.cpp:304 for sigma/dd), the
per-channel flags (render.h:486-492) and the per-kernel parameters
(render.h:347-361).  Defaults are the reference's defaults.

`WorldDesc` and `KernelParams` map one-to-one onto the C-ABI structs
`LeniaWorldDesc` and `LeniaKernelParams` declared in include/lenia_b200.h.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

# Enums (render.h:128-223); values are the reference's enumerator order.
ALPHA_GRID, ALPHA_GRID_GROWTH, ALPHA_GA, ALPHA_GA_DIFF = range(4)
GROWTH_NOGROWTH, GROWTH_RT, GROWTH_TRANSPOSITION = range(3)
MODE_SRT, MODE_RT, MODE_ADV = range(3)
BORDER_TORUS, BORDER_WALL, BORDER_NONE = range(3)
GRADIENT_CENTRAL_DIFF, GRADIENT_SOBEL = range(2)

MAX_CHANNELS = 4
MAX_BETA = 12
MAX_KERNELS = 64


@dataclass
class WorldDesc:
    """Grid shape, scalars and modes of one world (reference defaults)."""

    width: int = 32           # x and z extent (GRID_WIDTH, render.h:27)
    height: int = 32          # y extent (GRID_HEIGHT, render.h:28)
    channels: int = 3
    timestep: float = 0.1
    theta_a: float = 1.0
    n_alpha: float = 2.0      # N: unused by the reference (Q3)
    s_norm: float = 0.0
    gta: float = 0.1
    sta: float = 0.1
    v_damp: float = 0.9
    v_beta: float = 0.9       # unused by the reference
    iso_value: float = 0.5
    sigma: float = 0.5        # off_table.sigma
    dd: float = 1.0           # off_table.dd (used as int)
    alpha_mode: int = ALPHA_GRID
    growth_type: int = GROWTH_RT
    mode_type: int = MODE_SRT
    sobel_border: int = BORDER_NONE
    border: int = BORDER_NONE
    gradient_mode: int = GRADIENT_SOBEL
    adv_vel: bool = True
    mu_vel: bool = False
    blur_central_diff: bool = False
    osc_la: bool = False
    osc_flow: bool = False
    osc_div_flow: bool = False
    osc_vel: bool = False
    osc_la_amt: float = -0.001
    osc_flow_amt: float = -0.001
    osc_div_flow_amt: float = -0.001
    asymptotic: Sequence[bool] = (False, True, True, False)   # render.cpp:803-811
    soft_clip: Sequence[bool] = (False, False, False, False)
    rt_all_channels: bool = False  # False: SRT/RT move channels 0-2 only (Q7)
    alpha_index_fix: bool = False  # False: PREALPHA/GA channel offsets as the reference (Q20)
    exact_bell: bool = False       # False: growth from the reference's 256^3 table (Q1); True: bell(u, m, s)
    conserve_mass: bool = False    # True: each channel's total restored after every step (FP64 sums on the GPU)

    @property
    def depth(self) -> int:
        return self.width

    @property
    def cells(self) -> int:
        return self.width * self.height * self.width

    def as_dict(self) -> dict:
        d = dataclasses.asdict(self)
        d["asymptotic"] = [int(bool(x)) for x in (list(self.asymptotic) + [0] * 4)[:4]]
        d["soft_clip"] = [int(bool(x)) for x in (list(self.soft_clip) + [0] * 4)[:4]]
        return d


@dataclass
class KernelParams:
    """One convolution kernel (render.h:347-361)."""

    radius: int = 4
    beta_size: int = 1
    b: Sequence[float] = field(default_factory=lambda: [1.0])
    r_a: float = 1.0
    m: float = 0.3
    s: float = 0.15
    h: float = 1.0
    c0: int = 0   # source channel
    c1: int = 0   # destination channel

    def as_dict(self) -> dict:
        d = dataclasses.asdict(self)
        d["b"] = [float(x) for x in (list(self.b) + [0.0] * MAX_BETA)[:MAX_BETA]]
        return d


def _f32(x: float) -> float:
    return float(np.float32(x))


def sample_kernels(rng: np.random.Generator, channels: int, radius: int,
                   pairs: Sequence[tuple] | None = None) -> List[KernelParams]:
    """Kernel sets as the benchmark configurations draw them: one kernel per
    (source, destination) channel pair, 1-3 bell shells, b ~ U(0,1),
    m ~ U(0.1,0.5), s ~ U(0.01,0.18), h ~ U(0.01,1), r_a = 1."""
    if pairs is None:
        pairs = [(c0, c1) for c0 in range(channels) for c1 in range(channels)]
    ks = []
    for (c0, c1) in pairs:
        beta = int(rng.integers(1, 4))
        ks.append(KernelParams(
            radius=radius, beta_size=beta,
            b=[_f32(rng.uniform(0.0, 1.0)) for _ in range(beta)],
            r_a=1.0,
            m=_f32(rng.uniform(0.1, 0.5)),
            s=_f32(rng.uniform(0.01, 0.18)),
            h=_f32(rng.uniform(0.01, 1.0)),
            c0=c0, c1=c1))
    return ks


def seed_cube(rng: np.random.Generator, desc: WorldDesc, side: int) -> np.ndarray:
    """A ~ U(0,1) in the centred side^3 cube, zero elsewhere; shape (C, D, H, W)."""
    W, H, D, C = desc.width, desc.height, desc.depth, desc.channels
    A = np.zeros((C, D, H, W), dtype=np.float32)
    sx = min(side, W)
    sy = min(side, H)
    x0, y0 = (W - sx) // 2, (H - sy) // 2
    A[:, x0:x0 + sx, y0:y0 + sy, x0:x0 + sx] = rng.uniform(0.0, 1.0, size=(C, sx, sy, sx)).astype(np.float32)
    return A


@dataclass
class Workload:
    desc: WorldDesc
    kernels: List[KernelParams]
    A0: np.ndarray  # (C, D, H, W) float32


def config0(seed: int = 0, width: int = 32) -> Workload:
    """Plain step, 32^3, 3 channels, 9 kernels of radius 8, central differences,
    periodic borders, RT with sigma=0.65, dt=0.2, theta_A=2; seeded U(0,1) in
    the centred 16^3 cube."""
    rng = np.random.default_rng(seed)
    desc = WorldDesc(width=width, height=width, channels=3, timestep=0.2, theta_a=2.0,
                     sigma=0.65, dd=1.0, growth_type=GROWTH_RT, mode_type=MODE_RT,
                     sobel_border=BORDER_TORUS, border=BORDER_TORUS,
                     gradient_mode=GRADIENT_CENTRAL_DIFF, blur_central_diff=False,
                     mu_vel=False, asymptotic=(False,) * 4, soft_clip=(False,) * 4)
    ks = sample_kernels(rng, 3, radius=8)
    A0 = seed_cube(rng, desc, width // 2)
    return Workload(desc, ks, A0)


def config1(seed: int = 1, width: int = 128, mode: int = MODE_RT, radius: int = 13,
            gradient: int = GRADIENT_SOBEL) -> Workload:
    """Single world at 128^3, 4 channels, 16 kernels of radius 13, zero
    borders, Sobel gradients, RT (or advection) reintegration; the seed cube
    has half the grid's side."""
    rng = np.random.default_rng(seed)
    desc = WorldDesc(width=width, height=width, channels=4, timestep=0.2, theta_a=2.0,
                     sigma=0.65, dd=1.0, growth_type=GROWTH_RT, mode_type=mode,
                     sobel_border=BORDER_NONE, border=BORDER_NONE,
                     gradient_mode=gradient, blur_central_diff=(gradient == GRADIENT_CENTRAL_DIFF),
                     mu_vel=False, adv_vel=True, asymptotic=(False,) * 4, soft_clip=(False,) * 4)
    ks = sample_kernels(rng, 4, radius=radius)
    A0 = seed_cube(rng, desc, width // 2)
    return Workload(desc, ks, A0)


def config2(seed: int = 2, width: int = 256, radius: int = 20) -> Workload:
    """Precision workload: a width^3 grid with the plain step's modes
    (3 channels, 9 kernels drawn as in config 0 but of the given radius,
    central differences, RT with sigma 0.65, periodic borders) from the plain
    step's seeded U(0,1) cube scaled to half the side."""
    rng = np.random.default_rng(seed)
    desc = WorldDesc(width=width, height=width, channels=3, timestep=0.2, theta_a=2.0,
                     sigma=0.65, dd=1.0, growth_type=GROWTH_RT, mode_type=MODE_RT,
                     sobel_border=BORDER_TORUS, border=BORDER_TORUS,
                     gradient_mode=GRADIENT_CENTRAL_DIFF, blur_central_diff=False,
                     mu_vel=False, asymptotic=(False,) * 4, soft_clip=(False,) * 4)
    ks = sample_kernels(rng, 3, radius=radius)
    A0 = seed_cube(rng, desc, width // 2)
    return Workload(desc, ks, A0)


CONFIG3_SIZES = (24, 32, 36, 44, 48, 64, 96)


def config3(n_worlds: int = 4096, seed: int = 3, sizes: Sequence[int] = CONFIG3_SIZES) -> List[Workload]:
    """Batched worlds: per world a side drawn uniformly from `sizes` (cubic),
    3 channels, 9 kernels (one per channel pair) of radius side / 4 drawn as
    in config 0, central differences with periodic borders, RT or advection
    reintegration by a fair coin, and its own seeded U(0,1) cube of half the
    side.  World i draws from default_rng((seed, i))."""
    out = []
    for i in range(n_worlds):
        rng = np.random.default_rng((seed, i))
        w = int(sizes[int(rng.integers(0, len(sizes)))])
        mode = MODE_RT if rng.integers(0, 2) == 0 else MODE_ADV
        desc = WorldDesc(width=w, height=w, channels=3, timestep=0.2, theta_a=2.0,
                         sigma=0.65, dd=1.0, growth_type=GROWTH_RT, mode_type=mode,
                         sobel_border=BORDER_TORUS, border=BORDER_TORUS,
                         gradient_mode=GRADIENT_CENTRAL_DIFF, blur_central_diff=False,
                         mu_vel=False, adv_vel=True, asymptotic=(False,) * 4, soft_clip=(False,) * 4)
        ks = sample_kernels(rng, 3, radius=max(2, w // 4))
        out.append(Workload(desc, ks, seed_cube(rng, desc, w // 2)))
    return out
