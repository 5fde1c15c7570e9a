"""Test cases shared by the oracle and GPU parity tests: seeded workloads and
the mode variants the reference supports."""
from __future__ import annotations

import copy

import numpy as np

from lenia_b200 import params as P

# name -> WorldDesc overrides on top of the 32^3 plain-step configuration
VARIANTS = {
    "cfg0": {},
    "sobel_torus": dict(gradient_mode=P.GRADIENT_SOBEL, sobel_border=P.BORDER_TORUS),
    "sobel_wall": dict(gradient_mode=P.GRADIENT_SOBEL, sobel_border=P.BORDER_WALL, border=P.BORDER_WALL),
    "sobel_none": dict(gradient_mode=P.GRADIENT_SOBEL, sobel_border=P.BORDER_NONE, border=P.BORDER_NONE),
    "cd_wall": dict(sobel_border=P.BORDER_WALL, border=P.BORDER_WALL),
    "cd_none": dict(sobel_border=P.BORDER_NONE, border=P.BORDER_NONE),
    "cd_blur_torus": dict(blur_central_diff=True),
    "cd_blur_none": dict(blur_central_diff=True, sobel_border=P.BORDER_NONE, border=P.BORDER_NONE),
    "srt": dict(mode_type=P.MODE_SRT),
    "adv_vel": dict(mode_type=P.MODE_ADV, adv_vel=True),
    "adv_f": dict(mode_type=P.MODE_ADV, adv_vel=False),
    "mu_vel": dict(mu_vel=True),
    "mu_vel_wall": dict(mu_vel=True, border=P.BORDER_WALL),
    "nogrowth": dict(growth_type=P.GROWTH_NOGROWTH),
    "transposition": dict(growth_type=P.GROWTH_TRANSPOSITION),
    "transposition_softclip": dict(growth_type=P.GROWTH_TRANSPOSITION, soft_clip=(True, False, True, False)),
    "rt_softclip_asym": dict(soft_clip=(True, False, True, False), asymptotic=(False, True, True, False)),
    "dd2_sigma09": dict(dd=2.0, sigma=0.9),
    "snorm": dict(s_norm=0.5),
    "osc_la_flow": dict(osc_la=True, osc_flow=True),
    "osc_flow_vel": dict(osc_flow=True, osc_vel=True),
}


# name -> overrides of this library's clean-mode options (no counterpart in
# the reference: pinned GPU against the C restatement only)
CLEAN_VARIANTS = {
    "exact_bell": dict(exact_bell=True),
    "exact_bell_asym_softclip": dict(exact_bell=True, soft_clip=(True, False, True, False),
                                     asymptotic=(False, True, True, False)),
}


def variant(name: str, seed: int = 3, width: int = 32) -> P.Workload:
    wl = P.config0(seed=seed, width=width)
    for k, v in {**VARIANTS, **CLEAN_VARIANTS}[name].items():
        setattr(wl.desc, k, v)
    return wl


def two_channel_div_flow(seed: int = 5) -> P.Workload:
    """OSC_DIV_FLOW with two channels (three would read GA past its end in the
    reference's 32^3 build)."""
    wl = P.config0(seed=seed)
    wl.desc.channels = 2
    wl.kernels = [k for k in wl.kernels if k.c0 < 2 and k.c1 < 2]
    wl.A0 = wl.A0[:2].copy()
    wl.desc.osc_div_flow = True
    wl.desc.osc_div_flow_amt = -0.01
    return wl


def four_channels(seed: int = 7, width: int = 32, n_kernels: int = 12, radius: int = 6) -> P.Workload:
    rng = np.random.default_rng(seed)
    wl = P.config0(seed=seed, width=width)
    wl.desc.channels = 4
    wl.kernels = P.sample_kernels(rng, 4, radius=radius)[:n_kernels]
    wl.A0 = P.seed_cube(rng, wl.desc, width // 2)
    return wl


def as_oracle(wl: P.Workload):
    return wl.desc.as_dict(), [k.as_dict() for k in wl.kernels]


def diff_report(name: str, a: np.ndarray, b: np.ndarray) -> str:
    a = np.asarray(a, np.float32).ravel()
    b = np.asarray(b, np.float32).ravel()
    if a.shape != b.shape:
        return f"{name}: shape {a.shape} vs {b.shape}"
    eq = (a == b) | (np.isnan(a) & np.isnan(b))
    if eq.all():
        return ""
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    i = int(np.argmax(~eq))
    return (f"{name}: {int((~eq).sum())} of {a.size} differ, max |diff| {np.nanmax(d):.3e}, "
            f"first at {i}: {a[i]!r} vs {b[i]!r}")
