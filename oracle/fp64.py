"""Float64 restatement of the 3D Flow Lenia step: the oracle of the precision
study.  Test infrastructure only; the product never imports it.

It runs every operation of the reference step in double precision, on numpy
arrays or on float64 torch tensors (any device) through a small array shim.
What stays as in the reference is what defines the algorithm rather than its
rounding: the kernel support and shell index (float predicates of
init_kernel), the growth table's truncating index into a 256^3 grid of bell
values (lenia.h:79-84, lenia.cpp:93-101), PREALPHA's channel offsets (Q20),
and halo reads that return zero for cells outside the grid on two or more
axes (transpose_borders fills faces only).

Scope: the modes of the plain-step configurations: growth by RT into BACK,
RT reintegration with dd = 1, central-difference gradients without blur,
torus borders, no oscillators, mu from F.  Other modes raise
NotImplementedError.

Reference call sites restated (file:line):
  init_kernel             lenia.cpp:199-257
  fft_step / mt_fft_step  lenia.cpp:435-538, early growth 542-592
  h_central_diff          reintegration.cpp:260-315
  sobel_convolve(_h)      lenia.cpp:597-676 (PREALPHA, Q20)
  compute_f               lenia.cpp:679-719
  compute_f_mu            reintegration.cpp:321-602
  rt_border_torus         reintegration.cpp:607-1410 (RT branch)
  transpose_to_row_major  lenia.cpp:924-1044
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


class Xp:
    """numpy or torch (float64) behind one small interface."""

    def __init__(self, device=None):
        self.torch = None
        self.device = device
        if device is not None:
            import torch
            self.torch = torch

    def asarray(self, a):
        a = np.asarray(a, dtype=np.float64)
        if self.torch is None:
            return a.copy()
        return self.torch.as_tensor(a, dtype=self.torch.float64, device=self.device)

    def zeros(self, shape):
        if self.torch is None:
            return np.zeros(shape, np.float64)
        return self.torch.zeros(shape, dtype=self.torch.float64, device=self.device)

    def roll(self, a, shift, axis):
        if self.torch is None:
            return np.roll(a, shift, axis)
        return self.torch.roll(a, shift, axis)

    def rfftn(self, a):
        if self.torch is None:
            return np.fft.rfftn(a, axes=(-3, -2, -1))
        return self.torch.fft.rfftn(a, dim=(-3, -2, -1))

    def irfftn(self, a, shape):
        if self.torch is None:
            return np.fft.irfftn(a, s=shape, axes=(-3, -2, -1))
        return self.torch.fft.irfftn(a, s=shape, dim=(-3, -2, -1))

    def clip(self, a, lo, hi):
        if self.torch is None:
            return np.clip(a, lo, hi)
        return self.torch.clamp(a, lo, hi)

    def minimum(self, a, b):
        return np.minimum(a, b) if self.torch is None else self.torch.minimum(a, self._t(b, a))

    def maximum(self, a, b):
        return np.maximum(a, b) if self.torch is None else self.torch.maximum(a, self._t(b, a))

    def _t(self, b, like):
        if isinstance(b, (int, float)):
            return self.torch.full_like(like, float(b))
        return b

    def where(self, m, a, b):
        if self.torch is None:
            return np.where(m, a, b)
        return self.torch.where(m, a, self._t(b, a) if isinstance(b, (int, float)) else b)

    def exp(self, a):
        return np.exp(a) if self.torch is None else self.torch.exp(a)

    def trunc_int(self, a):
        if self.torch is None:
            return np.trunc(a).astype(np.int64)
        return self.torch.trunc(a).to(self.torch.int64)

    def f64(self, a):
        return a.astype(np.float64) if self.torch is None else a.to(self.torch.float64)

    def numpy(self, a):
        return a if self.torch is None else a.detach().cpu().numpy()

    def bool1d(self, a):
        a = np.asarray(a, dtype=bool)
        return a if self.torch is None else self.torch.as_tensor(a, device=self.device)


def _f32(x):
    return np.float32(x)


def kernel_grid64(desc, kp) -> np.ndarray:
    """init_kernel in double: support and shell index from the reference's
    float predicate, cell values b[i] * bell(frac(dist), 0.5, 0.15) in double,
    normalised by their double sum.  Shape (D, H, W), offsets wrapped."""
    W, H, D = desc.width, desc.height, desc.width
    rx = np.arange(-(W // 2), W - W // 2)
    ry = np.arange(-(H // 2), H - H // 2)
    rz = np.arange(-(D // 2), D - D // 2)
    z, y, x = np.meshgrid(rz, ry, rx, indexing="ij")
    fx, fy, fz = (np.abs(v).astype(np.float32) for v in (x, y, z))
    d32 = np.sqrt(fx * fx + fy * fy + fz * fz, dtype=np.float32)
    d32 = d32 / _f32(kp.radius) * _f32(kp.beta_size) / _f32(kp.r_a)
    inside = d32 < _f32(kp.beta_size)
    index = np.minimum(np.floor(d32).astype(np.int64), kp.beta_size - 1)
    d64 = np.sqrt(x.astype(np.float64) ** 2 + y ** 2 + z ** 2) / kp.radius * kp.beta_size / float(_f32(kp.r_a))
    frac = np.fmod(d64, 1.0)
    b = np.array([float(_f32(v)) for v in list(kp.b)[:kp.beta_size]], np.float64)
    val = np.where(inside, b[np.clip(index, 0, kp.beta_size - 1)] * np.exp(-((frac - 0.5) / 0.15) ** 2 / 2), 0.0)
    val = val / val.sum()
    out = np.zeros((D, H, W), np.float64)
    out[z % D, y % H, x % W] = val
    return out


@dataclass
class State:
    A: object     # (C, D, H, W)
    V: object     # (3, C, D, H, W)
    GA: object    # (C, D, H, W)
    SUM: object   # (D, H, W)


class Fp64Step:
    """One world of the float64 oracle.  After step(): .U (K, D, H, W),
    .F (3, C, D, H, W), .H, .BACK, and the new state.

    exact_bell=False keeps the reference's growth table (truncating index of
    u into bell values on a 1/255 grid); True evaluates the growth as the
    continuous bell(u, m, s) in double, the function the table samples;
    None follows the description's exact_bell flag."""

    def __init__(self, desc, kernels, xp: Xp = None, exact_bell: bool = None):
        self.xp = xp or Xp()
        self.exact_bell = bool(getattr(desc, "exact_bell", False)) if exact_bell is None else exact_bell
        self.desc = desc
        self.kernels = list(kernels)
        d = desc
        if d.growth_type != 1 or d.mode_type != 1 or d.gradient_mode != 0 or d.blur_central_diff or \
                d.border != 0 or d.sobel_border != 0 or int(d.dd) != 1 or d.mu_vel or \
                d.osc_la or d.osc_flow or d.osc_div_flow or any(d.soft_clip[:d.channels]):
            raise NotImplementedError("the float64 oracle covers the plain-step modes only")
        self.shape = (d.width, d.height, d.width)[::-1]  # (D, H, W)
        self.khat = [self.xp.rfftn(self.xp.asarray(kernel_grid64(d, kp))) for kp in self.kernels]
        self.lut_base = []
        for kp in self.kernels:
            mi = int(_f32(kp.m) * _f32(255))
            si = int(_f32(kp.s) * _f32(255))
            self.lut_base.append(mi * 65536 + si * 256)
        C = d.channels
        self.state = State(self.xp.zeros((C,) + self.shape), self.xp.zeros((3, C) + self.shape),
                           self.xp.zeros((C,) + self.shape), self.xp.zeros(self.shape))

    def set_state(self, A, V=None, GA=None, SUM=None):
        C = self.desc.channels
        xp = self.xp
        self.state = State(xp.asarray(np.asarray(A, np.float64).reshape((C,) + self.shape)),
                           xp.zeros((3, C) + self.shape) if V is None else
                           xp.asarray(np.asarray(V, np.float64).reshape((3, C) + self.shape)),
                           xp.zeros((C,) + self.shape) if GA is None else
                           xp.asarray(np.asarray(GA, np.float64).reshape((C,) + self.shape)),
                           xp.zeros(self.shape) if SUM is None else
                           xp.asarray(np.asarray(SUM, np.float64).reshape(self.shape)))

    # ------------------------------------------------------------ growth
    def _growth_value(self, k, u):
        """Entry of the growth table at the truncating index of u (double),
        or the exact bell of u."""
        xp = self.xp
        if self.exact_bell:
            kp = self.kernels[k]
            q = (u - float(_f32(kp.m))) / float(_f32(kp.s))
            return xp.exp(-(q * q) / 2.0)
        ui = xp.trunc_int(u * 255.0)
        f = ui + self.lut_base[k]
        valid = (f >= 0) & (f < (1 << 24))
        fm = (f >> 16) & 255
        fs = (f >> 8) & 255
        fu = f & 255
        x, m, s = xp.f64(fu) / 255.0, xp.f64(fm) / 255.0, xp.f64(fs) / 255.0
        q = (x - m) / s
        val = xp.exp(-(q * q) / 2.0)
        return xp.where(valid, val, 0.0)

    def _grad(self, f):
        """Central differences with torus borders: (x, y, z) components."""
        xp = self.xp
        return [(xp.roll(f, -1, ax) - xp.roll(f, 1, ax)) * 0.5 for ax in (-1, -2, -3)]

    def step(self):
        xp, d, st = self.xp, self.desc, self.state
        C, K = d.channels, len(self.kernels)
        D, H, W = self.shape
        N = D * H * W
        ahat = [xp.rfftn(st.A[c]) for c in range(C)]
        U = [xp.irfftn(ahat[kp.c0] * self.khat[k], self.shape) for k, kp in enumerate(self.kernels)]
        Hf = [xp.zeros(self.shape) for _ in range(C)]
        for k, kp in enumerate(self.kernels):
            l = self._growth_value(k, U[k])
            g = (l - st.A[kp.c1]) * float(_f32(kp.h)) if d.asymptotic[kp.c1] else l * float(_f32(kp.h))
            Hf[kp.c1] = Hf[kp.c1] + g
        dt = float(_f32(d.timestep))
        BACK = [xp.clip(st.A[c] + Hf[c] * dt, 0.0, 1.0) for c in range(C)]
        # gradients of H (U_S) and SUM (SUM_S), central differences
        NA = self._grad(st.SUM)
        NU = [self._grad(Hf[c]) for c in range(C)]
        # PREALPHA in the reference's flat layout (Q20)
        theta = float(_f32(d.theta_a))
        P = (W + 8) * (H + 8) * (W + 8)
        lim = 4 * N
        pre_flat = np.zeros(lim, np.float64) if xp.torch is None else xp.zeros((lim,))
        for c in range(C):
            off = c * N if d.alpha_index_fix else c * P
            if off >= lim:
                continue
            n = min(N, lim - off)
            v = xp.clip((st.A[c] / theta) ** 2, 0.0, 1.0).reshape(-1)[:n]
            pre_flat[off:off + n] = v
        F = []
        for dd in range(3):
            F.append([NU[c][dd] * (1.0 - pre_flat[c * N:(c + 1) * N].reshape(self.shape)) -
                      NA[dd] * pre_flat[c * N:(c + 1) * N].reshape(self.shape) for c in range(C)])
        # mu and V
        sigma = float(_f32(d.sigma))
        ma = float(_f32(d.dd)) - sigma
        damp = float(_f32(d.v_damp))
        pos = [xp.asarray(np.arange(n) + 0.5) for n in (W, H, D)]
        pshape = [(1, 1, W), (1, H, 1), (D, 1, 1)]
        MU = [[pos[dd].reshape(pshape[dd]) + xp.clip(F[dd][c] * dt, -ma, ma) for c in range(C)] for dd in range(3)]
        Vn = xp.zeros((3, C) + self.shape)
        for dd in range(3):
            for c in range(C):
                Vn[dd, c] = (st.V[dd, c] + F[dd][c]) * damp
        # RT reintegration, dd = 1, torus
        s2 = 1.0 / (4.0 * sigma * sigma)
        s23 = 1.0 / (2.0 * sigma * sigma * sigma)
        s_norm = float(_f32(d.s_norm))
        sn = s2 * (1.0 - s_norm) + s_norm * s23
        clip = min(2.0 * sigma, 1.0)
        si = 0.5 + sigma
        crt = C if d.rt_all_channels else min(C, 3)
        ext = (W, H, D)
        half = [float(e // 2) for e in ext]
        TT = [xp.zeros(self.shape) for _ in range(C)]
        idx = [np.arange(n) for n in (W, H, D)]
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    off = (ox, oy, oz)
                    outs = [((idx[a] + off[a] < 0) | (idx[a] + off[a] >= ext[a])).astype(np.int64) for a in range(3)]
                    nout = outs[0][None, None, :] + outs[1][None, :, None] + outs[2][:, None, None]
                    keep = xp.bool1d(nout < 2)

                    def at_src(f):
                        # the value at destination + offset, periodic
                        for a, ax in ((0, -1), (1, -2), (2, -3)):
                            if off[a]:
                                f = xp.roll(f, -off[a], ax)
                        return f

                    for c in range(crt):
                        w = None
                        for a in range(3):
                            m = pos[a].reshape(pshape[a]) - at_src(MU[a][c])
                            m = xp.where(m > half[a], m - ext[a], m)
                            m = xp.where(m < -half[a], m + ext[a], m)
                            m = xp.minimum(xp.maximum(si - abs(m), 0.0), clip)
                            w = m if w is None else w * m
                        TT[c] = TT[c] + xp.where(keep, at_src(BACK[c]) * w * sn, 0.0)
        # transpose_to_row_major
        gta, sta = float(_f32(d.gta)), float(_f32(d.sta))
        A_new = xp.zeros((C,) + self.shape)
        GA_new = xp.zeros((C,) + self.shape)
        ttsum = xp.zeros(self.shape)
        for c in range(C):
            tt = xp.clip(TT[c], 0.0, 1.0)
            ttsum = ttsum + tt
            GA_new[c] = (1.0 - gta) * st.GA[c] + tt * gta
            A_new[c] = tt
        SUM_new = (1.0 - sta) * st.SUM + ttsum * sta
        self.U = U
        self.F = F
        self.H = Hf
        self.BACK = BACK
        self.state = State(A_new, Vn, GA_new, SUM_new)

    def mass(self):
        """Total mass of each channel (double)."""
        return [float(self.state.A[c].sum()) for c in range(self.desc.channels)]
