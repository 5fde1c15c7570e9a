"""Accuracy of the project's FFT (LFFT) and of the half-spectrum convolution
that the CUDA library performs, against double-precision numpy transforms and
against the reference's complex-to-complex structure."""
import numpy as np
import pytest

from lenia_cases import as_oracle, variant
from oracle.oracle import RestateOracle

SIZES = [8, 12, 16, 20, 24, 28, 32, 36, 40, 44, 48, 56, 64, 96, 128, 256]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("sign", [-1, +1])
def test_lfft_matches_double_dft(oracle_built, n, sign):
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    got = RestateOracle.lfft_1d(x, sign).astype(np.complex128)
    xd = x.astype(np.complex128)
    want = np.fft.fft(xd) if sign < 0 else np.fft.ifft(xd) * n
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 2e-7 * np.log2(n) + 1e-7, err


def test_radix_plan():
    import ctypes
    lib = RestateOracle.lib()
    plans = {128: [8, 8, 2], 256: [8, 8, 4], 36: [4, 3, 3], 44: [4, 11], 24: [8, 3], 96: [8, 4, 3], 48: [8, 2, 3]}
    for n, want in plans.items():
        r = (ctypes.c_int * 16)()
        k = lib.ora_lfft_factor(n, r)
        assert list(r[:k]) == want, n


def test_half_spectrum_forward_matches_numpy(oracle_built):
    wl = variant("cfg0")
    p, ks = as_oracle(wl)
    o = RestateOracle(p, ks, fft_mode="half")
    W = wl.desc.width
    rng = np.random.default_rng(1)
    fa = rng.random(W ** 3, dtype=np.float64).astype(np.float32)
    fb = rng.random(W ** 3, dtype=np.float64).astype(np.float32)
    sa, sb = o.hs_forward(fa, fb)
    for f, s in ((fa, sa), (fb, sb)):
        want = np.fft.rfftn(f.reshape(W, W, W).astype(np.float64))      # [z][y][kx]
        want = np.transpose(want, (2, 0, 1)).ravel()                     # [kx][z][y]
        err = np.abs(s.astype(np.complex128) - want).max() / np.abs(want).max()
        assert err < 1e-6, err


def test_half_and_c2c_convolutions_agree(oracle_built):
    """The CUDA library's arithmetic (half) and the reference's structure (c2c)
    give the same u up to float rounding."""
    wl = variant("cfg0", seed=9)
    p, ks = as_oracle(wl)
    us = []
    for mode in ("half", "c2c"):
        o = RestateOracle(p, ks, fft_mode=mode)
        o.set_state(A=wl.A0.ravel())
        o.run_event("FFT")
        us.append(o.get("U").astype(np.float64))
    diff = np.abs(us[0] - us[1]).max()
    assert diff < 2e-6, diff
    assert np.abs(us[1]).max() > 0.01
