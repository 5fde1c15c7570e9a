"""The float64 oracle of the precision study (oracle/fp64.py) against the C
restatement (float32, pinned to the reference by the golden tests): one step
from the same state of the 32^3 plain step.

Both compute the same algorithm; they differ by float32 rounding only, which
moves u by about 1e-6.  F and the grid then differ only in cells whose u
crosses a growth-table bin (u * 255 truncated), a few in 10^4.
"""
import numpy as np
import pytest

from lenia_b200 import params as P


@pytest.mark.parametrize("seed", [5, 9])
def test_one_step_matches_float32_oracle(oracle_built, seed):
    from oracle import fp64
    wl = P.config0(seed=seed)
    d = wl.desc
    C, K = d.channels, len(wl.kernels)
    ora = oracle_built.RestateOracle(d.as_dict(), [k.as_dict() for k in wl.kernels])
    ora.set_state(A=wl.A0.ravel())
    f = fp64.Fp64Step(d, wl.kernels)
    f.set_state(wl.A0)
    ora.step(1)
    f.step()
    u32 = ora.get("U").reshape(K, -1).astype(np.float64)
    u64 = np.stack([x.ravel() for x in f.U])
    assert np.abs(u32 - u64).max() < 5e-6
    F32 = ora.get("F").reshape(3, C, -1).astype(np.float64)
    F64 = np.stack([np.stack([x.ravel() for x in row]) for row in f.F])
    assert np.mean(np.abs(F32 - F64) > 1e-4) < 1e-3
    A32 = ora.get("A").reshape(C, -1).astype(np.float64)
    A64 = np.asarray(f.state.A).reshape(C, -1)
    assert np.mean(np.abs(A32 - A64) > 1e-4) < 1e-3
    m32, m64 = A32.sum(axis=1), A64.sum(axis=1)
    assert np.all(np.abs(m32 - m64) <= 1e-5 * m64)


def test_kernel_grid_matches_float32_oracle(oracle_built):
    from oracle import fp64
    wl = P.config0(seed=3)
    d = wl.desc
    ora = oracle_built.RestateOracle(d.as_dict(), [k.as_dict() for k in wl.kernels])
    for k, kp in enumerate(wl.kernels):
        g32 = ora.kernel_grid(k).reshape(d.depth, d.height, d.width)
        g64 = fp64.kernel_grid64(d, kp)
        assert np.array_equal(g32 != 0, g64 != 0)
        assert np.abs(g32 - g64).max() <= 2e-5 * g64.max()  # float32 normalising sum
        assert abs(g64.sum() - 1.0) < 1e-12


def test_rejects_other_modes():
    from oracle import fp64
    wl = P.config1(seed=1, width=32)
    with pytest.raises(NotImplementedError):
        fp64.Fp64Step(wl.desc, wl.kernels)


def test_exact_bell_differs_only_by_table_quantisation(oracle_built):
    """The exact-bell variant agrees with the table variant on u (the
    convolution is the same) and its growth differs by at most one table
    step of the bell."""
    from oracle import fp64
    wl = P.config0(seed=5)
    a = fp64.Fp64Step(wl.desc, wl.kernels)
    b = fp64.Fp64Step(wl.desc, wl.kernels, exact_bell=True)
    for f in (a, b):
        f.set_state(wl.A0)
        f.step()
    for ua, ub in zip(a.U, b.U):
        assert np.array_equal(ua, ub)
    hsum = sum(float(np.float32(k.h)) for k in wl.kernels)
    for ha, hb in zip(a.H, b.H):
        assert 0 < np.abs(ha - hb).max() <= hsum * 0.2


def test_exact_bell_option_of_the_restatement(oracle_built):
    """exact_bell in the C restatement (float32) against the float64 oracle's
    exact bell: the growth agrees to float32 rounding, with no table steps."""
    from oracle import fp64
    wl = P.config0(seed=5)
    wl.desc.exact_bell = True
    d = wl.desc
    C = d.channels
    ora = oracle_built.RestateOracle(d.as_dict(), [k.as_dict() for k in wl.kernels])
    ora.set_state(A=wl.A0.ravel())
    ora.run_event("FFT")
    ora.run_event("FFT_MT")
    f = fp64.Fp64Step(d, wl.kernels)
    assert f.exact_bell
    f.set_state(wl.A0)
    f.step()
    H32 = ora.get("H").reshape(C, -1).astype(np.float64)
    H64 = np.stack([h.ravel() for h in f.H])
    assert np.abs(H32 - H64).max() < 1e-3  # u differs by ~1e-6, the bell slope is up to ~1/s
