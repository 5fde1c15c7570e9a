"""Failure detection: the library's device-side error reports.

The reference has no error handling (lenia.h:73: "does not bounds check").
Here a non-finite value reaching the growth stage and a tile-copy wait that
runs out are recorded on the device and reported by the next lenia_sync as
LENIA_ERR_NONFINITE / LENIA_ERR_TIMEOUT.  Both are provoked without any GPU
fault: a NaN written into the grid through the C ABI, and a wait limit of 0
polls (every wait gives up at once; the block drains its copies in flight and
returns).  After each error the same world, reset, steps bit for bit like the
oracle again.
"""
import numpy as np
import pytest

from lenia_b200 import _lib
from lenia_b200 import params as P
from lenia_cases import as_oracle
from oracle.oracle import RestateOracle

pytestmark = pytest.mark.gpu


def _oracle_after(wl, steps):
    p, ks = as_oracle(wl)
    ora = RestateOracle(p, ks, fft_mode="half")
    ora.set_state(A=wl.A0.ravel())
    ora.step(steps)
    return ora.get("A")


def _expect_status(fn, status):
    with pytest.raises(_lib.LeniaError) as ei:
        fn()
    assert ei.value.status == status, str(ei.value)


@pytest.mark.parametrize("growth", ["fused", "split", "exact_bell"])
def test_nan_in_grid_reports_nonfinite(growth):
    from lenia_b200.world import World
    wl = P.config0(seed=0)
    if growth == "exact_bell":
        wl.desc.exact_bell = True
    w = World(wl.desc, wl.kernels)
    w.set_tuning(0, growth == "split")
    a = wl.A0.ravel().copy()
    a[len(a) // 2] = np.nan
    w.set_state(a)
    w.step(1)
    _expect_status(w.sync, _lib.LENIA_ERR_NONFINITE)
    # the flag is cleared by the report; the world is usable again
    w.set_state(wl.A0.ravel())
    w.step(3)
    w.sync()
    got = w.get("A")
    w.close()
    assert np.array_equal(got, _oracle_after(wl, 3))


@pytest.mark.parametrize("mode", ["rt", "adv"])
def test_wait_limit_reports_timeout(mode):
    from lenia_b200.world import World
    wl = P.config0(seed=1)
    if mode == "adv":
        wl.desc.mode_type = P.MODE_ADV
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    w.step(1)
    w.sync()
    w.set_wait_limit(0)
    w.step(1)
    _expect_status(w.sync, _lib.LENIA_ERR_TIMEOUT)
    w.set_wait_limit(-1)
    w.set_state(wl.A0.ravel())
    w.step(3)
    w.sync()
    got = w.get("A")
    w.close()
    assert np.array_equal(got, _oracle_after(wl, 3))


def test_wait_limit_rejects_out_of_range():
    from lenia_b200.world import World
    wl = P.config0(seed=0)
    w = World(wl.desc, wl.kernels)
    _expect_status(lambda: w.set_wait_limit(1 << 40), _lib.LENIA_ERR_INVALID_ARG)
    w.set_wait_limit(1 << 20)
    w.set_state(wl.A0.ravel())
    w.step(2)
    w.sync()
    got = w.get("A")
    w.close()
    assert np.array_equal(got, _oracle_after(wl, 2))
