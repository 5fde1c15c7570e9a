"""Opt-in mass conservation (LeniaWorldDesc.conserve_mass): after every step
each channel is rescaled so that its total, summed in double on the GPU in a
fixed order, equals the total recorded when the grid was last written.  No
counterpart in the reference, whose RT reintegration with sigma 0.65 spreads
1.30 of a cell's mass per step."""
import numpy as np
import pytest

from lenia_b200 import params as P

pytestmark = pytest.mark.gpu


def _totals(a, C):
    return a.reshape(C, -1).astype(np.float64).sum(axis=1)


def test_one_step_is_the_plain_step_rescaled():
    from lenia_b200.world import World
    wl = P.config0(seed=12)
    C = wl.desc.channels
    plain = World(wl.desc, wl.kernels)
    wl.desc.conserve_mass = True
    cons = World(wl.desc, wl.kernels)
    for w in (plain, cons):
        w.set_state(wl.A0.ravel())
        w.step(1)
        w.sync()
    a_raw, a_cons = plain.get("A"), cons.get("A")
    target, total = _totals(wl.A0, C), _totals(a_raw, C)
    assert np.all(total > 1.2 * target)              # sigma 0.65: the plain step gains mass
    scale = (target / total).astype(np.float32)
    want = (a_raw.reshape(C, -1) * scale[:, None]).ravel()
    # the double totals differ from numpy's only in summation order: the float
    # scale factors may differ in their last bit
    assert np.allclose(a_cons, want, rtol=2.0 ** -22, atol=0)
    assert np.allclose(_totals(a_cons, C), target, rtol=1e-6)


def test_totals_held_over_many_steps_and_in_a_batch():
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wl = P.config0(seed=13)
    wl.desc.conserve_mass = True
    C = wl.desc.channels
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    w.step(20)
    w.sync()
    # every step rescales to the recorded totals with one float factor per
    # channel: the total is off by that factor's rounding and the products'
    # (each <= 2^-24 relative), about 1e-7, and the error does not accumulate
    assert np.allclose(_totals(w.get("A"), C), _totals(wl.A0, C), rtol=1e-6, atol=0)
    assert np.isfinite(w.get("A")).all()
    wls = P.config3(3, seed=15, sizes=(24, 32))
    for x in wls:
        x.desc.conserve_mass = True
    b = Batch([x.desc for x in wls], [x.kernels for x in wls], lanes=2)
    for i, x in enumerate(wls):
        b.set_state(i, x.A0)
    b.step(5)
    b.sync()
    for i, x in enumerate(wls):
        assert np.allclose(_totals(b.get(i, "A"), 3), _totals(x.A0, 3), rtol=1e-6, atol=0), i
