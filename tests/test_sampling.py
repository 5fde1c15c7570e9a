"""generate_random against the reference's own function (reference build
with the reference platform's rand())."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O
from lenia_b200.sampling import MsvcRand, generate_random

import lenia_cases as LC

needs_ref = pytest.mark.skipif(not os.path.exists(O.ref_path("lenia.cpp")), reason="reference sources absent")


def test_msvc_rand_known_sequence():
    """The MSVC runtime's well-known first outputs after srand(1)."""
    r = MsvcRand(1)
    assert [r.rand() for _ in range(10)] == [41, 18467, 6334, 26500, 19169, 15724, 11478, 29358, 26962, 24464]
    xs = [MsvcRand(7).rand() for _ in range(3)]
    assert all(0 <= x <= 32767 for x in xs)


@needs_ref
@pytest.mark.parametrize("seed", [1, 7, 1234, 99991])
@pytest.mark.parametrize("channels", [1, 3])
def test_generate_random_matches_reference(seed, channels):
    wl = LC.variant("cfg0")
    wl.desc.channels = channels
    wl.kernels = [k for k in wl.kernels if k.c0 < channels and k.c1 < channels]
    p, k = LC.as_oracle(wl)
    ref = O.RefOracle(p, k)
    lib = ref.lib()
    out = (O.OraKernel * 12)()
    nb = ctypes.c_float()
    n = lib.ref_generate_random(ctypes.c_uint(seed), out, 12, ctypes.byref(nb))
    ks, A0, neighborhood = generate_random(MsvcRand(seed), channels, 32, 32)
    assert n == len(ks) and nb.value == neighborhood
    for a, b in zip(out[:n], ks):
        assert a.radius == b.radius and a.beta_size == b.beta_size and (a.c0, a.c1) == (b.c0, b.c1)
        assert [np.float32(x) for x in a.b[:a.beta_size]] == [np.float32(x) for x in b.b]
        for name in ("m", "s", "h", "r_a"):
            assert np.float32(getattr(a, name)) == np.float32(getattr(b, name)), name
    # the seed grid: the reference build's exp(float) is the C library's expf,
    # the port rounds a double exp; five blobs are summed, so a cell can
    # differ by up to two units in the last place
    grid = ref.get("A").reshape(channels, 32, 32, 32)
    ulps = np.abs(grid.view(np.int32).astype(np.int64) - A0.view(np.int32).astype(np.int64))
    assert ulps.max() <= 2, ulps.max()
    assert (ulps == 0).mean() > 0.99
