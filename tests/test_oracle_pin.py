"""Pins the C restatement (oracle/restate) to the reference's own code.

The reference's lenia.cpp, reintegration.cpp, transposition.cpp and mesh.cpp
are compiled unmodified (oracle/_ref) and stepped by the serial event driver;
the restatement runs the same seeded inputs.  Both use the LFFT engine in
place of FFTW, so every field must agree bit for bit after every event of
every step, in every mode, except where the reference's documented
out-of-bounds writes land (Q20): SUM between SOBEL_TWO and REINTEGRATION,
SUM_S outside BLUR..SOBEL_ONE (both rewritten before their next read), and
ALPHA with three or more channels (GA read past its end).
"""
import os

import numpy as np
import pytest

from lenia_cases import VARIANTS, as_oracle, diff_report, four_channels, two_channel_div_flow, variant
from oracle.oracle import EVENTS, REF_DIR, REF_LIB, REF_LIB_128, RefOracle, RestateOracle

FIELDS = ["A", "V", "GA", "SUM", "H", "U_SUM", "BACK", "NA", "NU", "PREALPHA", "ALPHA", "F", "MU", "TT",
          "U_S", "SUM_S", "U", "H_RB", "U_SUM_RB", "RBB"]
SUM_TRANSIENT = {"SOBEL_TWO", "F", "MU", "TB"}
SUM_S_LIVE = {"BLUR", "TSB", "SOBEL_ONE"}

pytestmark = pytest.mark.skipif(
    not (os.path.isdir(REF_DIR) or os.path.exists(REF_LIB)),
    reason="reference sources / build unavailable")


def run_pin(wl, steps=2):
    p, ks = as_oracle(wl)
    ref = RefOracle(p, ks)
    ora = RestateOracle(p, ks, fft_mode="c2c")
    A0 = wl.A0.ravel()
    ref.set_state(A=A0)
    ora.set_state(A=A0)
    problems = []
    for step in range(steps):
        for ev in range(len(EVENTS)):
            ref.run_event(ev)
            ora.run_event(ev)
            for name in FIELDS:
                if name == "SUM" and EVENTS[ev] in SUM_TRANSIENT:
                    continue
                if name == "SUM_S" and EVENTS[ev] not in SUM_S_LIVE:
                    continue
                if name == "ALPHA" and wl.desc.channels >= 3:
                    continue
                r = diff_report(name, ref.get(name), ora.get(name))
                if r:
                    problems.append(f"step {step} {EVENTS[ev]} {r}")
    return problems


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_restatement_matches_reference(oracle_built, name):
    problems = run_pin(variant(name))
    assert not problems, "\n".join(problems[:10])


def test_restatement_matches_reference_div_flow(oracle_built):
    problems = run_pin(two_channel_div_flow())
    assert not problems, "\n".join(problems[:10])


def test_restatement_matches_reference_four_channels(oracle_built):
    problems = run_pin(four_channels())
    assert not problems, "\n".join(problems[:10])


def test_kernel_construction_matches_reference(oracle_built):
    wl = variant("cfg0", seed=11)
    p, ks = as_oracle(wl)
    ref = RefOracle(p, ks)
    ora = RestateOracle(p, ks, fft_mode="c2c")
    for k in range(len(ks)):
        assert np.array_equal(ref.kernel_grid(k), ora.kernel_grid(k)), k
        assert np.array_equal(ref.kernel_spectrum(k), ora.kernel_spectrum(k)), k
        # kernels are normalised: the cells sum to 1
        assert abs(float(ora.kernel_grid(k).astype(np.float64).sum()) - 1.0) < 1e-5
    assert np.array_equal(ref.blur_grid(), ora.blur_grid())
    assert abs(float(ora.blur_grid().astype(np.float64).sum()) - 1.0) < 1e-6


def test_bell_table_matches_reference(oracle_built):
    wl = variant("cfg0")
    p, ks = as_oracle(wl)
    ref = RefOracle(p, ks)
    rng = np.random.default_rng(0)
    for m, s, u in rng.integers(0, 256, size=(2000, 3)):
        a, b = ref.bell_lut(int(m), int(s), int(u)), RestateOracle.bell_lut(int(m), int(s), int(u))
        assert (a == b) or (np.isnan(a) and np.isnan(b)), (m, s, u, a, b)


def test_reference_slab_threads_match_serial(oracle_built):
    """The reference's two sim threads (each event's slabs at once) give the
    serial driver's bits: the reference arm of the benchmark times them."""
    from lenia_b200 import params as P
    wl = P.config0(seed=1)
    p, ks = as_oracle(wl)
    ref = RefOracle(p, ks)
    ref.set_state(A=wl.A0.ravel())
    ref.step(4)
    serial = {n: ref.get(n) for n in ("A", "GA", "SUM", "V")}
    z = np.zeros
    ref.set_state(A=wl.A0.ravel(), V=z(serial["V"].size, np.float32), GA=z(serial["GA"].size, np.float32),
                  SUM=z(serial["SUM"].size, np.float32))
    ref.step(4, slab_threads=True)
    for n, v in serial.items():
        assert np.array_equal(ref.get(n), v), n


@pytest.mark.skipif(not (os.path.isdir(REF_DIR) or os.path.exists(REF_LIB_128)),
                    reason="headline-size reference build unavailable")
def test_headline_size_reference_build_matches_restatement(oracle_built):
    """The reference built at 128^3 with 16 kernels (a generated render.h,
    oracle/Makefile) steps the headline world bit for bit like the
    restatement (complex-to-complex FFT structure)."""
    from lenia_b200 import params as P
    wl = P.config1(seed=1, width=128)
    p, ks = as_oracle(wl)
    ref = RefOracle(p, ks, lib=REF_LIB_128)
    ref.set_state(A=wl.A0.ravel())
    ref.step(1, slab_threads=True)
    ora = RestateOracle(p, ks, fft_mode="c2c")
    ora.set_state(A=wl.A0.ravel())
    ora.step(1)
    for n in ("A", "GA", "SUM", "U_SUM"):
        assert np.array_equal(ref.get(n), ora.get(n)), n


def test_float64_fft_build_differs_at_rounding_level(oracle_built):
    """The reference linked with the float64 FFT stand-in computes the same
    transform: after one growth stage u agrees with the float build within
    float rounding of the convolution."""
    from lenia_b200 import params as P
    from oracle.oracle import REF_LIB_FFT64
    wl = P.config0(seed=0)
    p, ks = as_oracle(wl)
    a = RefOracle(p, ks)
    b = RefOracle(p, ks, lib=REF_LIB_FFT64)
    for r in (a, b):
        r.set_state(A=wl.A0.ravel())
        r.run_event("FFT")
    ua, ub = a.get("U"), b.get("U")
    assert np.abs(ua.astype(np.float64) - ub).max() < 2e-6
    assert not np.array_equal(ua, ub)
