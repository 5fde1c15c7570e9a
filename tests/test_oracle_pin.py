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
from oracle.oracle import EVENTS, REF_DIR, REF_LIB, RefOracle, RestateOracle

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
