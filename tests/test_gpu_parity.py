"""Parity of the CUDA step with the CPU restatement (oracle/restate).

The restatement runs in its half-spectrum mode, which performs the CUDA
library's convolution arithmetic; every other stage is the reference's
arithmetic (pinned bit for bit to the reference's own code by
test_oracle_pin.py).  So the bar is bit-exact equality: after every stage
group of every step, every field, in every mode.
"""
import numpy as np
import pytest

from lenia_cases import CLEAN_VARIANTS, VARIANTS, as_oracle, diff_report, four_channels, two_channel_div_flow, variant
from lenia_b200 import params as P
from oracle.oracle import RestateOracle

pytestmark = pytest.mark.gpu

GROWTH_EVENTS = ["FFT", "FFT_MT"]
FLOW_EVENTS = ["TSB", "SOBEL_ONE", "SOBEL_TWO", "F", "MU", "TB"]


def make_pair(wl, debug=True):
    from lenia_b200.world import World
    p, ks = as_oracle(wl)
    ora = RestateOracle(p, ks, fft_mode="half")
    ora.set_state(A=wl.A0.ravel())
    gpu = World(wl.desc, wl.kernels)
    if debug:
        gpu.set_debug(True)
    gpu.set_state(wl.A0.ravel())
    return ora, gpu


def compare(ora, gpu, names, tag, problems):
    for n in names:
        r = diff_report(n, ora.get(n), gpu.get(n))
        if r:
            problems.append(f"{tag} {r}")


def staged_step(ora, gpu, desc, tag, problems):
    for ev in GROWTH_EVENTS:
        ora.run_event(ev)
    gpu.stage("GROWTH")
    names = ["U", "H", "U_SUM"] + (["BACK"] if desc.growth_type == P.GROWTH_RT else [])
    compare(ora, gpu, names, f"{tag} GROWTH", problems)
    ora.run_event("BLUR")
    gpu.stage("BLUR")
    if desc.gradient_mode == P.GRADIENT_CENTRAL_DIFF:
        compare(ora, gpu, ["U_S", "SUM_S"], f"{tag} BLUR", problems)
    for ev in FLOW_EVENTS:
        ora.run_event(ev)
    gpu.stage("FLOW")
    compare(ora, gpu, ["NA", "NU", "PREALPHA", "ALPHA", "F", "MU", "V"], f"{tag} FLOW", problems)
    ora.run_event("REINTEGRATION")
    gpu.stage("TRANSPORT")
    compare(ora, gpu, ["TT"], f"{tag} REINTEGRATION", problems)
    ora.run_event("TRM")
    ora.run_event("TMB")
    names = ["A", "GA", "SUM"]
    if desc.growth_type == P.GROWTH_TRANSPOSITION and any(desc.soft_clip[:desc.channels]):
        names.append("BACK")
    compare(ora, gpu, names, f"{tag} TRANSPORT", problems)


def run_staged(wl, steps=2):
    ora, gpu = make_pair(wl)
    problems = []
    for s in range(steps):
        staged_step(ora, gpu, wl.desc, f"step {s}", problems)
    gpu.sync()
    gpu.close()
    return problems


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_stages_bit_exact(cuda_lib, oracle_built, name):
    problems = run_staged(variant(name))
    assert not problems, "\n".join(problems[:12])


@pytest.mark.parametrize("name", sorted(CLEAN_VARIANTS))
def test_stages_bit_exact_clean_modes(cuda_lib, oracle_built, name):
    """The library's exact-bell growth (no growth table) against the C
    restatement with the same option."""
    wl = variant(name, seed=21)
    problems = run_staged(wl, steps=2)
    assert not problems, "\n".join(problems[:12])


def test_stages_bit_exact_div_flow(cuda_lib, oracle_built):
    problems = run_staged(two_channel_div_flow())
    assert not problems, "\n".join(problems[:12])


def test_stages_bit_exact_four_channels(cuda_lib, oracle_built):
    problems = run_staged(four_channels())
    assert not problems, "\n".join(problems[:12])


@pytest.mark.parametrize("width", [24, 36, 44, 48])
def test_stages_bit_exact_mixed_radix(cuda_lib, oracle_built, width):
    """Grid sizes whose transforms use radices 3 and 11."""
    problems = run_staged(variant("sobel_torus", seed=width, width=width), steps=1)
    assert not problems, "\n".join(problems[:12])


@pytest.mark.parametrize("width", [64, 96])
def test_stages_bit_exact_paired_plane_sizes(cuda_lib, oracle_built, width):
    """One-plane-per-block plane passes at 64 (radix 8 only) and 96 (8, 4, 3),
    whose butterflies run as paired FP32 instructions, against the scalar C
    restatement."""
    problems = run_staged(variant("sobel_torus", seed=width + 1, width=width), steps=1)
    assert not problems, "\n".join(problems[:12])


@pytest.mark.parametrize("shape", [(32, 24), (24, 40)])
def test_stages_bit_exact_non_cubic(cuda_lib, oracle_built, shape):
    """Width != height runs the runtime-sized kernels (the size-specialised
    ones cover cubic grids)."""
    w, h = shape
    wl = variant("sobel_torus", seed=w + h, width=w)
    wl.desc.height = h
    rng = np.random.default_rng(w * h)
    wl.A0 = P.seed_cube(rng, wl.desc, min(w, h) // 2)
    problems = run_staged(wl, steps=1)
    assert not problems, "\n".join(problems[:12])


def test_stages_bit_exact_split_planes(cuda_lib, oracle_built):
    """A kx plane of 100 x 256 complex values (200 KB) does not fit the
    one-pass plane transform: the y and z line transforms run as separate
    passes and stay bit-exact."""
    wl = variant("sobel_torus", seed=356, width=100)
    wl.desc.height = 256
    rng = np.random.default_rng(356)
    wl.A0 = P.seed_cube(rng, wl.desc, 32)
    problems = run_staged(wl, steps=1)
    assert not problems, "\n".join(problems[:12])


def test_growth_stage_bit_exact_256(cuda_lib, oracle_built):
    """256^3: the size-specialised row transforms with the split plane passes
    (a 256 x 256 plane exceeds shared memory) give the growth stage's u_k, H,
    U_SUM and BACK bit for bit (2 channels, 2 kernels keep the CPU side short)."""
    wl = P.config2(seed=9, width=256, radius=12)
    wl.desc.channels = 2
    wl.kernels = [k for k in wl.kernels if k.c0 < 2 and k.c1 < 2][:2]
    wl.A0 = wl.A0[:2].copy()
    ora, gpu = make_pair(wl)
    for ev in GROWTH_EVENTS:
        ora.run_event(ev)
    gpu.stage("GROWTH")
    gpu.sync()
    problems = []
    compare(ora, gpu, ["U", "H", "U_SUM", "BACK"], "256^3 GROWTH", problems)
    gpu.close()
    assert not problems, "\n".join(problems[:12])


def test_trajectory_bit_exact_cfg0(cuda_lib, oracle_built):
    """Whole steps (the production path, no debug outputs) stay bit-exact over
    100 steps of the 32^3 plain-step configuration."""
    from lenia_b200.world import World
    wl = P.config0(seed=0)
    p, ks = as_oracle(wl)
    ora = RestateOracle(p, ks, fft_mode="half")
    ora.set_state(A=wl.A0.ravel())
    gpu = World(wl.desc, wl.kernels)
    gpu.set_state(wl.A0.ravel())
    for chunk in range(10):
        ora.step(10)
        gpu.step(10)
        for n in ("A", "V", "GA", "SUM"):
            r = diff_report(n, ora.get(n), gpu.get(n))
            assert not r, f"after {10 * (chunk + 1)} steps: {r}"
    gpu.sync()


@pytest.mark.parametrize("growth_split", [False, True], ids=["fused_growth", "split_growth"])
def test_config1_step_bit_exact(cuda_lib, oracle_built, growth_split):
    """One full step of the 128^3 x 4 channel, 16-kernel configuration, with
    the growth stage as one fused pass or as inverse rows storing u_k followed
    by the growth from u_k (the form the autotuner picks for this world)."""
    from lenia_b200.world import World
    wl = P.config1(seed=1)
    p, ks = as_oracle(wl)
    ora = RestateOracle(p, ks, fft_mode="half")
    ora.set_state(A=wl.A0.ravel())
    gpu = World(wl.desc, wl.kernels)
    gpu.set_tuning(0, growth_split)
    gpu.set_state(wl.A0.ravel())
    ora.step(1)
    gpu.step(1)
    for n in ("A", "V", "GA", "SUM", "H", "U_SUM", "BACK", "MU"):
        r = diff_report(n, ora.get(n), gpu.get(n))
        assert not r, r
    gpu.sync()


@pytest.mark.parametrize("mode", ["rt", "advection"])
def test_config1_ten_steps_bit_exact(cuda_lib, oracle_built, mode):
    """The 128^3 x 4 channel, 16-kernel configuration with RT and with
    advection reintegration (adv_vel: the semi-Lagrangian pull of every
    channel, reintegration.cpp:1112-1260): whole production steps, autotuned
    as a user runs them, bit-exact after the first step and after ten."""
    from lenia_b200.world import World
    wl = P.config1(seed=4, mode=P.MODE_RT if mode == "rt" else P.MODE_ADV)
    p, ks = as_oracle(wl)
    ora = RestateOracle(p, ks, fft_mode="half")
    ora.set_state(A=wl.A0.ravel())
    gpu = World(wl.desc, wl.kernels)
    gpu.autotune(modes=("FFT",))
    gpu.set_state(wl.A0.ravel())
    for steps in (1, 9):
        ora.step(steps)
        gpu.step(steps)
        for n in ("A", "V", "GA", "SUM"):
            r = diff_report(n, ora.get(n), gpu.get(n))
            assert not r, f"{mode}: {r}"
    gpu.sync()
    gpu.close()
