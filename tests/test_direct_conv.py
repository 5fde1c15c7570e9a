"""Direct convolution on the tensor cores (LENIA_CONV_DIRECT_BF16 and
LENIA_CONV_DIRECT_BF16X3) against a float64 sum and the FP32 spectral path.

u_k = K_k (*) A_c0 on the torus (lenia.cpp:435-491).  The float64 reference
convolves the oracle's normalised kernel grid (the same grid both GPU paths
use, pinned by the oracle tests) with the grid by numpy FFT.  Error bounds,
with every kernel grid normalised to sum 1 and taps >= 0:
  BF16     each tap and cell value rounds to BF16 (relative error <= 2^-9
           each), so |du| <= 2^-8 max|A| plus FP32 accumulation;
  BF16X3   hi*hi + hi*lo + lo*hi leaves the lo*lo term and the rounding of
           the two lo parts, each at most 2^-18 of the product, so
           |du| <= 3 * 2^-18 max|A| from the split, plus the accumulation
           (the tensor cores' within one dz-run, FP32 adds between runs).
The growth fields (H, U_SUM, BACK) of a direct world follow bit for bit from
its own u_k through the reference's growth table (lenia.cpp:501-592).
"""
import numpy as np
import pytest

from lenia_b200 import params as P

pytestmark = pytest.mark.gpu


def _case(name):
    if name == "cfg0_32":
        return P.config0(seed=5)
    if name == "wide_144x40":
        # two x tiles of 128, rows of a non-cubic grid, radius 10
        rng = np.random.default_rng(11)
        desc = P.WorldDesc(width=144, height=40, channels=3, timestep=0.2, theta_a=2.0, sigma=0.65,
                           growth_type=P.GROWTH_RT, mode_type=P.MODE_RT, sobel_border=P.BORDER_TORUS,
                           border=P.BORDER_TORUS, gradient_mode=P.GRADIENT_CENTRAL_DIFF,
                           asymptotic=(False,) * 4)
        ks = P.sample_kernels(rng, 3, radius=10)
        return P.Workload(desc, ks, P.seed_cube(rng, desc, 40))
    if name == "plane_128":
        # 128 rows of one plane per tile (fewer tiles than rows run on
        # across planes with their y padding)
        return P.config2(seed=4, width=128, radius=10)
    if name == "four_ch_64":
        # four kernels per source channel: four accumulators of 128 columns
        return P.config1(seed=2, width=64, radius=13)
    raise KeyError(name)


def _oracle(wl, oracle_built):
    return oracle_built.RestateOracle(wl.desc.as_dict(), [k.as_dict() for k in wl.kernels])


def _u64(wl, ora):
    """float64 u_k of every kernel from the oracle's kernel grids."""
    d = wl.desc
    A = wl.A0.reshape(d.channels, d.depth, d.height, d.width).astype(np.float64)
    Ahat = [np.fft.rfftn(A[c]) for c in range(d.channels)]
    out = []
    for k, kp in enumerate(wl.kernels):
        g = ora.kernel_grid(k).reshape(d.depth, d.height, d.width).astype(np.float64)
        out.append(np.fft.irfftn(Ahat[kp.c0] * np.fft.rfftn(g), s=g.shape, axes=(0, 1, 2)))
    return np.stack(out)


def _worlds(wl, mode):
    from lenia_b200.world import World
    wf, wd = World(wl.desc, wl.kernels), World(wl.desc, wl.kernels)
    wd.set_conv_mode(mode)
    assert wd.conv_mode == mode and wf.conv_mode == "FFT"
    for w in (wf, wd):
        w.set_debug(True)
        w.set_state(wl.A0.ravel())
        w.stage("GROWTH")
        w.sync()
    return wf, wd


@pytest.mark.parametrize("case", ["cfg0_32", "wide_144x40", "four_ch_64", "plane_128"])
@pytest.mark.parametrize("mode", ["DIRECT_BF16X3", "DIRECT_BF16"])
def test_u_against_float64(cuda_lib, oracle_built, case, mode):
    wl = _case(case)
    ora = _oracle(wl, oracle_built)
    u64 = _u64(wl, ora)
    wf, wd = _worlds(wl, mode)
    K = len(wl.kernels)
    uf = wf.get("U").reshape(u64.shape).astype(np.float64)
    ud = wd.get("U").reshape(u64.shape).astype(np.float64)
    err_fft = np.abs(uf - u64).max()
    err_dir = np.abs(ud - u64).max()
    rms_dir = np.sqrt(np.mean((ud - u64) ** 2))
    amax = float(np.abs(wl.A0).max())
    print(f"{case} {mode}: max|u| {np.abs(u64).max():.4f}  err fft {err_fft:.3e}  direct {err_dir:.3e}  "
          f"rms direct {rms_dir:.3e}")
    assert np.isfinite(ud).all()
    assert err_fft < 1e-5
    if mode == "DIRECT_BF16":
        assert err_dir <= 2.0 ** -8 * amax + 1e-5
    else:
        assert err_dir <= 3 * 2.0 ** -18 * amax + 1e-5
        assert rms_dir < 2e-6
    issued, useful = wd.conv_macs()
    assert issued >= useful > 0
    parts = 3 if mode == "DIRECT_BF16X3" else 1
    d = wl.desc
    taps = sum(int(np.count_nonzero(ora.kernel_grid(i))) for i in range(K))
    assert useful == taps * d.width * d.height * d.depth * parts


@pytest.mark.parametrize("mode", ["DIRECT_BF16X3", "DIRECT_BF16"])
def test_growth_fields_follow_u(cuda_lib, oracle_built, mode):
    """H, U_SUM and BACK of a direct world from its own u_k, bit for bit."""
    wl = _case("cfg0_32")
    ora = _oracle(wl, oracle_built)
    _, wd = _worlds(wl, mode)
    d = wl.desc
    C, N, K = d.channels, d.cells, len(wl.kernels)
    U = wd.get("U").reshape(K, N)
    A = wl.A0.reshape(C, N).astype(np.float32)
    H = np.zeros((C, N), np.float32)
    US = np.zeros((C, N), np.float32)
    for k, kp in enumerate(wl.kernels):
        u = U[k]
        ui = (u * np.float32(255)).astype(np.int64)
        row = ora.lut_row(k)
        inside = (ui >= 0) & (ui < 256)
        l = np.zeros(N, np.float32)
        l[inside] = row[ui[inside]]
        if (~inside).any():
            base = int(kp.m * np.float32(255)) * 65536 + int(kp.s * np.float32(255)) * 256
            for i in np.nonzero(~inside)[0]:
                f = base + int(ui[i])
                l[i] = ora.bell_lut(f >> 16, (f >> 8) & 255, f & 255) if 0 <= f < 1 << 24 else 0.0
        US[kp.c1] = US[kp.c1] + u
        H[kp.c1] = H[kp.c1] + l * np.float32(kp.h)
    back = np.clip(A + H * np.float32(d.timestep), np.float32(0), np.float32(1))
    assert np.array_equal(wd.get("U_SUM").reshape(C, N).view(np.uint32), US.view(np.uint32))
    assert np.array_equal(wd.get("H").reshape(C, N).view(np.uint32), H.view(np.uint32))
    assert np.array_equal(wd.get("BACK").reshape(C, N).view(np.uint32), back.view(np.uint32))


def test_steps_track_fft_path(cuda_lib):
    """Whole steps with the BF16X3 convolution stay within FP32 noise of the
    spectral path's trajectory over 10 steps of config 0."""
    from lenia_b200.world import World
    wl = P.config0(seed=6)
    ws = {}
    for mode in ("FFT", "DIRECT_BF16X3"):
        w = World(wl.desc, wl.kernels)
        w.set_conv_mode(mode)
        w.set_state(wl.A0.ravel())
        w.step(10)
        w.sync()
        ws[mode] = w.get("A").astype(np.float64)
    a, b = ws["FFT"], ws["DIRECT_BF16X3"]
    assert np.isfinite(b).all()
    print("max|dA|", np.abs(a - b).max(), "mass", a.sum(), b.sum())
    assert abs(a.sum() - b.sum()) <= 1e-4 * a.sum()
    assert np.mean(np.abs(a - b) > 1e-3) < 0.01


def test_mode_switch_and_errors(cuda_lib):
    from lenia_b200 import _lib
    from lenia_b200.world import World
    wl = P.config0(seed=7)
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    w.set_conv_mode("DIRECT_BF16")
    w.step(2)
    w.set_conv_mode("FFT")
    assert w.conv_macs() == (0.0, 0.0)
    w.step(1)
    w.sync()
    with pytest.raises(_lib.LeniaError):
        w._check(w._lib.lenia_set_conv_mode(w.handle, 9))
    big = [P.KernelParams(radius=70, beta_size=1, b=[1.0], r_a=1.0, m=0.2, s=0.05, h=0.5, c0=0, c1=0)]
    desc = P.WorldDesc(width=32, height=32, channels=1, growth_type=P.GROWTH_RT, mode_type=P.MODE_RT)
    w2 = World(desc, big)
    st = w2._lib.lenia_set_conv_mode(w2.handle, _lib.CONV["DIRECT_BF16"])
    assert st == 7  # LENIA_ERR_UNSUPPORTED: radius * r_a above 64
    assert w2.conv_mode == "FFT"


@pytest.mark.parametrize("shape", [(32, 32), (40, 24)])
def test_autotune_keeps_state_and_picks_fastest(cuda_lib, shape):
    """The autotuner times FFT (every row tile of the runtime-sized kernels
    for a non-cubic grid) against BF16X3 and keeps the fastest; the grid state
    is untouched and a tuned FFT world steps bit-identically to an untuned
    one."""
    from lenia_b200.world import World
    w_, h_ = shape
    wl = P.config0(seed=8, width=w_)
    wl.desc.height = h_
    wl.A0 = P.seed_cube(np.random.default_rng(8), wl.desc, min(w_, h_) // 2)
    a, b = World(wl.desc, wl.kernels), World(wl.desc, wl.kernels)
    for w in (a, b):
        w.set_state(wl.A0.ravel())
        w.step(2)
    before = {n: a.get(n).copy() for n in ("A", "V", "GA", "SUM")}
    r = a.autotune()
    print(shape, r)
    ms = {k: v for k, v in r["ms"].items() if v is not None}
    assert set(ms) == {"FFT", "DIRECT_BF16X3"}
    assert r["conv_mode"] == min(ms, key=ms.get) and a.conv_mode == r["conv_mode"]
    for n, v in before.items():
        assert np.array_equal(a.get(n).view(np.uint32), v.view(np.uint32)), n
    if r["conv_mode"] == "FFT":
        a.step(3)
        b.step(3)
        for n in ("A", "V", "GA", "SUM"):
            assert np.array_equal(a.get(n).view(np.uint32), b.get(n).view(np.uint32)), n
    with pytest.raises(Exception):
        a.autotune(modes=())


@pytest.mark.parametrize("shape", [(32, 32), (40, 24), (96, 96)])
def test_split_growth_is_bit_identical(cuda_lib, shape):
    """The growth stage as two passes (inverse rows storing u_k, then the
    growth from u_k) gives the fused pass's fields bit for bit."""
    from lenia_b200.world import World
    w_, h_ = shape
    wl = P.config0(seed=16, width=w_)
    wl.desc.height = h_
    wl.A0 = P.seed_cube(np.random.default_rng(16), wl.desc, min(w_, h_) // 2)
    a, b = World(wl.desc, wl.kernels), World(wl.desc, wl.kernels)
    b.set_tuning(0, True)
    for w in (a, b):
        w.set_debug(True)
        w.set_state(wl.A0.ravel())
        w.step(3)
        w.sync()
    for n in ("A", "V", "GA", "SUM", "H", "U_SUM", "BACK", "U"):
        assert np.array_equal(a.get(n).view(np.uint32), b.get(n).view(np.uint32)), n
