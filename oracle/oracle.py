"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use it; the product never does).

ctypes front end for the two CPU oracles built by oracle/Makefile:

* `RefOracle`     — oracle/_ref/libleniaref.so: the reference's own
  lenia.cpp, reintegration.cpp, transposition.cpp and mesh.cpp compiled
  unmodified against shim headers, stepped by oracle/refshim/driver.cpp.
  Its grid is render.h's compile-time 32x32x32 with at most 12 kernels;
  `RefOracle(..., lib=REF_LIB_128)` is the same code built at 128^3 with at
  most 16 kernels (one instance per library per process: its state is
  the library's globals).
* `RestateOracle` — oracle/_build/liblenia_oracle.so: the C restatement
  (oracle/restate/lenia_oracle.c), any size.  fft_mode "c2c" follows the
  reference's complex-to-complex spectral structure; "half" follows the CUDA
  library's half-spectrum convolution.

Parameters are plain dicts whose keys are the fields of `ora_params` /
`ora_kernel` (oracle/restate/oracle_api.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libleniaref.so")
# The same sources built at the headline size (128^3, at most 16 kernels).
REF_LIB_128 = os.path.join(HERE, "_ref", "w128", "libleniaref.so")
# The 32^3 build linked with a float64 FFT stand-in (refshim/fftw_shim64.c):
# a second valid build of the reference, for its sensitivity to FFT rounding.
REF_LIB_FFT64 = os.path.join(HERE, "_ref", "fft64", "libleniaref.so")
ORACLE_LIB = os.path.join(HERE, "_build", "liblenia_oracle.so")

FIELDS = {
    "A": 0, "V": 1, "GA": 2, "SUM": 3, "H": 4, "U_SUM": 5, "BACK": 6, "NA": 7, "NU": 8,
    "PREALPHA": 9, "ALPHA": 10, "F": 11, "MU": 12, "TT": 13, "U_S": 14, "SUM_S": 15,
    "U": 16, "H_RB": 17, "U_SUM_RB": 18, "RBB": 19,
}
EVENTS = ["FFT", "FFT_MT", "BLUR", "TSB", "SOBEL_ONE", "SOBEL_TWO", "F", "MU", "TB",
          "REINTEGRATION", "TRM", "TMB"]


class OraParams(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("channels", ctypes.c_int),
        ("timestep", ctypes.c_float), ("theta_a", ctypes.c_float), ("n_alpha", ctypes.c_float),
        ("s_norm", ctypes.c_float), ("gta", ctypes.c_float), ("sta", ctypes.c_float),
        ("v_damp", ctypes.c_float), ("v_beta", ctypes.c_float), ("iso_value", ctypes.c_float),
        ("sigma", ctypes.c_float), ("dd", ctypes.c_float),
        ("alpha_mode", ctypes.c_int), ("growth_type", ctypes.c_int), ("mode_type", ctypes.c_int),
        ("sobel_border", ctypes.c_int), ("border", ctypes.c_int), ("gradient_mode", ctypes.c_int),
        ("adv_vel", ctypes.c_int), ("mu_vel", ctypes.c_int), ("blur_central_diff", ctypes.c_int),
        ("osc_la", ctypes.c_int), ("osc_flow", ctypes.c_int), ("osc_div_flow", ctypes.c_int),
        ("osc_vel", ctypes.c_int),
        ("osc_la_amt", ctypes.c_float), ("osc_flow_amt", ctypes.c_float),
        ("osc_div_flow_amt", ctypes.c_float),
        ("asymptotic", ctypes.c_int * 4), ("soft_clip", ctypes.c_int * 4),
        ("rt_all_channels", ctypes.c_int), ("alpha_index_fix", ctypes.c_int), ("exact_bell", ctypes.c_int),
    ]


class OraKernel(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_int), ("beta_size", ctypes.c_int), ("b", ctypes.c_float * 12),
        ("r_a", ctypes.c_float), ("m", ctypes.c_float), ("s", ctypes.c_float),
        ("h", ctypes.c_float), ("c0", ctypes.c_int), ("c1", ctypes.c_int),
    ]


def make_params(d: dict) -> OraParams:
    p = OraParams()
    for name, ctype in OraParams._fields_:
        v = d.get(name, 0)
        if name in ("asymptotic", "soft_clip"):
            arr = (ctypes.c_int * 4)(*[int(bool(x)) for x in (list(v) + [0] * 4)[:4]])
            setattr(p, name, arr)
        elif ctype is ctypes.c_int:
            setattr(p, name, int(v))
        else:
            setattr(p, name, float(np.float32(v)))
    return p


def make_kernels(ks) -> ctypes.Array:
    arr = (OraKernel * max(len(ks), 1))()
    for i, k in enumerate(ks):
        arr[i].radius = int(k["radius"])
        arr[i].beta_size = int(k["beta_size"])
        b = (list(k["b"]) + [0.0] * 12)[:12]
        for j in range(12):
            arr[i].b[j] = float(np.float32(b[j]))
        for name in ("r_a", "m", "s", "h"):
            setattr(arr[i], name, float(np.float32(k[name])))
        arr[i].c0 = int(k["c0"])
        arr[i].c1 = int(k["c1"])
    return arr


_build_lock = threading.Lock()

# Directory of the reference's sources (the project's checkout); tests read
# marching_cubes.h and lenia.cpp there, and oracle/Makefile builds from it.
REF_DIR = os.environ.get("LENIA_REFERENCE", "/root/reference")


def ref_path(name: str) -> str:
    """Path of a file of the reference's sources."""
    return os.path.join(REF_DIR, name)


def build(force: bool = False) -> None:
    """Builds both oracles with oracle/Makefile (the reference build only when
    the reference sources are present on this machine)."""
    with _build_lock:
        if force or not os.path.exists(ORACLE_LIB) or (
                os.path.isdir(REF_DIR) and not os.path.exists(REF_LIB)):
            subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_DIR}"], check=True)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _opt(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


class _Base:
    C: int
    N: int
    K: int

    def field_size(self, name: str) -> int:
        n, c, k = self.N, self.C, self.K
        return {"V": 3 * c * n, "NA": 3 * n, "NU": 3 * c * n, "F": 3 * c * n, "MU": 3 * c * n,
                "SUM": n, "SUM_S": n, "U": k * n}.get(name, c * n)


class RefOracle(_Base):
    """The reference's own code at its compile-time size (32^3, <=12 kernels,
    or 128^3, <=16 kernels with lib=REF_LIB_128)."""

    _libs: dict = {}

    @classmethod
    def lib(cls, path: str = REF_LIB):
        if path not in cls._libs:
            build()
            if not os.path.exists(path):
                raise FileNotFoundError(path)
            lib = ctypes.CDLL(path)
            lib.ref_init()
            lib.ref_get_field.restype = ctypes.c_int
            lib.ref_bell_lut.restype = ctypes.c_float
            lib.ref_bell_lut.argtypes = [ctypes.c_int] * 3
            cls._libs[path] = lib
        return cls._libs[path]

    def __init__(self, params: dict, kernels: list, lib: str = REF_LIB):
        self._path = lib
        lib = self.lib(lib)
        self.W = lib.ref_grid_width()
        self.Hh = lib.ref_grid_height()
        assert params["width"] == self.W and params["height"] == self.Hh, \
            f"this reference build is {self.W}x{self.Hh}x{self.W}"
        self.C = params["channels"]
        self.K = len(kernels)
        self.N = self.W * self.Hh * self.W
        self.params = params
        lib.ref_set_params(ctypes.byref(make_params(params)))
        if lib.ref_set_kernels(make_kernels(kernels), self.K) != 0:
            raise ValueError("too many kernels for the reference build")

    def set_state(self, A=None, V=None, GA=None, SUM=None):
        A, V, GA, SUM = (_opt(x) for x in (A, V, GA, SUM))
        self.lib(self._path).ref_set_state(*(None if x is None else _fp(x) for x in (A, V, GA, SUM)))

    def run_event(self, ev):
        self.lib(self._path).ref_run_event(EVENTS.index(ev) if isinstance(ev, str) else int(ev))

    def step(self, n=1, slab_threads: bool = False):
        """n steps; slab_threads runs each event's two slabs on two threads
        at once (the reference's two sim threads), else one after the other."""
        if slab_threads:
            self.lib(self._path).ref_step_slabs(int(n))
        else:
            self.lib(self._path).ref_step(int(n))

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.field_size(name), dtype=np.float32)
        self.lib(self._path).ref_get_field(FIELDS[name], _fp(out))
        return out

    def kernel_grid(self, k):
        out = np.zeros(self.N, dtype=np.float32)
        self.lib(self._path).ref_get_kernel_grid(int(k), _fp(out))
        return out

    def blur_grid(self):
        out = np.zeros(self.N, dtype=np.float32)
        self.lib(self._path).ref_get_blur_grid(_fp(out))
        return out

    def kernel_spectrum(self, k):
        out = np.zeros(2 * self.N, dtype=np.float32)
        self.lib(self._path).ref_get_kernel_spectrum(int(k), _fp(out))
        return out

    def bell_lut(self, m, s, u):
        return self.lib(self._path).ref_bell_lut(m, s, u)


class RestateOracle(_Base):
    """The C restatement, any grid size."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            build()
            lib = ctypes.CDLL(ORACLE_LIB)
            lib.ora_create.restype = ctypes.c_void_p
            lib.ora_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
            for fn in ("ora_destroy", "ora_set_state", "ora_run_event", "ora_step", "ora_get_field",
                       "ora_set_field", "ora_get_kernel_grid", "ora_get_kernel_hat",
                       "ora_get_lut_row", "ora_hs_forward", "ora_set_params",
                       "ora_get_kernel_spectrum", "ora_get_blur_grid"):
                getattr(lib, fn).argtypes = None
            lib.ora_get_field.restype = ctypes.c_long
            lib.ora_set_field.restype = ctypes.c_long
            lib.ora_get_kernel_hat.restype = ctypes.c_long
            lib.ora_get_kernel_spectrum.restype = ctypes.c_long
            lib.ora_bell_lut.restype = ctypes.c_float
            lib.ora_bell_lut.argtypes = [ctypes.c_int] * 3
            lib.ora_lfft_factor.restype = ctypes.c_int
            cls._lib = lib
        return cls._lib

    def __init__(self, params: dict, kernels: list, fft_mode: str = "half"):
        lib = self.lib()
        self.params = params
        self.W = params["width"]
        self.Hh = params["height"]
        self.C = params["channels"]
        self.K = len(kernels)
        self.N = self.W * self.Hh * self.W
        self._p = make_params(params)
        self._k = make_kernels(kernels)
        mode = {"c2c": 0, "half": 1}[fft_mode]
        self.h = lib.ora_create(ctypes.byref(self._p), self._k, self.K, mode)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib().ora_destroy(ctypes.c_void_p(h))
            self.h = None

    def set_params(self, params: dict):
        self._p = make_params(params)
        self.lib().ora_set_params(ctypes.c_void_p(self.h), ctypes.byref(self._p))

    def set_state(self, A=None, V=None, GA=None, SUM=None):
        A, V, GA, SUM = (_opt(x) for x in (A, V, GA, SUM))
        self.lib().ora_set_state(ctypes.c_void_p(self.h),
                                 *(None if x is None else _fp(x) for x in (A, V, GA, SUM)))

    def run_event(self, ev):
        self.lib().ora_run_event(ctypes.c_void_p(self.h),
                                 EVENTS.index(ev) if isinstance(ev, str) else int(ev))

    def step(self, n=1):
        self.lib().ora_step(ctypes.c_void_p(self.h), int(n))

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.field_size(name), dtype=np.float32)
        self.lib().ora_get_field(ctypes.c_void_p(self.h), FIELDS[name], _fp(out))
        return out

    def set(self, name: str, value: np.ndarray):
        v = np.ascontiguousarray(value, dtype=np.float32).ravel()
        assert v.size == self.field_size(name), (name, v.size)
        self.lib().ora_set_field(ctypes.c_void_p(self.h), FIELDS[name], _fp(v))

    def kernel_grid(self, k):
        out = np.zeros(self.N, dtype=np.float32)
        self.lib().ora_get_kernel_grid(ctypes.c_void_p(self.h), int(k), _fp(out))
        return out

    def blur_grid(self):
        out = np.zeros(self.N, dtype=np.float32)
        self.lib().ora_get_blur_grid(ctypes.c_void_p(self.h), _fp(out))
        return out

    def kernel_hat(self, k):
        KH = (self.W // 2 + 1) * (self.W // 2 + 1) * (self.Hh // 2 + 1)
        out = np.zeros(KH, dtype=np.float32)
        self.lib().ora_get_kernel_hat(ctypes.c_void_p(self.h), int(k), _fp(out))
        return out

    def kernel_spectrum(self, k):
        out = np.zeros(2 * self.N, dtype=np.float32)
        self.lib().ora_get_kernel_spectrum(ctypes.c_void_p(self.h), int(k), _fp(out))
        return out

    def lut_row(self, k):
        out = np.zeros(256, dtype=np.float32)
        self.lib().ora_get_lut_row(ctypes.c_void_p(self.h), int(k), _fp(out))
        return out

    def hs_forward(self, fa, fb=None):
        HS = (self.W // 2 + 1) * self.W * self.Hh
        fa = np.ascontiguousarray(fa, dtype=np.float32)
        oa = np.zeros(2 * HS, dtype=np.float32)
        ob = np.zeros(2 * HS, dtype=np.float32) if fb is not None else None
        fbp = None
        if fb is not None:
            fb = np.ascontiguousarray(fb, dtype=np.float32)
            fbp = _fp(fb)
        self.lib().ora_hs_forward(ctypes.c_void_p(self.h), _fp(fa), fbp, _fp(oa),
                                  None if ob is None else _fp(ob))
        return oa.view(np.complex64), (None if ob is None else ob.view(np.complex64))

    @classmethod
    def lfft_1d(cls, x: np.ndarray, sign: int) -> np.ndarray:
        y = np.ascontiguousarray(x, dtype=np.complex64).copy()
        cls.lib().ora_lfft_1d(y.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                              ctypes.c_int(y.size), ctypes.c_int(sign))
        return y

    @classmethod
    def bell_lut(cls, m, s, u):
        return cls.lib().ora_bell_lut(m, s, u)


class Mesh:
    """A marching-cubes mesh as flat arrays: positions and normals (V x 3
    float32), vertex channel (V int32, None from the reference build), indices
    (3T uint32) and the case index of every cube (C x N uint8, or None)."""

    def __init__(self, positions, normals, indices, vertex_channel=None, cases=None):
        self.positions = positions
        self.normals = normals
        self.indices = indices
        self.vertex_channel = vertex_channel
        self.cases = cases

    @property
    def n_vertices(self):
        return self.positions.shape[0]

    @property
    def n_triangles(self):
        return self.indices.size // 3


def mc_table(kind: str = "own") -> np.ndarray:
    """256 x 16 triangle table (edge indices, -1 terminated).  "own" is the
    restatement's table built from geometry (oracle/restate/mc_tables.c)."""
    assert kind == "own"
    lib = RestateOracle.lib()
    t = np.zeros(256 * 16, dtype=np.int32)
    lib.mc_own_table(t.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return t.reshape(256, 16)


def mesh_restated(fields, W: int, H: int, C: int, iso: float, cell: float = 3.5, offsets=None,
                  table: np.ndarray | None = None, slabs: int = 1, share_channels: bool = False,
                  halos=None, quirks: bool = False) -> Mesh:
    """Marching cubes of one C-channel field, or of a list of fields meshed
    together (the U/H views), by the restatement of generate_mesh_v1/v2/v3
    (ora_mesh_fields in oracle/restate/mc_tables.c).  offsets: one (x, y, z)
    per field added after interpolation; halos: per field the array its +1
    faces copy (None: the field); quirks: the reference's stale normal slots
    of fields 1 and 2 (then `unsure` flags vertices that read a slot never
    written)."""
    lib = RestateOracle.lib()
    if isinstance(fields, np.ndarray):
        fields = [fields]
    N = W * H * W
    fl = [np.ascontiguousarray(f, dtype=np.float32).ravel() for f in fields]
    assert all(f.size >= C * N for f in fl)
    F = len(fl)
    FP = ctypes.POINTER(ctypes.c_float)
    ptrs = (FP * F)(*[_fp(f) for f in fl])
    hptrs = None
    if halos is not None:
        hl = [None if h is None else np.ascontiguousarray(h, dtype=np.float32).ravel() for h in halos]
        hptrs = (FP * F)(*[_fp(h) if h is not None else FP() for h in hl])
    off = None
    if offsets is not None:
        off = np.ascontiguousarray(offsets, dtype=np.float32).reshape(F, 3)
    tab = None
    if table is not None:
        tab = np.ascontiguousarray(table, dtype=np.int32).ravel()
        assert tab.size == 256 * 16
    cases = np.zeros(F * C * N, dtype=np.uint8)
    cap_v = cap_i = 1024
    while True:
        pos = np.zeros(3 * cap_v, dtype=np.float32)
        nrm = np.zeros(3 * cap_v, dtype=np.float32)
        vch = np.zeros(cap_v, dtype=np.int32)
        unsure = np.zeros(cap_v, dtype=np.uint8)
        idx = np.zeros(cap_i, dtype=np.uint32)
        fn = np.zeros(cap_i, dtype=np.float32)
        nv, ni = ctypes.c_long(0), ctypes.c_long(0)
        rc = lib.ora_mesh_fields(ptrs, hptrs, ctypes.c_int(F), None if off is None else _fp(off),
                                 ctypes.c_int(W), ctypes.c_int(H), ctypes.c_int(C), ctypes.c_float(iso),
                                 ctypes.c_float(cell),
                                 None if tab is None else tab.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 ctypes.c_int(slabs), ctypes.c_int(1 if share_channels else 0),
                                 ctypes.c_int(1 if quirks else 0),
                                 cases.ctypes.data_as(ctypes.c_void_p), _fp(pos), _fp(nrm),
                                 vch.ctypes.data_as(ctypes.c_void_p), unsure.ctypes.data_as(ctypes.c_void_p),
                                 ctypes.c_long(cap_v), idx.ctypes.data_as(ctypes.c_void_p), _fp(fn),
                                 ctypes.c_long(cap_i), ctypes.byref(nv), ctypes.byref(ni))
        if rc == 0:
            break
        cap_v, cap_i = max(nv.value, 1), max(ni.value, 1)
    m = Mesh(pos[:3 * nv.value].reshape(-1, 3), nrm[:3 * nv.value].reshape(-1, 3), idx[:ni.value],
             vch[:nv.value], cases.reshape(F, C, N))
    m.face_normals = fn[:ni.value].reshape(-1, 3)
    m.unsure = unsure[:nv.value].astype(bool)
    return m


def mesh_reference(ref: "RefOracle", view: int = 0) -> Mesh:
    """The reference's own generate_mesh_v1 (view 0), v2 (1) or v3 (2) on its
    RBB / U_SUM_RB / H_RB snapshots (run a step, or the TMB event, first),
    both mesh threads concatenated, without stitching."""
    lib = ref.lib()
    cap_v = cap_i = 1024
    while True:
        pos = np.zeros(3 * cap_v, dtype=np.float32)
        nrm = np.zeros(3 * cap_v, dtype=np.float32)
        idx = np.zeros(cap_i, dtype=np.uint32)
        nv, ni = ctypes.c_long(0), ctypes.c_long(0)
        rc = lib.ref_mesh(ctypes.c_int(view), _fp(pos), _fp(nrm), ctypes.c_long(cap_v),
                          idx.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(cap_i), ctypes.byref(nv),
                          ctypes.byref(ni))
        if rc == 0:
            break
        cap_v, cap_i = max(nv.value, 1), max(ni.value, 1)
    return Mesh(pos[:3 * nv.value].reshape(-1, 3), nrm[:3 * nv.value].reshape(-1, 3), idx[:ni.value])
