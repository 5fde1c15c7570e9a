"""ctypes binding of the C ABI declared in include/lenia_b200.h.

The shared library is lenia_b200/liblenia_b200.so, built in-tree by
lenia_b200/build.py.  There is no fallback: if the library is missing the
import of the binding raises.
"""
from __future__ import annotations

import ctypes
import os

from .params import KernelParams, WorldDesc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblenia_b200.so")

MAX_CHANNELS = 4
MAX_BETA = 12

LENIA_OK = 0
LENIA_ERR_INVALID_ARG = 1
LENIA_ERR_OOM = 2
LENIA_ERR_CUDA = 3
LENIA_ERR_TIMEOUT = 4
LENIA_ERR_NONFINITE = 5
LENIA_ERR_NO_DEVICE = 6
LENIA_ERR_UNSUPPORTED = 7
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "NONFINITE",
                6: "NO_DEVICE", 7: "UNSUPPORTED"}

FIELD = {
    "A": 0, "V": 1, "GA": 2, "SUM": 3, "H": 4, "U_SUM": 5, "BACK": 6, "NA": 7, "NU": 8,
    "PREALPHA": 9, "ALPHA": 10, "F": 11, "MU": 12, "TT": 13, "U_S": 14, "SUM_S": 15,
    "U": 16, "H_RB": 17, "U_SUM_RB": 18, "RBB": 19,
}
STAGE = {"GROWTH": 0, "BLUR": 1, "FLOW": 2, "TRANSPORT": 3, "SNAPSHOT": 4}
CONV = {"FFT": 0, "DIRECT_BF16": 1, "DIRECT_BF16X3": 2}


class LeniaTuneResult(ctypes.Structure):
    _fields_ = [("conv_mode", ctypes.c_int), ("row_tile", ctypes.c_int), ("ms", ctypes.c_float * 3),
                ("growth_split", ctypes.c_int)]


class LeniaWorldDesc(ctypes.Structure):
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
        ("asymptotic", ctypes.c_int * MAX_CHANNELS), ("soft_clip", ctypes.c_int * MAX_CHANNELS),
        ("rt_all_channels", ctypes.c_int), ("alpha_index_fix", ctypes.c_int), ("exact_bell", ctypes.c_int),
        ("conserve_mass", ctypes.c_int),
    ]


class LeniaKernelParams(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_int), ("beta_size", ctypes.c_int), ("b", ctypes.c_float * MAX_BETA),
        ("r_a", ctypes.c_float), ("m", ctypes.c_float), ("s", ctypes.c_float),
        ("h", ctypes.c_float), ("c0", ctypes.c_int), ("c1", ctypes.c_int),
    ]


class LeniaMeshDesc(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("channels", ctypes.c_int),
        ("fields", ctypes.c_int), ("iso_value", ctypes.c_float), ("cell_size", ctypes.c_float),
        ("offset", (ctypes.c_float * 3) * 3), ("slabs", ctypes.c_int), ("share_channels", ctypes.c_int),
    ]


VIEW = {"NORMAL": 0, "U": 1, "H": 2}
MESH_ARRAY = {"positions": 0, "normals": 1, "vertex_channel": 2, "indices": 3, "face_normals": 4, "cases": 5}


def to_c_desc(desc: WorldDesc) -> LeniaWorldDesc:
    d = desc.as_dict()
    c = LeniaWorldDesc()
    for name, ctype in LeniaWorldDesc._fields_:
        v = d[name]
        if name in ("asymptotic", "soft_clip"):
            setattr(c, name, (ctypes.c_int * MAX_CHANNELS)(*[int(x) for x in v]))
        elif ctype is ctypes.c_int:
            setattr(c, name, int(v))
        else:
            setattr(c, name, float(v))
    return c


def to_c_kernels(kernels: list[KernelParams]):
    arr = (LeniaKernelParams * max(len(kernels), 1))()
    for i, k in enumerate(kernels):
        d = k.as_dict()
        arr[i].radius = int(d["radius"])
        arr[i].beta_size = int(d["beta_size"])
        for j in range(MAX_BETA):
            arr[i].b[j] = float(d["b"][j])
        for name in ("r_a", "m", "s", "h"):
            setattr(arr[i], name, float(d[name]))
        arr[i].c0 = int(d["c0"])
        arr[i].c1 = int(d["c1"])
    return arr


_lib = None


def load() -> ctypes.CDLL:
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python lenia_b200/build.py` (needs nvcc)")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    sigs = {
        "lenia_create": ([ctypes.POINTER(LeniaWorldDesc), ctypes.POINTER(LeniaKernelParams), ctypes.c_int,
                          ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
        "lenia_destroy": ([P], ctypes.c_int),
        "lenia_set_params": ([P, ctypes.POINTER(LeniaWorldDesc)], ctypes.c_int),
        "lenia_set_kernels": ([P, ctypes.POINTER(LeniaKernelParams), ctypes.c_int], ctypes.c_int),
        "lenia_set_field": ([P, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int], ctypes.c_int),
        "lenia_get_field": ([P, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int], ctypes.c_int),
        "lenia_field_size": ([P, ctypes.c_int], ctypes.c_size_t),
        "lenia_step": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_step_stage": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_set_stream": ([P, ctypes.c_void_p], ctypes.c_int),
        "lenia_sync": ([P], ctypes.c_int),
        "lenia_set_debug": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_set_wait_limit": ([P, ctypes.c_longlong], ctypes.c_int),
        "lenia_set_conv_mode": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_get_conv_mode": ([P], ctypes.c_int),
        "lenia_conv_macs": ([P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "lenia_autotune": ([P, ctypes.c_int, ctypes.POINTER(LeniaTuneResult)], ctypes.c_int),
        "lenia_set_tuning": ([P, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "lenia_set_snapshots": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_launches_per_step": ([P], ctypes.c_int),
        "lenia_set_profiling": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_profile_read": ([P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                ctypes.c_int], ctypes.c_int),
        "lenia_kernel_name": ([ctypes.c_int], ctypes.c_char_p),
        "lenia_convolve_noalloc": ([ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(LeniaKernelParams),
                                    ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
        "lenia_save": ([P, ctypes.POINTER(LeniaWorldDesc), ctypes.POINTER(LeniaKernelParams), ctypes.c_int,
                        ctypes.c_ulonglong, ctypes.c_char_p], ctypes.c_int),
        "lenia_load": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ulonglong)],
                       ctypes.c_int),
        "lenia_mlp_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_void_p)],
                             ctypes.c_int),
        "lenia_mlp_destroy": ([P], ctypes.c_int),
        "lenia_mlp_param_count": ([P], ctypes.c_longlong),
        "lenia_mlp_get_params": ([P, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
        "lenia_mlp_set_params": ([P, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
        "lenia_mlp_get_grads": ([P, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
        "lenia_mlp_forward": ([P, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
        "lenia_mlp_gradients": ([P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                 ctypes.c_void_p], ctypes.c_int),
        "lenia_mlp_train_step": ([P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                  ctypes.POINTER(ctypes.c_float), ctypes.c_void_p], ctypes.c_int),
        "lenia_mlp_last_error": ([P], ctypes.c_char_p),
        "lenia_batch_create": ([ctypes.POINTER(LeniaWorldDesc), ctypes.POINTER(LeniaKernelParams),
                                ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
        "lenia_batch_destroy": ([P], ctypes.c_int),
        "lenia_batch_size": ([P], ctypes.c_int),
        "lenia_batch_set_field": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int],
                                  ctypes.c_int),
        "lenia_batch_get_field": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int],
                                  ctypes.c_int),
        "lenia_batch_step": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_batch_set_stream": ([P, ctypes.c_void_p], ctypes.c_int),
        "lenia_batch_sync": ([P], ctypes.c_int),
        "lenia_batch_autotune": ([P, ctypes.c_int, ctypes.POINTER(LeniaTuneResult)], ctypes.c_int),
        "lenia_batch_launches_per_step": ([P], ctypes.c_int),
        "lenia_batch_set_batched_launches": ([P, ctypes.c_int], ctypes.c_int),
        "lenia_batch_grouped_worlds": ([P], ctypes.c_int),
        "lenia_world_stats": ([P, ctypes.c_float, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "lenia_batch_stats": ([P, ctypes.c_float, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "lenia_batch_last_error": ([P], ctypes.c_char_p),
        "lenia_mesher_create": ([ctypes.POINTER(LeniaMeshDesc), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
        "lenia_mesher_destroy": ([P], ctypes.c_int),
        "lenia_mesher_run": ([P, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p,
                              ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
        "lenia_mesh_desc_for_view": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.POINTER(LeniaMeshDesc)], ctypes.c_int),
        "lenia_mesher_get": ([P, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int], ctypes.c_int),
        "lenia_mesh_world": ([P, ctypes.c_int, P, ctypes.POINTER(ctypes.c_longlong),
                              ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
        "lenia_mc_triangle_table": ([ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "lenia_mesher_last_error": ([P], ctypes.c_char_p),
        "lenia_last_error": ([P], ctypes.c_char_p),
        "lenia_version": ([], ctypes.c_char_p),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    """The entry points include/lenia_b200.h declares."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "lenia_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(lenia_[a-z_0-9]+)\s*\(", text)))


class LeniaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"lenia status {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status
