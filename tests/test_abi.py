"""The C-ABI library: it loads, exports every entry point include/lenia_b200.h
declares, its structs match the header, and it refuses to run without a GPU
(no CPU fallback)."""
import ctypes
import os
import re

import pytest

from conftest import have_gpu
from lenia_b200 import _lib, params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(cuda_lib):
    declared = _lib.exported_symbols()
    assert "lenia_create" in declared and "lenia_step" in declared
    missing = [s for s in declared if not hasattr(cuda_lib, s)]
    assert not missing, missing


def test_struct_layout_matches_header():
    hdr = open(os.path.join(ROOT, "include", "lenia_b200.h")).read()
    body = re.search(r"typedef struct LeniaWorldDesc \{(.*?)\} LeniaWorldDesc;", hdr, re.S).group(1)
    names = re.findall(r"^\s*(?:int|float)\s+(\w+)", body, re.M)
    assert names == [n for n, _ in _lib.LeniaWorldDesc._fields_]
    body = re.search(r"typedef struct LeniaKernelParams \{(.*?)\} LeniaKernelParams;", hdr, re.S).group(1)
    names = re.findall(r"^\s*(?:int|float)\s+(\w+)", body, re.M)
    assert names == [n for n, _ in _lib.LeniaKernelParams._fields_]


def test_version(cuda_lib):
    assert b"sm_100a" in cuda_lib.lenia_version()


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_no_cpu_fallback(cuda_lib):
    wl = P.config0()
    h = ctypes.c_void_p()
    st = cuda_lib.lenia_create(ctypes.byref(_lib.to_c_desc(wl.desc)), _lib.to_c_kernels(wl.kernels),
                               len(wl.kernels), ctypes.byref(h))
    assert st == 6  # LENIA_ERR_NO_DEVICE


def test_params_mirror_reference_defaults():
    d = P.WorldDesc()
    # main.cpp:31-56 and main.cpp:304
    assert (d.gta, d.sta, d.v_damp, d.timestep, d.theta_a, d.sigma, d.dd) == (0.1, 0.1, 0.9, 0.1, 1.0, 0.5, 1.0)
    assert (d.growth_type, d.mode_type, d.gradient_mode, d.border) == (
        P.GROWTH_RT, P.MODE_SRT, P.GRADIENT_SOBEL, P.BORDER_NONE)
