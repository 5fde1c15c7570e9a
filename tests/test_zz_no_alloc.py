"""The allocation-free convolution entry point, lenia_convolve_noalloc.

It exists for callers that cannot allocate device memory (an embedding
application that has reserved the memory it may use, or a loop that must not
take the synchronisation an allocation can cause); it keeps its intermediate
buffers in one fixed device array.  Its result must equal, bit for bit, the u
that a world's growth stage computes for the same field and kernel, on two
calls in a row (the fixed array keeps the previous call's contents)."""
import ctypes

import numpy as np
import pytest

from lenia_b200 import _lib
from lenia_b200 import params as P

pytestmark = pytest.mark.gpu


def world_u(desc, kernel, A):
    from lenia_b200.world import World
    w = World(desc, [kernel])
    w.set_debug(True)
    w.set_state(A)
    w.stage("GROWTH")
    w.sync()
    u = w.get("U")
    w.close()
    return u


@pytest.mark.parametrize("width,height,seed", [(32, 32, 3), (64, 64, 4), (48, 48, 5), (48, 32, 6), (40, 64, 7)])
def test_noalloc_matches_growth_stage(cuda_lib, width, height, seed):
    import torch
    rng = np.random.default_rng(seed)
    desc = P.WorldDesc(width=width, height=height, channels=1, asymptotic=(False,) * 4)
    kernel = P.sample_kernels(rng, 1, radius=min(width, height) // 4)[0]
    A = P.seed_cube(rng, desc, min(width, height) // 2).ravel()
    want = world_u(desc, kernel, A)
    field = torch.from_numpy(A).cuda()
    out = torch.empty_like(field)
    ck = _lib.to_c_kernels([kernel])
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out.fill_(float("nan"))
        st = cuda_lib.lenia_convolve_noalloc(width, height, ctypes.c_void_p(field.data_ptr()), ck,
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        torch.cuda.synchronize()
        assert st == 0, f"call {call}: status {st}"
        got = out.cpu().numpy()
        assert np.array_equal(got, want), f"call {call}: {int((got != want).sum())} values differ"


def test_noalloc_rejects_grids_past_its_fixed_space(cuda_lib):
    import torch
    field = torch.zeros(128 ** 3, device="cuda")
    out = torch.zeros_like(field)
    ck = _lib.to_c_kernels([P.KernelParams(radius=4)])
    st = cuda_lib.lenia_convolve_noalloc(128, 128, ctypes.c_void_p(field.data_ptr()), ck,
                                         ctypes.c_void_p(out.data_ptr()), None)
    assert st == 1  # LENIA_ERR_INVALID_ARG
