"""Batches of independent worlds over the C ABI (lenia_batch_*), and the
partition of a batch across GPUs.

`Batch` steps many worlds of mixed sizes, channels, kernel sets and modes
with one CUDA-graph launch per step (inside it, batched launches that each
cover many worlds through device work lists, and per-world launches for the
worlds those do not take); each world's fields are bit-identical to those of
a `World` stepped alone.  `shard_worlds` splits a batch across
ranks (one process per GPU): worlds are independent, so the ranks exchange
nothing while stepping.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import numpy as np

from . import _lib
from .params import KernelParams, WorldDesc


def world_cost(desc: WorldDesc, n_kernels: int) -> int:
    """Work of one step of a world, in cell-channel-transforms (used to
    balance lanes and ranks)."""
    return desc.width * desc.height * desc.width * desc.channels * (1 + n_kernels)


def shard_worlds(costs: Sequence[int], world_size: int) -> List[List[int]]:
    """Longest-processing-time partition: worlds sorted by cost (ties by
    index), each to the rank with the least total so far (ties to the lowest
    rank).  Every rank computes the same partition from the same costs."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world_size
    parts: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


class Batch:
    def __init__(self, descs: Sequence[WorldDesc], kernel_sets: Sequence[Sequence[KernelParams]], lanes: int = 0):
        assert len(descs) == len(kernel_sets) and len(descs) > 0
        self._lib = _lib.load()
        self.descs = list(descs)
        self.kernel_sets = [list(k) for k in kernel_sets]
        n = len(descs)
        cd = (_lib.LeniaWorldDesc * n)(*[_lib.to_c_desc(d) for d in descs])
        allk = [k for ks in self.kernel_sets for k in ks]
        ck = _lib.to_c_kernels(allk)
        counts = (ctypes.c_int * n)(*[len(ks) for ks in self.kernel_sets])
        h = ctypes.c_void_p()
        st = self._lib.lenia_batch_create(cd, ck, counts, n, int(lanes), ctypes.byref(h))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, "lenia_batch_create failed")
        self._h = h

    def __len__(self) -> int:
        return len(self.descs)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lenia_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, self._lib.lenia_batch_last_error(self._h).decode())

    def field_size(self, i: int, name: str) -> int:
        d = self.descs[i]
        n = d.width * d.height * d.width
        return {"A": d.channels * n, "V": 3 * d.channels * n, "GA": d.channels * n, "SUM": n}[name]

    def set(self, i: int, name: str, value) -> None:
        a = np.ascontiguousarray(value, dtype=np.float32).ravel()
        self._check(self._lib.lenia_batch_set_field(self._h, i, _lib.FIELD[name], a.ctypes.data_as(ctypes.c_void_p),
                                                    a.size, 0))

    def set_state(self, i: int, A, V=None, GA=None, SUM=None) -> None:
        self.set(i, "A", A)
        for name, v in (("V", V), ("GA", GA), ("SUM", SUM)):
            self.set(i, name, np.zeros(self.field_size(i, name), np.float32) if v is None else v)

    def get(self, i: int, name: str) -> np.ndarray:
        out = np.zeros(self.field_size(i, name), dtype=np.float32)
        self._check(self._lib.lenia_batch_get_field(self._h, i, _lib.FIELD[name],
                                                    out.ctypes.data_as(ctypes.c_void_p), out.size, 0))
        return out

    def step(self, n: int = 1) -> None:
        self._check(self._lib.lenia_batch_step(self._h, int(n)))

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self._lib.lenia_batch_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def sync(self) -> None:
        self._check(self._lib.lenia_batch_sync(self._h))

    def autotune(self, modes=("FFT", "DIRECT_BF16X3")) -> List[dict]:
        """lenia_batch_autotune: per grid shape, the convolution mode and FFT
        row tile that time fastest on its first world, applied to every world
        of that shape; returns each world's choice."""
        mask = 0
        for m in modes:
            mask |= 1 << _lib.CONV[m]
        n = len(self.descs)
        res = (_lib.LeniaTuneResult * n)()
        self._check(self._lib.lenia_batch_autotune(self._h, mask, res))
        names = {v: k for k, v in _lib.CONV.items()}
        return [{"conv_mode": names[r.conv_mode], "row_tile": r.row_tile, "growth_split": bool(r.growth_split),
                 "ms": {names[i]: (float(r.ms[i]) if r.ms[i] >= 0 else None) for i in range(3)}} for r in res]

    def stats(self, fill_threshold: float = 0.1) -> List[np.ndarray]:
        """Grid statistics of every world (channels x 9 doubles each)."""
        total = sum(d.channels for d in self.descs) * 9
        out = np.zeros(total, dtype=np.float64)
        self._check(self._lib.lenia_batch_stats(self._h, ctypes.c_float(fill_threshold),
                                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        res, off = [], 0
        for d in self.descs:
            res.append(out[off:off + 9 * d.channels].reshape(d.channels, 9))
            off += 9 * d.channels
        return res

    def launches_per_step(self) -> int:
        return int(self._lib.lenia_batch_launches_per_step(self._h))

    def set_batched_launches(self, on: bool = True) -> None:
        """Batched launches (one per stage and grid size over the worlds that
        qualify) on or off; off steps every world through its own launches.
        The fields are the same either way."""
        self._check(self._lib.lenia_batch_set_batched_launches(self._h, 1 if on else 0))

    def grouped_worlds(self) -> int:
        """Worlds stepped by the batched launches."""
        return int(self._lib.lenia_batch_grouped_worlds(self._h))
