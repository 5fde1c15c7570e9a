"""Host-side mirror of the reference's step API over the C ABI.

`World` owns one simulated grid on the GPU.  Its methods follow the
reference's interface for the step: the parameter globals become a
`WorldDesc`, the Kernel structs a list of `KernelParams`, the arrays are
fields (`get` / `set`), and the event sequence of render.cpp:357-604 is
`step()` (whole steps) or `stage()` (one stage group).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .params import KernelParams, WorldDesc


class World:
    def __init__(self, desc: WorldDesc, kernels: Sequence[KernelParams]):
        self._lib = _lib.load()
        self.desc = desc
        self.kernels = list(kernels)
        self._cdesc = _lib.to_c_desc(desc)
        self._ckern = _lib.to_c_kernels(self.kernels)
        h = ctypes.c_void_p()
        st = self._lib.lenia_create(ctypes.byref(self._cdesc), self._ckern, len(self.kernels), ctypes.byref(h))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, "lenia_create failed")
        self._h = h

    # -------------------------------------------------------------- helpers
    def _check(self, st: int):
        if st != _lib.LENIA_OK:
            msg = self._lib.lenia_last_error(self._h).decode()
            raise _lib.LeniaError(st, msg)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lenia_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def C(self) -> int:
        return self.desc.channels

    @property
    def N(self) -> int:
        return self.desc.cells

    def field_size(self, name: str) -> int:
        return int(self._lib.lenia_field_size(self._h, _lib.FIELD[name]))

    # --------------------------------------------------------------- fields
    def set(self, name: str, value) -> None:
        """Writes a field from a numpy array (host) or a CUDA torch tensor.
        The device copy runs on the world's stream; with a tensor this call
        first waits for the device's pending work (the tensor's producer may
        run on another stream) and returns once the copy is done."""
        n = self.field_size(name) if name not in ("U_S", "SUM_S") else None
        if hasattr(value, "is_cuda") and value.is_cuda:
            import torch
            t = value.contiguous()
            torch.cuda.synchronize(t.device)
            self._check(self._lib.lenia_set_field(self._h, _lib.FIELD[name], ctypes.c_void_p(t.data_ptr()),
                                                  t.numel(), 1))
            torch.cuda.synchronize(t.device)
            return
        a = np.ascontiguousarray(value, dtype=np.float32).ravel()
        self._check(self._lib.lenia_set_field(self._h, _lib.FIELD[name], a.ctypes.data_as(ctypes.c_void_p),
                                              a.size, 0))
        del n

    def get(self, name: str, out=None):
        """Reads a field into a new numpy array, or into `out` (numpy or CUDA
        tensor).  Into a tensor the copy runs on the world's stream and this
        call returns once it is done, so `out` is ready on any stream."""
        n = self.field_size(name)
        if n == 0:
            raise _lib.LeniaError(1, f"field {name} is not available (enable debug or snapshots)")
        if out is not None and hasattr(out, "is_cuda") and out.is_cuda:
            import torch
            self._check(self._lib.lenia_get_field(self._h, _lib.FIELD[name], ctypes.c_void_p(out.data_ptr()),
                                                  out.numel(), 1))
            torch.cuda.synchronize(out.device)
            return out
        a = np.empty(n, dtype=np.float32) if out is None else out
        self._check(self._lib.lenia_get_field(self._h, _lib.FIELD[name], a.ctypes.data_as(ctypes.c_void_p),
                                              a.size, 0))
        return a

    def set_state(self, A: np.ndarray, V: Optional[np.ndarray] = None, GA: Optional[np.ndarray] = None,
                  SUM: Optional[np.ndarray] = None) -> None:
        """A new world state (the reference's reseed: every field zero, then A)."""
        C, N = self.C, self.N
        self.set("A", A)
        self.set("V", np.zeros(3 * C * N, np.float32) if V is None else V)
        self.set("GA", np.zeros(C * N, np.float32) if GA is None else GA)
        self.set("SUM", np.zeros(N, np.float32) if SUM is None else SUM)

    # ---------------------------------------------------------------- steps
    def step(self, n: int = 1) -> None:
        self._check(self._lib.lenia_step(self._h, int(n)))

    def stage(self, name: str) -> None:
        self._check(self._lib.lenia_step_stage(self._h, _lib.STAGE[name]))

    def sync(self) -> None:
        self._check(self._lib.lenia_sync(self._h))

    def set_debug(self, on: bool = True) -> None:
        self._check(self._lib.lenia_set_debug(self._h, int(on)))

    def set_wait_limit(self, polls: int = -1) -> None:
        """Poll limit of the first wait for each tile copy in the flow and
        transport kernels (-1: the default; 0: every wait gives up at once, so
        the next sync raises a timeout error)."""
        self._check(self._lib.lenia_set_wait_limit(self._h, int(polls)))

    def set_snapshots(self, on: bool = True) -> None:
        self._check(self._lib.lenia_set_snapshots(self._h, int(on)))

    def set_conv_mode(self, mode: str) -> None:
        """'FFT' (FP32 spectral path), 'DIRECT_BF16' or 'DIRECT_BF16X3'
        (spatial convolution on the tensor cores, FP32 accumulation)."""
        self._check(self._lib.lenia_set_conv_mode(self._h, _lib.CONV[mode]))

    @property
    def conv_mode(self) -> str:
        m = int(self._lib.lenia_get_conv_mode(self._h))
        return {v: k for k, v in _lib.CONV.items()}[m]

    def conv_macs(self) -> tuple:
        """(issued, useful) tensor multiply-adds of one direct convolution."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.lenia_conv_macs(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def autotune(self, modes=("FFT", "DIRECT_BF16X3")) -> dict:
        """Times the growth stage per allowed convolution mode (and the FFT
        path's row tiles) and keeps the fastest (lenia_autotune)."""
        mask = 0
        for m in modes:
            mask |= 1 << _lib.CONV[m]
        r = _lib.LeniaTuneResult()
        self._check(self._lib.lenia_autotune(self._h, mask, ctypes.byref(r)))
        names = {v: k for k, v in _lib.CONV.items()}
        return {"conv_mode": names[r.conv_mode], "row_tile": r.row_tile, "growth_split": bool(r.growth_split),
                "ms": {names[i]: (float(r.ms[i]) if r.ms[i] >= 0 else None) for i in range(3)}}

    def set_tuning(self, row_tile: int = 0, growth_split: bool = False) -> None:
        """The FFT path's tuning (lenia_set_tuning): row tile of the
        runtime-sized row transforms and the split (two-pass) growth."""
        self._check(self._lib.lenia_set_tuning(self._h, int(row_tile), int(bool(growth_split))))

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self._lib.lenia_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def set_params(self, desc: WorldDesc) -> None:
        self._cdesc = _lib.to_c_desc(desc)
        self._check(self._lib.lenia_set_params(self._h, ctypes.byref(self._cdesc)))
        self.desc = desc

    def set_kernels(self, kernels: Sequence[KernelParams]) -> None:
        self.kernels = list(kernels)
        self._ckern = _lib.to_c_kernels(self.kernels)
        self._check(self._lib.lenia_set_kernels(self._h, self._ckern, len(self.kernels)))

    def set_profiling(self, on: bool = True) -> None:
        self._check(self._lib.lenia_set_profiling(self._h, int(on)))

    def profile_read(self) -> dict:
        """Per-kernel device time since the last read: {name: (ms, launches)}."""
        n = 32
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        k = self._lib.lenia_profile_read(self._h, ms, cnt, n)
        out = {}
        for i in range(max(k, 0)):
            name = self._lib.lenia_kernel_name(i).decode()
            if cnt[i]:
                out[name] = (float(ms[i]), int(cnt[i]))
        return out

    def save(self, path: str, step: int = 0) -> None:
        """Checkpoint (lenia_save): parameters, kernels, A, V, GA, SUM."""
        self._check(self._lib.lenia_save(self._h, ctypes.byref(self._cdesc), self._ckern, len(self.kernels),
                                         ctypes.c_ulonglong(step), path.encode()))

    @classmethod
    def load(cls, path: str):
        """(World, step) from a checkpoint written by save()."""
        from .params import KernelParams, WorldDesc
        lib = _lib.load()
        h = ctypes.c_void_p()
        step = ctypes.c_ulonglong()
        st = lib.lenia_load(path.encode(), ctypes.byref(h), ctypes.byref(step))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, f"lenia_load({path!r}) failed")
        w = cls.__new__(cls)
        w._lib = lib
        w._h = h
        hdr = read_checkpoint_header(path)
        w.desc = hdr["desc"]
        w.kernels = hdr["kernels"]
        w._cdesc = _lib.to_c_desc(w.desc)
        w._ckern = _lib.to_c_kernels(w.kernels)
        return w, int(step.value)

    def stats(self, fill_threshold: float = 0.1) -> np.ndarray:
        """Grid statistics (channels x 9 doubles, see lenia_world_stats)."""
        out = np.zeros((self.C, 9), dtype=np.float64)
        self._check(self._lib.lenia_world_stats(self._h, ctypes.c_float(fill_threshold),
                                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    @property
    def launches_per_step(self) -> int:
        return int(self._lib.lenia_launches_per_step(self._h))


def read_checkpoint_header(path: str) -> dict:
    """The parameters, kernels and step of a checkpoint file (the layout is
    documented in lenia_b200/csrc/checkpoint.cu)."""
    import struct
    from .params import KernelParams, WorldDesc
    data = open(path, "rb").read()
    if data[:8] != b"LENIACKP":
        raise ValueError(f"{path} is not a checkpoint")
    version, _flags, nwords = struct.unpack_from("<III", data, 8)
    off = 20
    raw = data[off:off + 4 * nwords]
    off += 4 * nwords
    # an older, shorter descriptor: trailing fields read as 0
    raw = raw + bytes(max(0, ctypes.sizeof(_lib.LeniaWorldDesc) - len(raw)))
    cdesc = _lib.LeniaWorldDesc.from_buffer_copy(raw)
    d = {}
    for name, ctype in _lib.LeniaWorldDesc._fields_:
        v = getattr(cdesc, name)
        d[name] = tuple(bool(x) for x in v) if name in ("asymptotic", "soft_clip") else v
    desc = WorldDesc(**{k: (bool(v) if isinstance(getattr(WorldDesc(), k), bool) else v) for k, v in d.items()})
    (nk,) = struct.unpack_from("<I", data, off)
    off += 4
    kernels = []
    for _ in range(nk):
        radius, beta = struct.unpack_from("<ii", data, off)
        off += 8
        b = list(struct.unpack_from("<12f", data, off))
        off += 48
        r_a, m, s, h = struct.unpack_from("<4f", data, off)
        off += 16
        c0, c1 = struct.unpack_from("<ii", data, off)
        off += 8
        kernels.append(KernelParams(radius=radius, beta_size=beta, b=b[:beta], r_a=r_a, m=m, s=s, h=h, c0=c0, c1=c1))
    (step,) = struct.unpack_from("<Q", data, off)
    off += 8
    (nf,) = struct.unpack_from("<I", data, off)
    off += 4
    fields = []
    for _ in range(nf):
        fid, n = struct.unpack_from("<IQ", data, off)
        off += 12 + 4 * n
        fields.append(fid)
    mass_target = None
    if _flags & 1:
        (nc,) = struct.unpack_from("<I", data, off)
        mass_target = list(struct.unpack_from(f"<{nc}d", data, off + 4))
    return {"version": version, "flags": _flags, "desc": desc, "kernels": kernels, "step": step,
            "fields": fields, "mass_target": mass_target}
