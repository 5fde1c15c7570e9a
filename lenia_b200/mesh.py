"""Marching cubes over the C ABI: the reference's generate_mesh_v1/v2/v3
(mesh.cpp) with its buffer reset and concatenation (render.cpp:153-212),
headless.

`Mesher` meshes every channel of one to three fields (a World's snapshots,
or CUDA tensors of channels x depth x height x width floats) and returns flat
arrays:
positions and normals (V x 3), the creating channel of each vertex, triangle
indices (T x 3), face normals (T x 3) and, on request, the case index of every
cube.  `write_ply` / `write_obj` dump a mesh to a file.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib

CELL_SIZE = 3.5     # render.h:26
MESH_THREADS = 2    # render.h:15


@dataclass
class MeshArrays:
    positions: np.ndarray       # (V, 3) float32
    normals: np.ndarray         # (V, 3) float32, unnormalised
    vertex_channel: np.ndarray  # (V,) int32: channel + channels * field
    indices: np.ndarray         # (T, 3) uint32
    face_normals: np.ndarray    # (T, 3) float32
    cases: Optional[np.ndarray] = None  # (F, C, N) uint8

    @property
    def n_vertices(self) -> int:
        return self.positions.shape[0]

    @property
    def n_triangles(self) -> int:
        return self.indices.shape[0]


def triangle_table() -> np.ndarray:
    """The library's 256 x 16 triangle table (edge indices, -1 terminated)."""
    lib = _lib.load()
    t = np.zeros(256 * 16, dtype=np.int32)
    if lib.lenia_mc_triangle_table(t.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) != 0:
        raise RuntimeError("lenia_mc_triangle_table failed")
    return t.reshape(256, 16)


class Mesher:
    """Iso-surface extraction for fields of one shape.

    fields > 1 meshes several fields together (the reference's U and H
    views), each with its own vertex map and its own offset (one (x, y, z)
    per field).  slabs=2, share_channels=True reproduce the reference's two
    mesh threads and its vertex maps shared by all channels; slabs=1,
    share_channels=False give one mesh per channel without seam duplicates."""

    def __init__(self, width: int, height: int, channels: int, iso_value: float = 0.5,
                 cell_size: float = CELL_SIZE, fields: int = 1, offsets=None, slabs: int = MESH_THREADS,
                 share_channels: bool = True):
        d = _lib.LeniaMeshDesc()
        d.width, d.height, d.channels, d.fields = width, height, channels, fields
        d.iso_value, d.cell_size = float(iso_value), float(cell_size)
        if offsets is not None:
            for f, o in enumerate(offsets):
                for a in range(3):
                    d.offset[f][a] = float(o[a])
        d.slabs, d.share_channels = int(slabs), 1 if share_channels else 0
        self._init(d)

    @classmethod
    def for_view(cls, view: str, width: int, height: int, channels: int, iso_value: float = 0.5) -> "Mesher":
        """A mesher set up as the reference meshes view NORMAL, U or H."""
        lib = _lib.load()
        d = _lib.LeniaMeshDesc()
        st = lib.lenia_mesh_desc_for_view(_lib.VIEW[view], width, height, channels, float(iso_value),
                                          ctypes.byref(d))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, "lenia_mesh_desc_for_view failed")
        m = cls.__new__(cls)
        m._init(d)
        return m

    def _init(self, d):
        self._lib = _lib.load()
        self.width, self.height, self.channels, self.fields = d.width, d.height, d.channels, d.fields
        self._d = d
        h = ctypes.c_void_p()
        st = self._lib.lenia_mesher_create(ctypes.byref(d), ctypes.byref(h))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, "lenia_mesher_create failed")
        self._h = h
        self._world = None  # a World whose stream the last run used, kept alive for get()
        self.n_vertices = 0
        self.n_triangles = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lenia_mesher_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, self._lib.lenia_mesher_last_error(self._h).decode())

    def run(self, fields, halos=None, stream: int = 0) -> tuple[int, int]:
        """Meshes CUDA tensors (one per field, channels x depth x height x
        width float32; a single tensor for one field) on `stream` (a
        cudaStream_t as int; 0 = default).  halos: per field the tensor whose
        periodic copy the +1 faces hold (None: the field).  Returns (V, T)."""
        if not isinstance(fields, (list, tuple)):
            fields = [fields]
        if len(fields) != self.fields:
            raise ValueError(f"the mesher meshes {self.fields} fields")
        n = self.channels * self.width * self.height * self.width
        keep = []

        def ptrs(ts):
            arr = (ctypes.c_void_p * 3)()
            for i, t in enumerate(ts):
                if t is None:
                    continue
                if not (hasattr(t, "is_cuda") and t.is_cuda):
                    raise TypeError("Mesher.run takes CUDA tensors; use run_world for a World")
                t = t.contiguous()
                if t.numel() != n:
                    raise ValueError("field shape does not match the mesher")
                keep.append(t)
                arr[i] = t.data_ptr()
            return arr

        fp = ptrs(fields)
        hp = ptrs(halos) if halos is not None else None
        nv, nt = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._lib.lenia_mesher_run(self._h, fp, hp, ctypes.c_void_p(stream), ctypes.byref(nv),
                                               ctypes.byref(nt)))
        self._world = None
        self.n_vertices, self.n_triangles = nv.value, nt.value
        return self.n_vertices, self.n_triangles

    def run_world(self, world, view: str = "NORMAL") -> tuple[int, int]:
        """Meshes a World's snapshots as the reference's view NORMAL (RBB), U
        (+ U_SUM_RB) or H (+ U_SUM_RB, H_RB) on the world's stream."""
        nv, nt = ctypes.c_longlong(), ctypes.c_longlong()
        st = self._lib.lenia_mesh_world(world.handle, _lib.VIEW[view], self._h, ctypes.byref(nv), ctypes.byref(nt))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, self._lib.lenia_last_error(world.handle).decode())
        self._world = world
        self.n_vertices, self.n_triangles = nv.value, nt.value
        return self.n_vertices, self.n_triangles

    def get(self, name: str) -> np.ndarray:
        """One array of the last mesh, copied to the host."""
        nv, nt = self.n_vertices, self.n_triangles
        n_cells = self.channels * self.width * self.height * self.width
        shape, dtype = {
            "positions": ((nv, 3), np.float32), "normals": ((nv, 3), np.float32),
            "vertex_channel": ((nv,), np.int32), "indices": ((nt, 3), np.uint32),
            "face_normals": ((nt, 3), np.float32),
            "cases": ((self.fields, self.channels, n_cells // self.channels), np.uint8),
        }[name]
        out = np.zeros(shape, dtype=dtype)
        self._check(self._lib.lenia_mesher_get(self._h, _lib.MESH_ARRAY[name], out.ctypes.data_as(ctypes.c_void_p),
                                               out.size, 0))
        return out

    def arrays(self, cases: bool = False) -> MeshArrays:
        return MeshArrays(self.get("positions"), self.get("normals"), self.get("vertex_channel"),
                          self.get("indices"), self.get("face_normals"), self.get("cases") if cases else None)


def write_ply(path: str, m: MeshArrays) -> None:
    """Binary little-endian PLY: vertex x y z nx ny nz (float), channel
    (uchar); faces as uchar-counted uint lists."""
    with open(path, "wb") as f:
        f.write(("ply\nformat binary_little_endian 1.0\n"
                 f"element vertex {m.n_vertices}\n"
                 "property float x\nproperty float y\nproperty float z\n"
                 "property float nx\nproperty float ny\nproperty float nz\n"
                 "property uchar channel\n"
                 f"element face {m.n_triangles}\n"
                 "property list uchar uint vertex_indices\nend_header\n").encode())
        v = np.zeros(m.n_vertices, dtype=[("p", "<f4", 3), ("n", "<f4", 3), ("c", "u1")])
        v["p"], v["n"], v["c"] = m.positions, m.normals, m.vertex_channel.astype(np.uint8)
        f.write(v.tobytes())
        fc = np.zeros(m.n_triangles, dtype=[("k", "u1"), ("i", "<u4", 3)])
        fc["k"], fc["i"] = 3, m.indices
        f.write(fc.tobytes())


def write_obj(path: str, m: MeshArrays) -> None:
    """Wavefront OBJ with vertex normals (1-based indices)."""
    with open(path, "w") as f:
        for p in m.positions:
            f.write(f"v {p[0]:.9g} {p[1]:.9g} {p[2]:.9g}\n")
        for n in m.normals:
            f.write(f"vn {n[0]:.9g} {n[1]:.9g} {n[2]:.9g}\n")
        for a, b, c in m.indices.astype(np.int64) + 1:
            f.write(f"f {a}//{a} {b}//{b} {c}//{c}\n")
