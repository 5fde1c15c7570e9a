"""Marching cubes (mesh.cpp:34-431): tables, the restatement pinned to the
reference build, and the CUDA mesher against the restatement.

The reference's tables (marching_cubes.h) are third-party data and are not in
this repository: the tests that need them read the reference's header at test
time and skip when it is absent."""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from lenia_b200 import params as P

import lenia_cases as LC

REF_MC = O.ref_path("marching_cubes.h")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_MC), reason="reference sources absent")


def _ref_tables():
    src = open(REF_MC).read()

    def parse(name):
        body = src[src.index(name):]
        body = body[body.index("{"):body.index(";")]
        body = re.sub(r"//[^\n]*", "", body)
        return [int(x, 0) for x in re.findall(r"-?0x[0-9a-fA-F]+|-?\d+", body)]

    edge_table = np.array(parse("EDGE_TABLE[256]"), dtype=np.int64)
    tri_table = np.array(parse("TRIANGLE_TABLE[256][16]"), dtype=np.int32).reshape(256, 16)
    e2v = np.array(parse("EDGE_TO_VERTICES[][2]"), dtype=np.int32).reshape(12, 2)
    return edge_table, tri_table, e2v


def _counts(table):
    return np.array([(row != -1).sum() // 3 for row in table])


def _lib_table():
    from lenia_b200 import mesh
    return mesh.triangle_table()


# ---------------------------------------------------------------- tables

@needs_ref
def test_edge_geometry_matches_reference():
    import ctypes
    lib = O.RestateOracle.lib()
    edge_table, _, e2v = _ref_tables()
    a, b = ctypes.c_int(), ctypes.c_int()
    for e in range(12):
        lib.mc_edge_corners(e, ctypes.byref(a), ctypes.byref(b))
        assert (a.value, b.value) == tuple(e2v[e]), e
    assert [lib.mc_edge_mask(c) for c in range(256)] == list(edge_table)


@needs_ref
def test_triangle_counts_match_reference():
    _, tri_table, _ = _ref_tables()
    ref = _counts(tri_table)
    own = _counts(O.mc_table())
    differ = np.nonzero(ref != own)[0].tolist()
    assert differ == [], f"cases whose triangle count differs from the reference's: {differ}"


def test_library_table_equals_oracle_table():
    assert np.array_equal(_lib_table(), O.mc_table())


def test_table_uses_exactly_the_intersected_edges():
    import ctypes
    lib = O.RestateOracle.lib()
    t = O.mc_table()
    assert (t[0] == -1).all() and (t[255] == -1).all()
    for c in range(256):
        used = {int(e) for e in t[c] if e != -1}
        mask = lib.mc_edge_mask(c)
        assert used == {e for e in range(12) if mask >> e & 1}, c
        tris = t[c][t[c] != -1].reshape(-1, 3)
        assert all(len(set(tr)) == 3 for tr in tris), c
    del ctypes


def _closed_field(seed, W=24, H=24, C=2):
    """Smooth blobs away from the border: every channel's surface is closed."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(W), np.arange(H), np.arange(W), indexing="ij")
    f = np.zeros((C, W, H, W), np.float32)
    for c in range(C):
        for _ in range(4):
            cz, cy, cx = rng.uniform(6, W - 6), rng.uniform(6, H - 6), rng.uniform(6, W - 6)
            r = rng.uniform(2.0, 4.5)
            f[c] += np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2 * r * r)).astype(np.float32)
        f[c] += rng.uniform(-0.08, 0.08, size=f[c].shape).astype(np.float32)
        f[c, :2] = f[c, -2:] = 0
        f[c, :, :2] = f[c, :, -2:] = 0
        f[c, :, :, :2] = f[c, :, :, -2:] = 0
    return f, W, H, C


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_own_table_meshes_are_watertight(seed):
    """With one consistent rule for ambiguous faces, neighbouring cubes agree
    on every shared face: each mesh edge borders exactly two triangles."""
    f, W, H, C = _closed_field(seed)
    m = O.mesh_restated(f, W, H, C, 0.35, slabs=1, share_channels=False)
    assert m.n_triangles > 100
    tri = m.indices.reshape(-1, 3).astype(np.int64)
    edges = np.sort(np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]), axis=1)
    _, counts = np.unique(edges, axis=0, return_counts=True)
    assert (counts == 2).all(), np.bincount(counts)


# ------------------------------------------- restatement vs reference build

def _ref_state(wl, steps):
    p, k = LC.as_oracle(wl)
    ref = O.RefOracle(p, k)
    ref.set_state(A=wl.A0)
    ref.step(steps)   # the last event of a step is TMB: RBB holds this step's grid
    return ref, p


SHIFT = np.float32(32 * 3.5)
VIEW_OFFSETS = np.array([[0, 0, 0], [SHIFT, 0, 0], [0, 0, SHIFT]], np.float32)


@needs_ref
@pytest.mark.parametrize("case", [("cfg0", 1), ("cfg0", 5), ("sobel_none", 2), ("four", 3)])
@pytest.mark.parametrize("view", [0, 1, 2])
def test_restatement_reproduces_reference_mesh(case, view):
    """generate_mesh_v1/v2/v3 of the reference build (two mesh threads,
    vertex maps shared by channels, no stitching) equal the restatement run
    with the reference's own table, its halo sources (the +1 faces of
    U_SUM_RB and H_RB copy U_SUM and H) and its normal-slot quirks: positions
    and indices bit for bit, normals bit for bit except on vertices whose
    normal read a slot the reference never wrote (uninitialised memory)."""
    name, steps = case
    wl = LC.four_channels() if name == "four" else LC.variant(name)
    ref, p = _ref_state(wl, steps)
    _, tri_table, _ = _ref_tables()
    fields = [ref.get("RBB"), ref.get("U_SUM_RB"), ref.get("H_RB")][:view + 1]
    halos = [ref.get("A"), ref.get("U_SUM"), ref.get("H")][:view + 1]
    a = O.mesh_reference(ref, view)
    b = O.mesh_restated(fields, 32, 32, p["channels"], np.float32(p["iso_value"]), offsets=VIEW_OFFSETS[:view + 1],
                        table=tri_table, slabs=2, share_channels=True, halos=halos, quirks=True)
    assert a.n_triangles > 1000
    assert a.n_vertices == b.n_vertices and a.n_triangles == b.n_triangles
    assert np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.positions.view(np.uint32), b.positions.view(np.uint32))
    same = (a.normals.view(np.uint32) == b.normals.view(np.uint32)).all(axis=1)
    assert (same | b.unsure).all()
    if view == 0:
        assert not b.unsure.any()
    assert b.unsure.mean() < 0.05


@needs_ref
def test_reference_mesh_of_empty_grid_is_empty():
    wl = LC.variant("cfg0")
    p, k = LC.as_oracle(wl)
    ref = O.RefOracle(p, k)
    ref.set_state(A=np.zeros_like(wl.A0))
    ref.run_event("TMB")
    m = O.mesh_reference(ref)
    assert m.n_vertices == 0 and m.n_triangles == 0


def test_restatement_own_vs_reference_table_same_case_indices():
    """Case indices and triangle counts do not depend on the table's
    triangulation: the restatement's count equals the sum of per-case counts."""
    wl = LC.variant("cfg0")
    f = wl.A0
    m = O.mesh_restated(f, 32, 32, 3, 0.5, slabs=2, share_channels=True)
    counts = _counts(O.mc_table())
    assert m.n_triangles == int(counts[m.cases].sum())


def test_quirk_free_normals_are_face_normal_sums():
    """Without the quirks every vertex normal is the sum, in creation order,
    of the face normals of the triangles that use it."""
    wl = LC.four_channels()
    rng = np.random.default_rng(4)
    fields = [wl.A0, rng.uniform(0, 1, wl.A0.shape).astype(np.float32)]
    m = O.mesh_restated(fields, 32, 32, 4, 0.5, offsets=VIEW_OFFSETS[:2], slabs=2, share_channels=True)
    tri = m.indices.reshape(-1, 3)
    acc = np.zeros_like(m.normals)
    for t in range(tri.shape[0]):
        for v in tri[t]:
            acc[v] = (acc[v] + m.face_normals[t]).astype(np.float32)
    assert np.array_equal(acc.view(np.uint32), m.normals.view(np.uint32))


# ------------------------------------------------------------ CUDA mesher

def _gpu_mesh(fields, W, H, C, iso, halos=None, **kw):
    import torch
    from lenia_b200.mesh import Mesher
    if isinstance(fields, np.ndarray):
        fields = [fields]
    ts = [torch.from_numpy(np.ascontiguousarray(f, np.float32).reshape(-1)).cuda() for f in fields]
    hs = None
    if halos is not None:
        hs = [None if h is None else torch.from_numpy(np.ascontiguousarray(h, np.float32).reshape(-1)).cuda()
              for h in halos]
    ms = Mesher(W, H, C, iso_value=iso, fields=len(ts), **kw)
    ms.run(ts, halos=hs)
    torch.cuda.synchronize()
    return ms.arrays(cases=True)


def _assert_same(g, o, label=""):
    assert g.n_vertices == o.n_vertices and g.n_triangles == o.n_triangles, label
    assert np.array_equal(g.cases.ravel(), o.cases.ravel()), label
    assert np.array_equal(g.indices.ravel(), o.indices), label
    assert np.array_equal(g.vertex_channel, o.vertex_channel), label
    assert np.array_equal(g.positions.view(np.uint32), o.positions.view(np.uint32)), label
    assert np.array_equal(g.face_normals.view(np.uint32), o.face_normals.view(np.uint32)), label
    assert np.array_equal(g.normals.view(np.uint32), o.normals.view(np.uint32)), label


MODES = [dict(slabs=2, share_channels=True), dict(slabs=1, share_channels=False),
         dict(slabs=3, share_channels=True), dict(slabs=1, share_channels=True, offsets=[(112.0, 0.0, -3.5)])]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", range(len(MODES)))
def test_gpu_mesh_matches_restatement_seed_cube(mode):
    wl = LC.variant("cfg0")
    kw = MODES[mode]
    o = O.mesh_restated(wl.A0, 32, 32, 3, 0.5, **kw)
    g = _gpu_mesh(wl.A0, 32, 32, 3, 0.5, **kw)
    assert o.n_triangles > 10000
    _assert_same(g, o, str(kw))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(24, 40, 2), (40, 24, 4), (17, 9, 1)])
def test_gpu_mesh_matches_restatement_shapes(shape):
    W, H, C = shape
    rng = np.random.default_rng(W * 100 + H)
    f = rng.uniform(0, 1, size=(C, W, H, W)).astype(np.float32)
    f[:, :, :, ::5] = 0.5      # corners exactly at the iso value
    for kw in MODES:
        o = O.mesh_restated(f, W, H, C, 0.5, **kw)
        g = _gpu_mesh(f, W, H, C, 0.5, **kw)
        _assert_same(g, o, f"{shape} {kw}")


@pytest.mark.gpu
@pytest.mark.parametrize("nfields", [2, 3])
def test_gpu_mesh_matches_restatement_fields(nfields):
    """Fields meshed together (the U and H views), each with its own halo
    source and offset, in both slab/sharing modes."""
    W, H, C = 24, 20, 3
    rng = np.random.default_rng(nfields)
    fields = [rng.uniform(0, 1, size=(C, W, H, W)).astype(np.float32) for _ in range(nfields)]
    halos = [None] + [rng.uniform(0, 1, size=(C, W, H, W)).astype(np.float32) for _ in range(nfields - 1)]
    offs = [(0, 0, 0), (84.0, 0, 0), (0, 0, 84.0)][:nfields]
    for kw in (dict(slabs=2, share_channels=True), dict(slabs=1, share_channels=False)):
        o = O.mesh_restated(fields, W, H, C, 0.5, offsets=offs, halos=halos, **kw)
        g = _gpu_mesh(fields, W, H, C, 0.5, halos=halos, offsets=offs, **kw)
        assert o.n_triangles > 10000
        _assert_same(g, o, f"{nfields} {kw}")


@pytest.mark.gpu
def test_gpu_mesh_empty_and_full():
    for value in (0.0, 1.0):
        f = np.full((2, 16, 16, 16), value, np.float32)
        o = O.mesh_restated(f, 16, 16, 2, 0.5, slabs=2, share_channels=True)
        g = _gpu_mesh(f, 16, 16, 2, 0.5, slabs=2, share_channels=True)
        _assert_same(g, o, f"value {value}")
        if value == 0.0:
            assert g.n_triangles == 0 and g.n_vertices == 0


def _world_after(wl, steps):
    from lenia_b200.world import World
    w = World(wl.desc, wl.kernels)
    w.set_snapshots(True)
    w.set_state(wl.A0)
    w.step(steps)
    return w


@pytest.mark.gpu
@pytest.mark.parametrize("view", ["NORMAL", "U", "H"])
def test_gpu_mesh_of_world_views(view):
    """lenia_mesh_world for each view equals the restatement of the world's
    snapshots with the reference's halo sources and offsets."""
    from lenia_b200.mesh import Mesher
    wl = LC.four_channels()
    w = _world_after(wl, 3)
    nf = {"NORMAL": 1, "U": 2, "H": 3}[view]
    fields = [w.get("RBB"), w.get("U_SUM_RB"), w.get("H_RB")][:nf]
    halos = [w.get("A"), w.get("U_SUM"), w.get("H")][:nf]
    ms = Mesher.for_view(view, 32, 32, 4, iso_value=wl.desc.iso_value)
    ms.run_world(w, view)
    g = ms.arrays(cases=True)
    o = O.mesh_restated(fields, 32, 32, 4, np.float32(wl.desc.iso_value), offsets=VIEW_OFFSETS[:nf], halos=halos,
                        slabs=2, share_channels=True)
    assert o.n_triangles > 1000
    _assert_same(g, o, view)


@pytest.mark.gpu
def test_gpu_snapshot_copy_deferred():
    """The grid snapshot (RBB) is the grid at the end of the last step that
    took one, however it is read: meshed in place, read out, after steps
    without snapshots, and after the grid itself is overwritten."""
    from lenia_b200.mesh import Mesher
    wl = LC.four_channels()
    w = _world_after(wl, 3)
    ms = Mesher.for_view("NORMAL", 32, 32, 4, iso_value=wl.desc.iso_value)
    ms.run_world(w, "NORMAL")                 # reads the grid buffer in place
    lazy = ms.arrays(cases=True)
    a3 = w.get("A")
    assert np.array_equal(w.get("RBB").view(np.uint32), a3.view(np.uint32))
    ms.run_world(w, "NORMAL")                 # reads the copy
    copied = ms.arrays(cases=True)
    for name in ("positions", "normals", "vertex_channel", "indices", "face_normals", "cases"):
        a, b = getattr(copied, name), getattr(lazy, name)
        assert a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
    # steps without snapshots leave the snapshot of step 3 (its buffer is
    # overwritten two steps later)
    w.step(1)
    w.set_snapshots(False)
    a4 = w.get("A")
    w.step(3)
    w.set_snapshots(True)
    assert np.array_equal(w.get("RBB").view(np.uint32), a4.view(np.uint32))
    # a snapshot, then the grid replaced: RBB keeps the stepped grid
    w.step(1)
    a5 = w.get("A")
    w.set_state(np.zeros_like(a5))
    assert np.array_equal(w.get("RBB").view(np.uint32), a5.view(np.uint32))
    ms.close()
    w.close()


@pytest.mark.gpu
def test_gpu_mesh_config1_size():
    """128^3 x 4 channels, the single-world size, after two steps."""
    from lenia_b200.mesh import Mesher
    wl = P.config1()
    w = _world_after(wl, 2)
    A = w.get("RBB")
    for kw in (dict(slabs=2, share_channels=True), dict(slabs=1, share_channels=False)):
        ms = Mesher(128, 128, 4, iso_value=wl.desc.iso_value, **kw)
        ms.run_world(w, "NORMAL")
        g = ms.arrays(cases=True)
        o = O.mesh_restated(A, 128, 128, 4, np.float32(wl.desc.iso_value), **kw)
        assert o.n_triangles > 10000
        _assert_same(g, o, str(kw))


def test_ply_and_obj_dumps(tmp_path):
    """The PLY/OBJ writers emit every vertex and face of a mesh."""
    from lenia_b200.mesh import MeshArrays, write_obj, write_ply
    f, W, H, C = _closed_field(5, W=16, H=16, C=1)
    o = O.mesh_restated(f, W, H, C, 0.35, slabs=1, share_channels=False)
    m = MeshArrays(o.positions, o.normals, o.vertex_channel, o.indices.reshape(-1, 3), o.face_normals)
    ply = tmp_path / "m.ply"
    write_ply(str(ply), m)
    data = ply.read_bytes()
    head, body = data.split(b"end_header\n", 1)
    assert f"element vertex {m.n_vertices}".encode() in head
    assert f"element face {m.n_triangles}".encode() in head
    assert len(body) == m.n_vertices * 25 + m.n_triangles * 13
    faces = np.frombuffer(body[m.n_vertices * 25:], dtype=[("k", "u1"), ("i", "<u4", 3)])
    assert (faces["k"] == 3).all() and np.array_equal(faces["i"], m.indices)
    obj = tmp_path / "m.obj"
    write_obj(str(obj), m)
    lines = obj.read_text().splitlines()
    assert sum(l.startswith("v ") for l in lines) == m.n_vertices
    assert sum(l.startswith("f ") for l in lines) == m.n_triangles
