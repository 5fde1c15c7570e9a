"""Checkpoints (lenia_save / lenia_load): round trip, header, integrity."""
import struct
import zlib

import numpy as np
import pytest

from lenia_b200 import params as P

pytestmark = pytest.mark.gpu


def _world(steps=3):
    from lenia_b200.world import World
    wl = P.config0(seed=4)
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    w.step(steps)
    return wl, w


def test_round_trip_then_identical_trajectories(tmp_path):
    from lenia_b200.world import World, read_checkpoint_header
    wl, w = _world()
    path = str(tmp_path / "w.ckp")
    w.save(path, step=3)
    data = open(path, "rb").read()
    assert zlib.crc32(data[:-4]) == struct.unpack("<I", data[-4:])[0]   # IEEE CRC-32 trailer
    hdr = read_checkpoint_header(path)
    assert hdr["step"] == 3 and hdr["desc"].width == 32 and len(hdr["kernels"]) == len(wl.kernels)
    assert all(np.float32(a.m) == np.float32(b.m) and a.c0 == b.c0 and a.c1 == b.c1
               for a, b in zip(hdr["kernels"], wl.kernels))
    w2, step = World.load(path)
    assert step == 3
    for name in ("A", "V", "GA", "SUM"):
        assert np.array_equal(w.get(name).view(np.uint32), w2.get(name).view(np.uint32)), name
    w.step(4)
    w2.step(4)
    for name in ("A", "V", "GA", "SUM"):
        assert np.array_equal(w.get(name).view(np.uint32), w2.get(name).view(np.uint32)), name
    w.close()
    w2.close()


def test_corrupt_and_foreign_versions_are_rejected(tmp_path):
    from lenia_b200.world import World
    from lenia_b200._lib import LeniaError
    _, w = _world(1)
    path = str(tmp_path / "w.ckp")
    w.save(path)
    w.close()
    data = bytearray(open(path, "rb").read())
    bad = bytearray(data)
    bad[len(bad) // 2] ^= 0x40
    open(tmp_path / "bad.ckp", "wb").write(bad)
    with pytest.raises(LeniaError) as e:
        World.load(str(tmp_path / "bad.ckp"))
    assert e.value.status == 1
    v2 = bytearray(data[:-4])
    v2[8:12] = struct.pack("<I", 2)
    v2 += struct.pack("<I", zlib.crc32(bytes(v2)))
    open(tmp_path / "v2.ckp", "wb").write(v2)
    with pytest.raises(LeniaError) as e:
        World.load(str(tmp_path / "v2.ckp"))
    assert e.value.status == 7


def test_conserve_mass_resume_matches_continuous_run(tmp_path):
    """A conserve_mass world saved mid-run and resumed steps bit for bit like
    the world that never stopped: the checkpoint carries the target totals
    (recorded at the last write of the grid), not the restored grid's."""
    from lenia_b200.world import World, read_checkpoint_header
    wl = P.config0(seed=5)
    wl.desc.conserve_mass = True
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    target = w.get("A").reshape(wl.desc.channels, -1).astype(np.float64).sum(axis=1)
    w.step(4)
    path = str(tmp_path / "m.ckp")
    w.save(path, step=4)
    hdr = read_checkpoint_header(path)
    assert hdr["flags"] & 1 and hdr["mass_target"] is not None
    assert np.allclose(hdr["mass_target"], target, rtol=1e-12, atol=0)
    w2, _ = World.load(path)
    w.step(6)
    w2.step(6)
    for name in ("A", "V", "GA", "SUM"):
        assert np.array_equal(w.get(name).view(np.uint32), w2.get(name).view(np.uint32)), name
    w.close()
    w2.close()
