"""Batches of worlds: bit-identity with worlds stepped alone (GPU), and the
partition of a batch across ranks (CPU, gloo)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from lenia_b200 import params as P
from lenia_b200.batch import shard_worlds, world_cost


def test_config3_draws_every_size_and_mode():
    wls = P.config3(64, seed=1)
    assert {wl.desc.width for wl in wls} == set(P.CONFIG3_SIZES)
    assert {wl.desc.mode_type for wl in wls} == {P.MODE_RT, P.MODE_ADV}
    again = P.config3(3, seed=1)
    assert all(np.array_equal(a.A0, b.A0) for a, b in zip(wls[:3], again))


def test_shard_worlds_partitions_and_balances():
    wls = P.config3(200, seed=2)
    costs = [world_cost(wl.desc, len(wl.kernels)) for wl in wls]
    for n in (1, 2, 3, 8):
        parts = shard_worlds(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: no rank exceeds the mean by more than the largest world
        assert max(loads) - sum(loads) / n <= max(costs)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, n_worlds, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        wls = P.config3(n_worlds, seed=5)
        costs = [world_cost(wl.desc, len(wl.kernels)) for wl in wls]
        mine = shard_worlds(costs, world_size)[rank]
        every = [None] * world_size
        dist.all_gather_object(every, mine)
        import torch
        t = torch.tensor([float(sum(costs[i] for i in mine)), float(len(mine))], dtype=torch.float64)
        dist.all_reduce(t)
        q.put((rank, every, float(t[0]), int(t[1]), float(sum(costs))))
    finally:
        dist.destroy_process_group()


def test_shards_over_gloo_ranks():
    """Two gloo ranks compute the same partition independently; the shards
    are disjoint and cover the batch, and the reduced totals match."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, 40, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    every0, every1 = res[0][1], res[1][1]
    assert every0 == every1
    assert sorted(i for part in every0 for i in part) == list(range(40))
    assert not set(every0[0]) & set(every0[1])
    assert res[0][2] == res[0][4] and res[0][3] == 40


@pytest.mark.gpu
def test_batch_matches_worlds_stepped_alone():
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wls = P.config3(7, seed=11, sizes=(24, 32, 36, 48))
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=3)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    alone = []
    for wl in wls:
        w = World(wl.desc, wl.kernels)
        w.set_state(wl.A0.ravel())
        alone.append(w)
    for steps in (3, 2):   # an odd count first: the batch alternates its two graphs
        b.step(steps)
        for w in alone:
            w.step(steps)
        b.sync()
        for i, w in enumerate(alone):
            for name in ("A", "V", "GA", "SUM"):
                got, want = b.get(i, name), w.get(name)
                assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (i, name, steps)
    # every world takes the batched launches: fewer launches than worlds x stages
    assert b.grouped_worlds() == len(wls)
    assert 0 < b.launches_per_step() < 6 * len(wls)
    for w in alone:
        w.close()
    b.close()


@pytest.mark.gpu
def test_batched_job_lists_beyond_one_launch():
    """7,300 worlds of 24^3 with 9 kernels give 65,700 inverse-plane jobs of
    one grid size, more than one launch's grid.y holds (65,535): the job list
    runs as two launches, and worlds on both sides of the split step bit for
    bit as stepped alone."""
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wls = P.config3(7300, seed=31, sizes=(24,))
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=4)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    assert b.grouped_worlds() == len(wls)
    b.step(1)
    b.sync()
    for i in (0, 7280, 7283, 7299):
        w = World(wls[i].desc, wls[i].kernels)
        w.set_state(wls[i].A0.ravel())
        w.step(1)
        for name in ("A", "V", "GA", "SUM"):
            got, want = b.get(i, name), w.get(name)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (i, name)
        w.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
def test_config3_mix_matches_worlds_stepped_alone(batched):
    """Every config-3 size (24 .. 96), RT and advection, plus two worlds the
    batched launches do not take (dd = 2, and central differences with the
    blur), stepped in one batch with the batched launches on and off: every
    world bit for bit as stepped alone."""
    import dataclasses
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wls = P.config3(16, seed=21)
    extra = P.config3(2, seed=22, sizes=(32,))
    extra[0] = P.Workload(dataclasses.replace(extra[0].desc, mode_type=P.MODE_RT, sigma=1.2, dd=2.0),
                          extra[0].kernels, extra[0].A0)
    extra[1] = P.Workload(dataclasses.replace(extra[1].desc, blur_central_diff=True), extra[1].kernels, extra[1].A0)
    wls = wls + extra
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=4)
    if not batched:
        b.set_batched_launches(False)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    assert b.grouped_worlds() == (16 if batched else 0)
    alone = []
    for wl in wls:
        w = World(wl.desc, wl.kernels)
        w.set_state(wl.A0.ravel())
        alone.append(w)
    for steps in (1, 2):
        b.step(steps)
        for w in alone:
            w.step(steps)
        b.sync()
        for i, w in enumerate(alone):
            for name in ("A", "V", "GA", "SUM"):
                got, want = b.get(i, name), w.get(name)
                assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (i, wls[i].desc.width, name,
                                                                                     steps)
    for w in alone:
        w.close()
    b.close()


@pytest.mark.gpu
def test_batch_autotune_then_matches_worlds_with_the_same_choice():
    """After lenia_batch_autotune every world of a grid shape carries the
    shape's choice, and the batch (graphs captured again) still matches
    worlds stepped alone with that choice bit for bit."""
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wls = P.config3(6, seed=13, sizes=(24, 36, 48))
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=2)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    b.step(1)
    res = b.autotune()
    print(res)
    by_shape = {}
    for wl, r in zip(wls, res):
        key = (wl.desc.width, wl.desc.height)
        assert by_shape.setdefault(key, (r["conv_mode"], r["row_tile"])) == (r["conv_mode"], r["row_tile"])
        assert r["ms"]["FFT"] is not None and r["ms"]["DIRECT_BF16X3"] is not None
    alone = []
    for wl, r in zip(wls, res):
        w = World(wl.desc, wl.kernels)
        w.set_conv_mode(r["conv_mode"])
        w.set_state(wl.A0.ravel())
        w.step(1)
        alone.append(w)
    b.step(3)
    for w in alone:
        w.step(3)
    b.sync()
    for i, w in enumerate(alone):
        for name in ("A", "V", "GA", "SUM"):
            got, want = b.get(i, name), w.get(name)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (i, name)
    for w in alone:
        w.close()
    b.close()


@pytest.mark.gpu
def test_batch_runs_the_direct_convolution_in_its_graphs():
    """With the autotuner restricted to BF16X3 every world of the batch
    convolves on the tensor cores inside the captured step graphs, bit for
    bit as worlds stepped alone in that mode."""
    from lenia_b200.batch import Batch
    from lenia_b200.world import World
    wls = P.config3(4, seed=14, sizes=(24, 32))
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=2)
    for i, wl in enumerate(wls):
        b.set_state(i, wl.A0)
    res = b.autotune(modes=("DIRECT_BF16X3",))
    assert all(r["conv_mode"] == "DIRECT_BF16X3" for r in res)
    alone = []
    for wl in wls:
        w = World(wl.desc, wl.kernels)
        w.set_conv_mode("DIRECT_BF16X3")
        w.set_state(wl.A0.ravel())
        alone.append(w)
    b.step(3)
    for w in alone:
        w.step(3)
    b.sync()
    for i, w in enumerate(alone):
        w.sync()
        for name in ("A", "V", "GA", "SUM"):
            got, want = b.get(i, name), w.get(name)
            assert np.isfinite(got).all()
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (i, name)
    for w in alone:
        w.close()
    b.close()


@pytest.mark.gpu
def test_batch_rejects_scratch_fields():
    from lenia_b200.batch import Batch
    from lenia_b200._lib import LeniaError
    wls = P.config3(2, seed=12, sizes=(24,))
    b = Batch([wl.desc for wl in wls], [wl.kernels for wl in wls], lanes=2)
    with pytest.raises(LeniaError):
        b._check(b._lib.lenia_batch_get_field(b._h, 0, 4, None, 0, 0))  # H lives in the lane
    b.close()
