"""The multi-rank launcher (lenia_b200/launch.py) and bench.py's use of it,
on CPU: two gloo ranks rendezvous on 127.0.0.1 and all-reduce; bench.py
started as one process with --gpus 2 launches its own two ranks."""
import json
import os
import sys
import textwrap

import pytest

from lenia_b200.launch import maybe_spawn, spawn_ranks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = textwrap.dedent("""
    import datetime, json, os
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, n = dist.get_rank(), dist.get_world_size()
    assert r == int(os.environ["RANK"]) and n == int(os.environ["WORLD_SIZE"])
    t = torch.tensor([float(r + 1)])
    dist.all_reduce(t)
    if r == 0:
        print(json.dumps({"world": n, "sum": float(t.item()), "addr": os.environ["MASTER_ADDR"]}), flush=True)
    dist.barrier()
    dist.destroy_process_group()
""")


def test_spawn_ranks_gloo_allreduce(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    r = spawn_ranks(str(script), [], 2, timeout=180, capture=True)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert lines == [{"world": 2, "sum": 3.0, "addr": "127.0.0.1"}]


def test_maybe_spawn_runs_in_place_for_one_rank_or_inside_a_rank(monkeypatch):
    assert maybe_spawn("unused.py", [], 1) is None
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert maybe_spawn("unused.py", [], 2) is None


def test_bench_reference_arm_launches_its_own_ranks(oracle_built):
    import subprocess
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "2", "--warmup", "1", "--width", "32"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
