"""One process per GPU: re-runs a script as N ranks under torch.distributed.run.

`spawn_ranks(script, argv, n)` starts `python -m torch.distributed.run
--nnodes 1 --nproc-per-node n --master-addr 127.0.0.1 --master-port P script
argv...` and returns its exit code; each rank reads RANK / LOCAL_RANK /
WORLD_SIZE / MASTER_ADDR / MASTER_PORT from its environment.  A script that is
asked for n ranks but was started as a single process (no WORLD_SIZE in the
environment) calls `maybe_spawn`, which launches the ranks and tells the
caller to return the launcher's exit code instead of running itself.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys
from typing import Optional, Sequence


def free_port() -> int:
    """A TCP port on 127.0.0.1 that was free a moment ago."""
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return int(s.getsockname()[1])


def spawn_ranks(script: str, argv: Sequence[str], n: int, port: Optional[int] = None, timeout: Optional[float] = None,
                env: Optional[dict] = None, capture: bool = False):
    """Runs `script argv...` as n ranks (torch.distributed.run, one node,
    rendezvous on 127.0.0.1).  Returns the exit code, or with capture=True the
    CompletedProcess (stdout and stderr as text)."""
    if n < 1:
        raise ValueError(f"need at least one rank, got {n}")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={int(n)}",
           "--master-addr=127.0.0.1", f"--master-port={port or free_port()}", script, *argv]
    e = dict(os.environ if env is None else env)
    e.setdefault("OMP_NUM_THREADS", "1")
    r = subprocess.run(cmd, env=e, timeout=timeout, text=True,
                       stdout=subprocess.PIPE if capture else None, stderr=subprocess.PIPE if capture else None)
    return r if capture else r.returncode


def maybe_spawn(script: str, argv: Sequence[str], n: int) -> Optional[int]:
    """None when this process is already a rank (WORLD_SIZE set) or n == 1:
    the caller runs.  Otherwise launches n ranks of `script argv` and returns
    their exit code, which the caller returns as its own."""
    if n <= 1 or "WORLD_SIZE" in os.environ:
        return None
    return spawn_ranks(script, argv, n)
