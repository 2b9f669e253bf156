"""The replica bookkeeping of multi-GPU runs (tertia_b200/replicas.py) with
two gloo ranks on the host: the launcher's environment, the barrier, the
maximum of the per-rank times and the whole-job rate.  The data path has no
collective (one independent march per GPU), so this is all that crosses
ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from tertia_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, w, local = replicas.dist_env()
    replicas.init(w, local, backend="gloo", timeout_s=60)
    replicas.barrier(w)
    ms = 10.0 + 5.0 * r                     # rank 1 is the slower one
    ms_max = replicas.max_over_ranks(ms, w, device="cpu")
    rate = replicas.whole_job_rate(1000.0, w, ms_max)
    replicas.barrier(w)
    replicas.finish(w)
    out.put((r, w, local, ms_max, rate))


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for r, w, local, ms_max, rate in got:
        assert w == world and local == r
        assert ms_max == 15.0
        assert rate == pytest.approx(world * 1000.0 / 0.015)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.dist_env() == (0, 1, 0)
    replicas.init(1, 0)
    replicas.barrier(1)
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.whole_job_rate(2.0e9, 1, 250.0) == pytest.approx(8.0e9)
    replicas.finish(1)
