"""The multi-GPU path (independent replicas, gendil_b200.replicas) as world-size-2 gloo process
groups on CPU: barriers, the max-over-ranks timing and the whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from gendil_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    ms = r.max(10.0 + rank)  # the slowest rank's time wins
    out.put((rank, r.world, ms, r.throughput(1000, ms)))
    r.close()


def test_replicas_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(world))
    for rank, w, ms, rate in res:
        assert w == 2 and ms == 11.0
        assert rate == pytest.approx(2 * 1000 / 11e-3)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from gendil_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.world == 1 and r.dist is None
    assert r.max(3.5) == 3.5
    r.close()
