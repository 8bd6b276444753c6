"""Multi-process host logic of the replica-parallel path, on CPU with gloo (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from soliton_solver_b200.replicas import replica_seed, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q, mode):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    from soliton_solver_b200 import replicas
    try:
        replicas.init("gloo", timeout_s=10.0)
        if mode == "ok":
            mine = list(replicas.shard(10, rank, world))
            t = replicas.max_over_ranks(1.5 + rank)
            s = replicas.sum_over_ranks(len(mine))
            replicas.barrier()
            q.put((rank, mine, t, s))
        elif mode == "dead_peer":
            if rank == 1:
                raise SystemExit(0)  # leaves between steps, before the collective
            try:
                replicas.max_over_ranks(1.0)
                q.put((rank, "no error"))
            except Exception as exc:  # the peer never joins: the collective errors out
                q.put((rank, type(exc).__name__))
    finally:
        if dist.is_initialized():
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def _run(mode, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    for p in procs:
        p.join(60)
        if p.is_alive():
            p.kill()
    while not q.empty():
        out.append(q.get())
    return out


def test_shard_partition_properties():
    for n in (0, 1, 7, 10, 256):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shard(n, r, world)]
            assert got == list(range(n))
            sizes = [len(shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)
    assert len({replica_seed(7, r) for r in range(8)}) == 8


def test_gloo_two_ranks_max_and_partition():
    out = sorted(_run("ok"))
    assert len(out) == 2
    (r0, m0, t0, s0), (r1, m1, t1, s1) = out
    assert m0 + m1 == list(range(10))
    assert t0 == t1 == 2.5          # max over ranks of 1.5 + rank
    assert s0 == s1 == 10.0


def test_gloo_dead_peer_is_detected_by_timeout():
    out = _run("dead_peer")
    assert out and out[0][0] == 0
    assert out[0][1] != "no error"
