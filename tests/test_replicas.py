"""Replica host logic on CPU: two gloo ranks on 127.0.0.1 (no GPU).

Covers what the multi-GPU bench relies on: the max-over-ranks timing
reduction, the barrier, the member sharding, and a rank that fails before a
collective ending its peer's wait with an error rather than a hang."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from suetes_b200 import replicas
    try:
        w, r, _ = replicas.init(backend="gloo", timeout_s=10)
        if r == fail_rank:
            raise SystemExit(0)  # leaves before the collective
        m = replicas.max_over_ranks(10.0 * (r + 1), w)
        replicas.barrier(w)
        q.put((r, "ok", m, list(replicas.shard(7, r, w))))
        replicas.finalize(w)
    except SystemExit:
        q.put((rank, "left", None, None))
    except Exception as e:  # the peer's collective must fail, not hang
        q.put((rank, "error", type(e).__name__, None))


def _run(world, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_two_rank_max_barrier_and_shard():
    out = _run(2)
    assert [o[1] for o in out] == ["ok", "ok"]
    assert all(o[2] == 20.0 for o in out)
    shards = [o[3] for o in out]
    assert shards[0] + shards[1] == list(range(7)) and abs(len(shards[0]) - len(shards[1])) <= 1


def test_rank_leaving_ends_peer_collective_with_error():
    out = _run(2, fail_rank=1)
    assert out[1][1] == "left"
    assert out[0][1] == "error"


def test_shard_covers_every_unit_once():
    from suetes_b200.replicas import shard
    for n in (0, 1, 5, 32, 33):
        for world in (1, 2, 3, 8):
            got = [u for r in range(world) for u in shard(n, r, world)]
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)
