"""The multi-GPU path of this library is independent replicas (no collective
on the data path): the rank bookkeeping, the partition of independent
systems and the max-over-ranks timing reduction of qbx.replicas, run here as
two gloo processes on the CPU."""
import os
import socket

import pytest

from qbx import replicas


@pytest.mark.parametrize("n,world", [(32, 1), (32, 2), (32, 3), (7, 4), (3, 8)])
def test_shard_partitions(n, world):
    parts = [replicas.shard(n, r, world) for r in range(world)]
    flat = [i for p in parts for i in p]
    assert sorted(flat) == list(range(n))
    sizes = [len(p) for p in parts]
    assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from qbx import replicas as rp
    rp.init("gloo", timeout_s=60)
    r, w, _ = rp.dist_env()
    idx = rp.shard(32, r, w)
    m = rp.max_over_ranks(10.0 + r)
    rp.barrier()
    q.put((r, idx, m))
    rp.finalize()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[0] for o in out] == [0, 1]
    assert sorted(out[0][1] + out[1][1]) == list(range(32))
    assert all(o[2] == 11.0 for o in out)
