"""Band-pair sharding bookkeeping on the CPU.

The library splits the band pairs of one cell over GPUs
(qbx_shard_pairs: contiguous ranges whose sizes differ by one at most), sums
the partial densities over the GPUs and broadcasts each GPU's H*psi bands to
the others.  Here two gloo processes play the GPUs: each computes, with the
oracle (oracle/qbox_np.py), the density and the local H*psi of the band
pairs the library's rule gives it, then the same collectives (an allreduce
of the density, a broadcast of each rank's band block) run over gloo.  The
results must equal the whole-cell oracle to 1e-12: this pins the partition
and the reduction bookkeeping that the NCCL path follows.
"""
import os
import socket

import numpy as np
import pytest

from qbx import capi, sharding, systems


@pytest.mark.parametrize("nst", [1, 2, 7, 16, 128, 1024, 1023])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_pair_ranges_cover_every_pair_once(nst, world):
    npairs = (nst + 1) // 2
    r = sharding.pair_ranges(nst, world)
    assert r[0][0] == 0 and r[-1][1] == npairs
    for (a, b), (c, _) in zip(r, r[1:]):
        assert b == c
    sizes = [b - a for a, b in r]
    assert max(sizes) - min(sizes) <= 1
    bands = sharding.band_ranges(nst, world)
    assert sum(b - a for a, b in bands) == nst


def test_pair_ranges_reject_bad_arguments():
    with pytest.raises(capi.QbxError):
        capi.shard_pairs(16, 2, 2)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from oracle import qbox_np
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = systems.si8()
        es = qbox_np.ElectronicStep(s)
        es.update_density()
        es.update_vhxc()
        nst = s.nbands
        b0, b1 = sharding.band_ranges(nst, world)[rank]
        # the partial density of this rank's bands
        rho = np.zeros(es.wgrid.N)
        for n in range(b0, b1):
            psi = es.wgrid.backward(es.c[n]).real.ravel()
            rho += es.occ[n] / es.omega * psi * psi
        t = torch.from_numpy(rho)
        dist.all_reduce(t)
        # the local H*psi of this rank's bands, the other blocks from their owners
        hc = np.zeros_like(es.c)
        v = es.v_r.ravel()
        for n in range(b0, b1):
            f = es.wgrid.backward(es.c[n]).ravel() * v
            hc[n] = es.wgrid.forward(f)
        h = torch.from_numpy(hc.view(np.float64).copy())
        for r, (a, b) in enumerate(sharding.band_ranges(nst, world)):
            blk = h[a:b].contiguous()
            dist.broadcast(blk, src=r)
            h[a:b] = blk
        ref_hc = np.zeros_like(es.c)
        es.rs_mul_add(es.v_r.ravel(), ref_hc)
        ok_rho = np.abs(t.numpy() - es.rhor.ravel()).max() < 1e-12 * np.abs(es.rhor).max()
        got = h.numpy().view(np.complex128)
        ok_hc = np.abs(got - ref_hc).max() < 1e-12 * max(1.0, np.abs(ref_hc).max())
        out.put((rank, bool(ok_rho), bool(ok_hc)))
    finally:
        dist.destroy_process_group()


def test_sharded_density_and_hpsi_on_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res) == [(0, True, True), (1, True, True)], res
