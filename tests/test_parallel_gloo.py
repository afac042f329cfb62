"""The list-partitioned search's host side on two CPU ranks (gloo): each rank
scans its contiguous list range (the oracle stands in for the GPU engine),
the exchange step all-gathers the per-rank top-k in rank order, and the merge
rule (score, then rank order, then each rank's own order) reproduces the
unpartitioned search exactly, ties included."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from harmonyclient_b200.parallel import gather_and_merge, list_ranges


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from harmonyclient_b200 import datasets
        from oracle import port as op
        from oracle import shard
        # Integer-valued data: many exactly equal distances, so ties matter.
        x, q = datasets.gmm_uint8(6000, 40, d=16, ncomp=30, sigma=6.0, seed=3)
        nlist, nprobe, k = 24, 8, 20
        cent = op.kmeans(x, nlist)
        lists = op.build_lists(x, cent)
        P, _ = op.probes(q, cent, nprobe)
        lo, hi = list_ranges(nlist, world)[rank]
        mine = np.where((P >= lo) & (P < hi), P, -1)
        D, I = op.scan_probes(q, lists, mine, k)
        Dm, Im = gather_and_merge(torch.from_numpy(D), torch.from_numpy(I), None,
                                  lambda a, b: tuple(map(torch.from_numpy, shard.merge_parts(a.numpy(), b.numpy()))))
        if rank == 0:
            Dr, Ir = op.scan_probes(q, lists, P, k)
            out.put((Dm.numpy(), Im.numpy(), Dr, Ir))
    finally:
        dist.destroy_process_group()


def test_list_partition_merge_equals_unpartitioned():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    Dm, Im, Dr, Ir = out.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    np.testing.assert_array_equal(Im, Ir)
    np.testing.assert_array_equal(Dm, Dr)


def test_list_ranges_cover_in_order():
    for nlist, world in [(10, 3), (1024, 8), (5, 5)]:
        r = list_ranges(nlist, world)
        assert r[0][0] == 0 and r[-1][1] == nlist
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert all(lo < hi for lo, hi in r)
