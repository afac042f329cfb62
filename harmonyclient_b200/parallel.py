"""Search over one index whose inverted lists are split across GPUs.

One process per GPU (torch.distributed, NCCL between GPUs).  Rank r holds the
contiguous list range ``list_ranges(nlist, world)[r]`` of a shared set of
centroids (trained once, broadcast from rank 0), so an index larger than one
GPU's memory is spread over several.  A search runs on every rank with the
same queries: each scans only its own share of every query's probed lists
(the other lists are empty on that rank), the per-rank top-k lists are
exchanged with one all-gather and merged on the device (``merge_topk``).  With
ranges in rank order the merged answer equals the single-GPU index's, ties
included.  This is the reference's vector partition across teams
(src/Index.cpp:288-325, with the per-team heaps forwarded and merged by the
master, src/Index.cpp:1133-1181), with the MPI transfers replaced by one
collective.
"""
import ctypes as C

import numpy as np

from . import _lib
from .index import METRIC_L2, Index, check


def list_ranges(nlist, world):
    """Contiguous, rank-ordered list ranges [lo, hi) covering 0..nlist-1."""
    if world < 1 or world > nlist:
        raise ValueError("need 1 <= world <= nlist")
    b = [nlist * r // world for r in range(world + 1)]
    return [(b[r], b[r + 1]) for r in range(world)]


def merge_topk(D, I, metric=METRIC_L2, stream=0):
    """Best k per query of parts top-k lists (torch CUDA tensors D [parts, n,
    k] float32 and I [parts, n, k] int64, each list best first)."""
    import torch
    parts, n, k = D.shape
    oD = torch.empty((n, k), dtype=torch.float32, device=D.device)
    oI = torch.empty((n, k), dtype=torch.int64, device=D.device)
    D, I = D.contiguous(), I.contiguous()
    check(_lib.load().hy_merge_topk(C.c_void_p(D.data_ptr()), C.c_void_p(I.data_ptr()), parts, n, k, int(metric),
                                    C.c_void_p(oD.data_ptr()), C.c_void_p(oI.data_ptr()), C.c_void_p(stream)))
    return oD, oI


def gather_and_merge(D, I, group, merge):
    """The exchange step: all-gather every rank's (n, k) top-k into
    [world, n, k] (rank order) and merge.  `merge` maps (D, I) stacked that
    way to the final (D, I)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    gD = [torch.empty_like(D) for _ in range(world)]
    gI = [torch.empty_like(I) for _ in range(world)]
    dist.all_gather(gD, D.contiguous(), group=group)
    dist.all_gather(gI, I.contiguous(), group=group)
    return merge(torch.stack(gD), torch.stack(gI))


class ListShardedIndex:
    """This rank's shard of a list-partitioned index (see the module text)."""

    def __init__(self, d, nlist, nprobe, metric=METRIC_L2, group=None, device=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.metric = metric
        self.lo, self.hi = list_ranges(nlist, self.world)[self.rank]
        self.index = Index(d, nlist, nprobe, metric, device=device)
        self.index.set_list_range(self.lo, self.hi)

    def train(self, x):
        """Rank 0 trains the centroids; every rank receives them."""
        import torch
        import torch.distributed as dist
        if self.rank == 0:
            self.index.train(x)
            cent = torch.from_numpy(self.index.centroid_codes).cuda()
        else:
            cent = torch.empty((self.index.nlist, self.index.d), dtype=torch.float32, device="cuda")
        dist.broadcast(cent, 0, group=self.group)
        self.index.centroid_codes = cent.cpu().numpy()

    def add(self, x):
        """Every rank passes the whole base; each keeps its own lists."""
        self.index.add(x)

    def search_device(self, dq, k):
        """Search device queries dq (n x d, torch CUDA) on every rank; returns
        the merged (D, I) as torch CUDA tensors.  Everything runs on torch's
        current stream, the stream the collective is ordered on."""
        import torch
        stream = torch.cuda.current_stream().cuda_stream
        n = dq.shape[0]
        dD = torch.empty((n, k), dtype=torch.float32, device=dq.device)
        dI = torch.empty((n, k), dtype=torch.int64, device=dq.device)
        self.index.search_device(n, dq.data_ptr(), k, dD.data_ptr(), dI.data_ptr(), stream)
        return gather_and_merge(dD, dI, self.group, lambda D, I: merge_topk(D, I, self.metric, stream))

    def search(self, q, k):
        import torch
        dq = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float32)).cuda()
        D, I = self.search_device(dq, k)
        return D.cpu().numpy(), I.cpu().numpy()
