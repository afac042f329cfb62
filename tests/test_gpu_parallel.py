"""List partition on one GPU: indexes holding contiguous list ranges of the
same centroids, searched alone and merged with the engine's merge kernel,
return exactly the unpartitioned index's answer (plain and bf16 forms, L2 and
inner product)."""
import numpy as np
import pytest
import torch

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets
from harmonyclient_b200.parallel import list_ranges, merge_topk
from oracle import shard

pytestmark = pytest.mark.gpu


def _shards(x, cent, d, nlist, nprobe, metric, world):
    out = []
    for lo, hi in list_ranges(nlist, world):
        s = hb.Index(d, nlist, nprobe, metric)
        s.centroid_codes = cent
        s.set_list_range(lo, hi)
        s.add(x)
        out.append(s)
    return out


@pytest.mark.parametrize("metric", [hb.METRIC_L2, hb.METRIC_IP])
@pytest.mark.parametrize("form", ["plain", "bf16"])
@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_search_equals_whole_index(metric, form, world):
    x, q = datasets.gmm_uint8(30_000, 300, d=64, ncomp=200, sigma=15.0, seed=7)
    if metric == hb.METRIC_IP:
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    nlist, nprobe, k = 60, 12, 30
    whole = hb.Index(64, nlist, nprobe, metric)
    whole.train(x)
    whole.add(x)
    cent = whole.centroid_codes
    whole.set_form(form)
    D0, I0 = whole.search(q, k)
    parts = _shards(x, cent, 64, nlist, nprobe, metric, world)
    assert sum(p.info().ntotal for p in parts) == x.shape[0]
    Ds, Is = [], []
    for p in parts:
        p.set_form(form)
        D, I = p.search(q, k)
        Ds.append(D)
        Is.append(I)
    Dm, Im = merge_topk(torch.from_numpy(np.stack(Ds)).cuda(), torch.from_numpy(np.stack(Is)).cuda(), metric)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(Im.cpu().numpy(), I0)
    np.testing.assert_array_equal(Dm.cpu().numpy(), D0)
    # the engine's merge kernel follows the merge rule of the restatement
    Dr, Ir = shard.merge_parts(np.stack(Ds), np.stack(Is), metric)
    np.testing.assert_array_equal(Im.cpu().numpy(), Ir)


def test_list_range_rejects_bad_ranges():
    idx = hb.Index(8, 10, 2)
    with pytest.raises(hb.HyError):
        idx.set_list_range(5, 5)
    with pytest.raises(hb.HyError):
        idx.set_list_range(0, 11)
