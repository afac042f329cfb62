"""FP64 brute-force search on the GPU (torch), the recall oracle of the
measurement at full size — TEST AND MEASUREMENT INFRASTRUCTURE ONLY (bench.py
and tests use it to score results; the engine never calls it).

Distances are |q|^2 + |x|^2 - 2 q.x in float64 for the ranking (exact for
integer-valued data below 2^26 per term), and sum((q - x)^2) in float64 for the
returned rows.
"""
import numpy as np

METRIC_IP, METRIC_L2 = 0, 1


def topk(x, q, k, metric=METRIC_L2, chunk=128, device="cuda"):
    """Exact top-k (ids, float64 distances) of every query; L2 ascending, IP
    descending (distance = inner product)."""
    import torch
    X = torch.from_numpy(np.ascontiguousarray(x)).to(device=device, dtype=torch.float64)
    xn = (X * X).sum(1)
    I = np.empty((q.shape[0], k), np.int64)
    D = np.empty((q.shape[0], k), np.float64)
    for s in range(0, q.shape[0], chunk):
        Q = torch.from_numpy(np.ascontiguousarray(q[s:s + chunk])).to(device=device, dtype=torch.float64)
        ip = Q @ X.T
        if metric == METRIC_L2:
            dist = (Q * Q).sum(1, keepdim=True) + xn[None, :] - 2.0 * ip
            v, i = torch.topk(dist, k, dim=1, largest=False)
        else:
            v, i = torch.topk(ip, k, dim=1, largest=True)
        I[s:s + chunk] = i.cpu().numpy()
        D[s:s + chunk] = v.cpu().numpy()
        del ip
    return D, I


def exact_distances(x, q, I, metric=METRIC_L2, device="cuda"):
    """float64 distance of every (query, returned row) pair; NaN where the id
    is -1."""
    import torch
    X = torch.from_numpy(np.ascontiguousarray(x)).to(device=device, dtype=torch.float64)
    out = np.full(I.shape, np.nan)
    for s in range(0, q.shape[0], 256):
        Q = torch.from_numpy(np.ascontiguousarray(q[s:s + 256])).to(device=device, dtype=torch.float64)
        ids = torch.from_numpy(np.maximum(I[s:s + 256], 0)).to(device)
        R = X[ids]  # (b, k, d)
        if metric == METRIC_L2:
            v = ((Q[:, None, :] - R) ** 2).sum(-1)
        else:
            v = (Q[:, None, :] * R).sum(-1)
        v = v.cpu().numpy()
        v[I[s:s + 256] < 0] = np.nan
        out[s:s + 256] = v
    return out


def score(D, I, Dt, It, x, q, at=10, metric=METRIC_L2):
    """recall@at of (D, I) against the exact top-k (Dt, It), and the relative
    error of every returned distance against its float64 value."""
    at = min(at, I.shape[1], It.shape[1])
    rec = float(np.mean([len(set(a[:at]) & set(b[:at])) / at for a, b in zip(I.tolist(), It.tolist())]))
    ex = exact_distances(x, q, I, metric)
    ok = ~np.isnan(ex)
    rel = np.abs(D[ok].astype(np.float64) - ex[ok]) / np.maximum(np.abs(ex[ok]), 1e-30)
    return {"recall": rec, "dist_rel_err_max": float(rel.max()) if rel.size else 0.0,
            "dist_rel_err_mean": float(rel.mean()) if rel.size else 0.0}
