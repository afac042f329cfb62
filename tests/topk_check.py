"""Tie-aware comparison of top-k results.

Two result rows agree when (1) their sorted distance lists agree within
`rtol` (exactly when rtol == 0), and (2) the ids whose distance is clearly
better than the k-th distance (below kth*(1 - 2*rtol), or strictly below it
when rtol == 0) are the same set in both.  Ids tied with the k-th distance
may legitimately differ: which of several equal candidates survives depends
on the heap's internal order in the reference."""
import numpy as np


def row_agree(Da, Ia, Db, Ib, rtol, metric=1):
    Da, Db = np.asarray(Da, np.float64), np.asarray(Db, np.float64)
    if metric == 1:
        fin = Da < 3e38
    else:
        fin = Da > -3e38
    if not np.array_equal(fin, (Db < 3e38) if metric == 1 else (Db > -3e38)):
        return False, "different number of filled entries"
    a, b = Da[fin], Db[fin]
    if rtol == 0:
        if not np.array_equal(a, b):
            return False, f"distances differ: {a[:5]} vs {b[:5]}"
    else:
        if not np.allclose(a, b, rtol=rtol, atol=1e-6 * max(1.0, float(np.max(np.abs(a))) if a.size else 1.0)):
            return False, f"distances differ beyond rtol: max rel {np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-30))}"
    if a.size == 0:
        return True, ""
    kth = a[-1]
    if metric == 1:
        margin = kth * (1 - 2 * rtol) if rtol else kth
        sa = set(Ia[fin][a < margin].tolist()) if rtol == 0 else set(Ia[fin][a < margin].tolist())
        sb = set(Ib[fin][b < margin].tolist())
    else:
        margin = kth + abs(kth) * 2 * rtol if rtol else kth
        sa = set(Ia[fin][a > margin].tolist())
        sb = set(Ib[fin][b > margin].tolist())
    if sa != sb:
        return False, f"id sets differ below the k-th distance: {sorted(sa ^ sb)[:6]}"
    return True, ""


def assert_topk_equal(Da, Ia, Db, Ib, rtol=0.0, metric=1, skip_rows=()):
    bad = []
    for r in range(Da.shape[0]):
        if r in skip_rows:
            continue
        ok, why = row_agree(Da[r], Ia[r], Db[r], Ib[r], rtol, metric)
        if not ok:
            bad.append((r, why))
    assert not bad, f"{len(bad)} rows disagree, first: {bad[:3]}"


def probe_tied_rows(q, cent, probes, metric=1, rel=1e-5):
    """Rows whose nprobe-th and (nprobe+1)-th centroid distances are within
    `rel` in FP64: their probe set may legitimately flip between FP32
    summation orders."""
    q64, c64 = q.astype(np.float64), cent.astype(np.float64)
    npb = probes.shape[1]
    out = set()
    if npb >= cent.shape[0]:
        return out
    for i in range(q.shape[0]):
        if metric == 1:
            dd = ((c64 - q64[i]) ** 2).sum(1)
            s = np.sort(dd)
            if s[npb] - s[npb - 1] <= rel * max(s[npb], 1e-30):
                out.add(i)
        else:
            dd = -(c64 @ q64[i])
            s = np.sort(dd)
            if s[npb] - s[npb - 1] <= rel * max(abs(s[npb]), 1e-30):
                out.add(i)
    return out


def recall_at(I, I_true, k):
    hits = 0
    for a, b in zip(I[:, :k], I_true[:, :k]):
        hits += len(set(a.tolist()) & set(b.tolist()))
    return hits / (I.shape[0] * k)
