"""CPU restatement of the list-partitioned search's merge step — TEST
INFRASTRUCTURE ONLY (the engine merges with its own kernel).

merge_parts(D, I, metric): per query, the best k of parts top-k lists
([parts][n][k], best first), ordered by (score, part, rank) so that equal
distances keep the parts' order and then each part's own order; unfilled
entries (id -1) come last as FLT_MAX (L2) / -FLT_MAX (IP) with id -1.
"""
import numpy as np

METRIC_IP, METRIC_L2 = 0, 1
FLT_MAX = np.float32(3.4028234663852886e38)


def merge_parts(D, I, metric=METRIC_L2):
    D = np.asarray(D, np.float32)
    I = np.asarray(I, np.int64)
    parts, n, k = D.shape
    oD = np.empty((n, k), np.float32)
    oI = np.empty((n, k), np.int64)
    for q in range(n):
        cand = []
        for p in range(parts):
            for r in range(k):
                if I[p, q, r] >= 0:
                    sc = D[p, q, r] if metric == METRIC_L2 else -D[p, q, r]
                    cand.append((float(sc), p, r))
        cand.sort()
        for i in range(k):
            if i < len(cand):
                _, p, r = cand[i]
                oD[q, i], oI[q, i] = D[p, q, r], I[p, q, r]
            else:
                oD[q, i] = FLT_MAX if metric == METRIC_L2 else -FLT_MAX
                oI[q, i] = -1
    return oD, oI
