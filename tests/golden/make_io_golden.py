"""Generates the dataset / result-file / recall fixtures in tests/golden/io/
by running the REFERENCE's own readers and metrics (src/utils.h, through
oracle/_ref compiled unmodified from the Harmony sources).

    make -C oracle ref && python tests/golden/make_io_golden.py

The small input files are written here from numpy seeds and kept with the
reference's outputs: io/a.fvecs, io/b.bvecs (the reference's layout),
io/c.txt, the reference's own result files io/r.bin and io/r.txt, and
io/expected.npz (loaded rows, file info, recall values).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from harmonyclient_b200 import datafiles as io  # noqa: E402
from oracle import ref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "io")


def recall_cases(rng):
    """(name, I, D, GT, GD, nq, k, metric, gt_k) cases with -1 padding,
    ties at the k-th distance, gt_k > k and both metrics."""
    out = []
    for c in range(8):
        nq, k = int(rng.integers(2, 6)), int(rng.integers(2, 8))
        gt_k = k + (c % 3)
        metric = c % 2
        GT = np.stack([rng.permutation(40)[:gt_k] for _ in range(nq)]).astype(np.int64)
        GD = np.sort(rng.uniform(1, 10, (nq, gt_k)).astype(np.float32), axis=1)
        if metric == 0:
            GD = -GD
        I = np.where(rng.uniform(0, 1, (nq, k)) < 0.6, GT[:, :k], rng.integers(0, 40, (nq, k))).astype(np.int64)
        D = np.abs(GD[:, :k] + rng.normal(0, 0.5, (nq, k)).astype(np.float32))
        if c == 3:
            I[0, k - 1] = -1  # a short result list
            D[1, 0] = GD[1, k - 1]  # a tie at the k-th ground-truth distance
        if c == 5:
            D[0, 0] = -1.0  # the reference returns 0 for a negative first distance
        out.append((f"case{c}", I, D.astype(np.float32), GT, GD.astype(np.float32), nq, k, metric, gt_k))
    return out


def main():
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(11)
    exp = {}
    x = rng.normal(0, 3, (7, 5)).astype(np.float32)
    io.write_fvecs(os.path.join(OUT, "a.fvecs"), x)
    b = rng.integers(0, 256, (6, 8)).astype(np.uint8)
    io.write_bvecs(os.path.join(OUT, "b.bvecs"), b)
    with open(os.path.join(OUT, "c.txt"), "w") as f:
        for i in range(4):
            f.write(",".join([str(100 + i)] + [f"{v:.4f}" for v in rng.normal(0, 1, 3)]) + "\n")
    for name in ("a.fvecs", "b.bvecs", "c.txt"):
        p = os.path.join(OUT, name)
        exp[f"{name}_info"] = np.array(ref.xvecs_info(p), np.int64)
        exp[f"{name}_all"] = ref.load_xvecs(p)
        if not name.endswith(".txt"):
            exp[f"{name}_2_4"] = ref.load_xvecs(p, 2, 4)
    labels = rng.integers(-1, 1000, (3, 4)).astype(np.int64)
    dist = rng.uniform(0, 50, (3, 4)).astype(np.float32)
    exp["res_labels"], exp["res_dist"] = labels, dist
    for ext in ("bin", "txt"):
        p = os.path.join(OUT, f"r.{ext}")
        ref.write_results(labels, dist, p)
        exp[f"r_{ext}_labels"], exp[f"r_{ext}_dist"] = ref.load_results(p, 3, 4)
    for name, I, D, GT, GD, nq, k, metric, gt_k in recall_cases(rng):
        exp[f"{name}_in"] = np.array([nq, k, metric, gt_k], np.int64)
        exp[f"{name}_I"], exp[f"{name}_D"], exp[f"{name}_GT"], exp[f"{name}_GD"] = I, D, GT, GD
        exp[f"{name}_out"] = np.array([ref.recall(w, I, D, GT, GD, nq, k, metric, gt_k) for w in range(3)],
                                      np.float32)
    np.savez(os.path.join(OUT, "expected.npz"), **exp)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
