"""Parameters and seeded inputs of the golden cases (shared by the fixture
generator and the tests)."""
import numpy as np

from harmonyclient_b200 import datasets

CASES = {
    # BASELINE config 1 exactly: 10k x 128 gmm, nlist 100, nprobe 10, k 10.
    "c1": dict(kind="gmm_float", nb=10_000, nq=100, d=128, nlist=100, nprobe=10, k=10, metric=1, seed=0),
    # Config-2-shaped but small: integer-valued [0,255] data, k 100.
    "int_small": dict(kind="gmm_uint8", nb=20_000, nq=100, d=128, ncomp=256, nlist=64, nprobe=8, k=100, metric=1,
                      seed=1),
    # index_test.cpp:124-192 analogue: inner product on L2-normalised rows.
    "ip_small": dict(kind="normal_unit", nb=5_000, nq=50, d=32, nlist=50, nprobe=5, k=10, metric=0, seed=2),
    # index_test.cpp:71-122 analogue: nprobe = nlist is exhaustive.
    "exhaustive": dict(kind="uniform", nb=20_000, nq=50, d=16, nlist=141, nprobe=141, k=10, metric=1, seed=3),
    # Odd dimension (not a multiple of 4 or of 4 blocks).
    "odd_dim": dict(kind="gmm_float", nb=3_000, nq=40, d=21, nlist=30, nprobe=6, k=7, metric=1, seed=4),
    # Inner product with the reference's OPT_TRIANGLE cos-bound window
    # (src/Index.cpp:1509-1546) on unit-norm rows and queries.
    # Clustered unit-norm data, so that rows sit close to their centroid and
    # the window excludes most rows of the lists a query probes far away.
    "ip_tri": dict(kind="sphere_gmm", nb=20_000, nq=200, d=32, nlist=50, nprobe=10, k=10, metric=0, seed=6,
                   opt_level=1),
    # A tiny index written to disk by the reference (format fixture).
    "tiny_file": dict(kind="gmm_float", nb=500, nq=0, d=8, nlist=8, nprobe=4, k=5, metric=1, seed=5),
}


def data(name):
    c = CASES[name]
    rng = np.random.default_rng(c["seed"])
    if c["kind"] == "gmm_float":
        x, q = datasets.gmm_float(c["nb"], max(c["nq"], 1), d=c["d"], ncomp=min(100, c["nb"] // 20), seed=c["seed"])
    elif c["kind"] == "gmm_uint8":
        x, q = datasets.gmm_uint8(c["nb"], c["nq"], d=c["d"], ncomp=c["ncomp"], seed=c["seed"])
    elif c["kind"] == "normal_unit":
        x = rng.standard_normal((c["nb"] + c["nq"], c["d"])).astype(np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        x, q = x[: c["nb"]], x[c["nb"]:]
    elif c["kind"] == "sphere_gmm":
        # one random unit direction per list, rows = direction + 0.05 N(0, I),
        # normalised
        cen = rng.standard_normal((c["nlist"], c["d"])).astype(np.float32)
        cen /= np.linalg.norm(cen, axis=1, keepdims=True)
        comp = rng.integers(0, c["nlist"], c["nb"] + c["nq"])
        x = cen[comp] + np.float32(0.05) * rng.standard_normal((c["nb"] + c["nq"], c["d"])).astype(np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        x, q = x[: c["nb"]], x[c["nb"]:]
    elif c["kind"] == "uniform":
        x = rng.uniform(0, 1, (c["nb"] + c["nq"], c["d"])).astype(np.float32)
        x, q = x[: c["nb"]], x[c["nb"]:]
    else:
        raise ValueError(c["kind"])
    return np.ascontiguousarray(x), np.ascontiguousarray(q[: c["nq"]])
