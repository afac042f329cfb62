"""Seeded synthetic workloads shaped like the configurations this engine is
measured on.  The datasets the reference names (sift1m, msong, nuswide, …)
are not available offline, so Gaussian mixtures of the same shapes and value
ranges stand in for them.  Every generator is deterministic in its seed.

* ``c1`` — 10,000 x 128 float32 from a 100-component isotropic mixture
  (centres U[0,100], sigma 8, clipped at 0); 100 queries; nlist 100,
  nprobe 10, k 10.
* ``c2`` — 1,000,000 x 128 integer-valued float32 in [0,255] from a
  4,096-component mixture (centres U[0,255], sigma 20, rounded and clipped);
  10,000 queries; nlist 1024, nprobe 16/64/256, k 100.
* ``c3`` — 1,000,000 x 420 from a 2,048-component mixture (per-dim mean
  U[-1,1], sigma 0.3); 10,000 queries; nlist 2048, nprobe 64.
* ``c4`` — ``c2``'s generator with 16,384 components weighted Zipf(1.1);
  65,536 queries with per-query nprobe U[8,128]; nlist 16,384, k 10.
* ``c5`` — 2,000,000 x 500 sparse non-negative (2,048 components, 10% of dims
  non-zero per component, Exp(1) values), L2-normalised; 20,000 queries;
  nlist 4096, k 10.
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    base: np.ndarray
    queries: np.ndarray
    nlist: int
    nprobe: int
    k: int
    metric: int = 1  # METRIC_L2
    extra: dict = field(default_factory=dict)


def _mixture(rng, n, centres, sigma, weights=None, chunk=1 << 18):
    ncomp, d = centres.shape
    comp = rng.choice(ncomp, size=n, p=weights) if weights is not None else rng.integers(0, ncomp, size=n)
    out = np.empty((n, d), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        out[s:e] = centres[comp[s:e]] + np.float32(sigma) * rng.standard_normal((e - s, d), dtype=np.float32)
    return out


def gmm_float(n, nq, d=128, ncomp=100, lo=0.0, hi=100.0, sigma=8.0, seed=0):
    """Isotropic mixture with uniform centres, clipped at 0 (config c1)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(lo, hi, size=(ncomp, d)).astype(np.float32)
    x = np.maximum(_mixture(rng, n, centres, sigma), 0.0)
    q = np.maximum(_mixture(rng, nq, centres, sigma), 0.0)
    return x, q


def gmm_uint8(n, nq, d=128, ncomp=4096, sigma=20.0, seed=0, zipf=None, query_seed=None):
    """Integer-valued mixture in [0,255] (configs c2 and, with zipf, c4).
    With query_seed the queries are drawn from the same mixture by their own
    generator (other query sets over the same base; n may then be 0)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 255.0, size=(ncomp, d)).astype(np.float32)
    w = None
    if zipf is not None:
        w = 1.0 / np.arange(1, ncomp + 1, dtype=np.float64) ** zipf
        w /= w.sum()
    x = _mixture(rng, n, centres, sigma, w)
    np.clip(np.rint(x, out=x), 0, 255, out=x)
    q = _mixture(rng if query_seed is None else np.random.default_rng(query_seed), nq, centres, sigma, w)
    np.clip(np.rint(q, out=q), 0, 255, out=q)
    return x, q


def gmm_dense(n, nq, d=420, ncomp=2048, sigma=0.3, seed=0, query_seed=None):
    """Mixture with per-dimension means U[-1,1] (config c3); query_seed as
    in gmm_uint8."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-1.0, 1.0, size=(ncomp, d)).astype(np.float32)
    x = _mixture(rng, n, centres, sigma)
    q = _mixture(rng if query_seed is None else np.random.default_rng(query_seed), nq, centres, sigma)
    return x, q


def sparse_nonneg(n, nq, d=500, ncomp=2048, density=0.1, seed=0, chunk=1 << 17, query_seed=None):
    """Sparse non-negative rows, L2-normalised (config c5): each component owns
    a random support of density*d dims; a row draws Exp(1) values on its
    component's support.  query_seed as in gmm_uint8."""
    rng = np.random.default_rng(seed)
    nnz = max(1, int(round(density * d)))
    supports = np.stack([rng.choice(d, size=nnz, replace=False) for _ in range(ncomp)])

    def draw(m, g):
        comp = g.integers(0, ncomp, size=m)
        out = np.zeros((m, d), np.float32)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            vals = g.exponential(1.0, size=(e - s, nnz)).astype(np.float32)
            rows = np.arange(e - s)[:, None]
            out[s:e][rows, supports[comp[s:e]]] = vals
            nr = np.linalg.norm(out[s:e], axis=1, keepdims=True)
            out[s:e] /= np.maximum(nr, 1e-30)
        return out

    x = draw(n, rng)
    return x, draw(nq, rng if query_seed is None else np.random.default_rng(query_seed))


def c1(seed=0):
    x, q = gmm_float(10_000, 100, seed=seed)
    return Workload("c1: 10k x 128 gmm, nlist 100, nprobe 10, k 10", x, q, nlist=100, nprobe=10, k=10)


def c2(seed=0, nb=1_000_000, nq=10_000, nprobe=64, k=100):
    x, q = gmm_uint8(nb, nq, seed=seed)
    return Workload(f"c2: {nb} x 128 uint8-valued gmm, nlist 1024, nprobe {nprobe}, k {k}", x, q, nlist=1024,
                    nprobe=nprobe, k=k)


def c3(seed=0, nb=1_000_000, nq=10_000, k=10):
    x, q = gmm_dense(nb, nq, seed=seed)
    return Workload(f"c3: {nb} x 420 gmm, nlist 2048, nprobe 64, k {k}", x, q, nlist=2048, nprobe=64, k=k)


def c4(seed=0, nb=10_000_000, nq=65_536):
    x, q = gmm_uint8(nb, nq, ncomp=16_384, seed=seed, zipf=1.1)
    rng = np.random.default_rng(seed + 1)
    nprobe = rng.integers(8, 129, size=nq).astype(np.int32)
    return Workload(f"c4: {nb} x 128 zipf gmm, nlist 16384, nprobe U[8,128], k 10", x, q, nlist=16_384, nprobe=128,
                    k=10, extra={"nprobe_per_query": nprobe})


def c5(seed=0, nb=2_000_000, nq=20_000):
    x, q = sparse_nonneg(nb, nq, seed=seed)
    return Workload(f"c5: {nb} x 500 sparse, nlist 4096, k 10", x, q, nlist=4096, nprobe=256, k=10)
