"""Generates the golden fixtures in this directory by running the REFERENCE's
own code (oracle/_ref, compiled unmodified from the Harmony sources).

    make -C oracle ref && python tests/golden/make_golden.py [case ...]

Inputs are not stored: every case regenerates its data from a numpy seed
(harmonyclient_b200.datasets / numpy.random.default_rng), and the fixture
keeps only the reference's outputs plus the parameters.  The reference runs
with one OpenMP thread so its k-means float accumulation is deterministic.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from tests.golden import cases  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def heap_kat():
    """heap_test.cpp:7-91: top-20 of 100 uniform values through the heap, for
    the max-heap (L2) and the min-heap (IP)."""
    rng = np.random.default_rng(7)
    vals = rng.uniform(0, 1, 100).astype(np.float32)
    ids = np.arange(100, dtype=np.int64)
    out = {"vals": vals}
    for m, name in ((1, "l2"), (0, "ip")):
        v, i = ref.heap_topk(m, vals, ids, 20)
        out[f"{name}_v"], out[f"{name}_i"] = v, i
    np.savez(os.path.join(OUT, "heap_kat.npz"), **out)


def ivf_case(name):
    c = cases.CASES[name]
    x, q = cases.data(name)
    R = ref.RefIndex(c["d"], c["nlist"], c["nprobe"], c["metric"])
    R.train(x)
    cent = R.centroids()
    if c.get("opt_level"):
        R.set_opt_level(c["opt_level"])
    R.add(x)
    D, I = R.search(q, c["k"])
    P = R.probes(q)
    sizes = np.array([R.list_size(l) for l in range(c["nlist"])], np.int64)
    out = dict(centroids=cent, D=D, I=I, probes=P, list_sizes=sizes)
    l0 = int(np.argmax(sizes))
    out["big_list"] = np.int64(l0)
    out["big_list_ids"] = R.get_list(l0)[0]
    if c["metric"] == 1:
        tops = R.warmup_tops(q, c["k"], P, 10, c["k"])
        Dp, Ip = R.search_prune(q, c["k"], P, tops)
        out.update(tops=tops, Dp=Dp, Ip=Ip)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    return R


def index_file():
    """A small .index file written by the reference's Index::save_index."""
    c = cases.CASES["tiny_file"]
    x, _ = cases.data("tiny_file")
    R = ref.RefIndex(c["d"], c["nlist"], c["nprobe"], c["metric"])
    R.train(x)
    R.add(x)
    R.save(os.path.join(OUT, "tiny_ref.index"))
    q = x[:16]
    D, I = R.search(q, 5)
    np.savez(os.path.join(OUT, "tiny_ref_search.npz"), D=D, I=I)


if __name__ == "__main__":
    # With case names as arguments only those fixtures are written.
    ref.set_threads(1)
    only = sys.argv[1:]
    if not only:
        heap_kat()
    for n in cases.CASES:
        if n != "tiny_file" and (not only or n in only):
            ivf_case(n)
            print("wrote", n)
    if not only:
        index_file()
    print("done")
