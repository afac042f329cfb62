"""ctypes binding of oracle/_build/libhy_oracle.so — this project's CPU
restatement of the reference algorithm (oracle/hy_oracle.cpp).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "libhy_oracle.so")
_lib = None

METRIC_IP, METRIC_L2 = 0, 1


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "lib"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    L = C.CDLL(LIB)
    sz, vp = C.c_size_t, C.c_void_p
    L.oc_l2.argtypes = [vp, vp, sz]
    L.oc_l2.restype = C.c_float
    L.oc_ip.argtypes = [vp, vp, sz]
    L.oc_ip.restype = C.c_float
    L.oc_heap_topk.argtypes = [C.c_int, sz, vp, vp, sz, vp, vp]
    L.oc_probes.argtypes = [sz, vp, sz, vp, sz, C.c_int, sz, vp, vp]
    L.oc_assign.argtypes = [sz, vp, sz, vp, sz, C.c_int, vp, vp]
    L.oc_build_lists.argtypes = [sz, sz, C.c_int, vp, vp, vp, vp]
    L.oc_scan_probes.argtypes = [sz, vp, sz, vp, vp, vp, C.c_int, sz, vp, sz, vp, vp]
    L.oc_warmup_tops.argtypes = [sz, vp, sz, vp, vp, sz, vp, sz, sz, sz, vp]
    L.oc_scan_prune.argtypes = [sz, vp, sz, vp, vp, vp, sz, vp, vp, sz, sz, vp, vp, vp]
    L.oc_kmeans.argtypes = [sz, vp, sz, sz, C.c_int, C.c_int, sz, C.c_int, C.c_int, vp]
    L.oc_bruteforce_f64.argtypes = [sz, vp, sz, vp, sz, C.c_int, sz, vp, vp]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _i64(a):
    return np.ascontiguousarray(a, np.int64)


def heap_topk(metric, vals, ids, k):
    vals, ids = _f32(vals), _i64(ids)
    ov, oi = np.empty(k, np.float32), np.empty(k, np.int64)
    load().oc_heap_topk(metric, vals.size, _p(vals), _p(ids), k, _p(ov), _p(oi))
    return ov, oi


def probes(q, cent, nprobe, metric=METRIC_L2):
    q, cent = _f32(q), _f32(cent)
    nprobe = min(nprobe, cent.shape[0])
    P = np.empty((q.shape[0], nprobe), np.int64)
    Pd = np.empty((q.shape[0], nprobe), np.float32)
    load().oc_probes(q.shape[0], _p(q), cent.shape[0], _p(cent), q.shape[1], metric, nprobe, _p(P), _p(Pd))
    return P, Pd


def assign(x, cent, metric=METRIC_L2):
    x, cent = _f32(x), _f32(cent)
    lab = np.empty(x.shape[0], np.int64)
    dis = np.empty(x.shape[0], np.float32)
    load().oc_assign(x.shape[0], _p(x), cent.shape[0], _p(cent), x.shape[1], metric, _p(lab), _p(dis))
    return lab, dis


class Lists:
    """Inverted lists in CSR form: offsets[nlist+1], ids[nb], codes[nb, d]."""

    def __init__(self, offsets, ids, codes):
        self.offsets, self.ids, self.codes = _i64(offsets), _i64(ids), _f32(codes)

    @property
    def nlist(self):
        return self.offsets.size - 1

    def list(self, l):
        a, b = self.offsets[l], self.offsets[l + 1]
        return self.ids[a:b], self.codes[a:b]


def build_lists(x, cent, metric=METRIC_L2):
    """Index::add: assign rows, size lists, order rows by distance to centroid."""
    x = _f32(x)
    lab, dis = assign(x, cent, metric)
    nlist = cent.shape[0]
    off = np.empty(nlist + 1, np.int64)
    order = np.empty(x.shape[0], np.int64)
    load().oc_build_lists(x.shape[0], nlist, metric, _p(lab), _p(dis), _p(off), _p(order))
    return Lists(off, order, x[order])


def scan_probes(q, lists, P, k, metric=METRIC_L2):
    q, P = _f32(q), _i64(P)
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    load().oc_scan_probes(q.shape[0], _p(q), q.shape[1], _p(lists.offsets), _p(lists.ids), _p(lists.codes), metric,
                          P.shape[1], _p(P), k, _p(D), _p(I))
    return D, I


def search(q, cent, lists, nprobe, k, metric=METRIC_L2):
    P, _ = probes(q, cent, nprobe, metric)
    return scan_probes(q, lists, P, k, metric)


def warmup_tops(q, lists, P, k, warmup_list=10, warmup_list_size=None):
    q, P = _f32(q), _i64(P)
    if warmup_list_size is None:
        warmup_list_size = k
    t = np.empty(q.shape[0], np.float32)
    load().oc_warmup_tops(q.shape[0], _p(q), q.shape[1], _p(lists.offsets), _p(lists.codes), P.shape[1], _p(P), k,
                          warmup_list, warmup_list_size, _p(t))
    return t


def scan_prune(q, lists, P, tops, k, nblocks=4):
    q, P, tops = _f32(q), _i64(P), _f32(tops)
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    sk = C.c_int64()
    load().oc_scan_prune(q.shape[0], _p(q), q.shape[1], _p(lists.offsets), _p(lists.ids), _p(lists.codes), P.shape[1],
                         _p(P), _p(tops), k, nblocks, _p(D), _p(I), C.byref(sk))
    return D, I, sk.value


def kmeans(x, nlist, niter=20, seed=6666, max_points_per_centroid=256, metric=METRIC_L2, fp64=True):
    x = _f32(x)
    c = np.empty((nlist, x.shape[1]), np.float32)
    load().oc_kmeans(x.shape[0], _p(x), x.shape[1], nlist, niter, seed, max_points_per_centroid, metric, int(fp64),
                     _p(c))
    return c


def bruteforce_f64(x, q, k, metric=METRIC_L2):
    x, q = _f32(x), _f32(q)
    D = np.empty((q.shape[0], k), np.float64)
    I = np.empty((q.shape[0], k), np.int64)
    load().oc_bruteforce_f64(x.shape[0], _p(x), q.shape[0], _p(q), x.shape[1], metric, k, _p(D), _p(I))
    return D, I
