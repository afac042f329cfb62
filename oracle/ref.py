"""ctypes binding of oracle/_ref/libharmony_ref_*.so — the reference's own code.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Build with
``make -C oracle ref`` where the reference sources are present; the built
``.so`` files are what travel to other machines.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return all(x in flags for x in ("avx512f", "avx512bw", "avx512dq", "avx512vl"))
    except OSError:
        return False


def lib_path():
    v = "v4" if _cpu_has_avx512() else "v3"
    return os.path.join(_HERE, "_ref", f"libharmony_ref_{v}.so")


def available():
    return os.path.exists(lib_path())


def load():
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not os.path.exists(p):
        raise RuntimeError(f"reference oracle library missing: {p} (run make -C oracle ref)")
    L = C.CDLL(p)
    sz, vp, fp, ip64 = C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p
    L.ref_last_error.restype = C.c_char_p
    L.ref_index_new.argtypes = [sz, sz, sz, C.c_int, C.POINTER(C.c_void_p)]
    L.ref_index_free.argtypes = [vp]
    L.ref_index_free.restype = None
    L.ref_set_threads.argtypes = [C.c_int]
    L.ref_train.argtypes = [vp, sz, fp, C.c_int]
    L.ref_set_centroids.argtypes = [vp, fp]
    L.ref_get_centroids.argtypes = [vp, fp]
    L.ref_set_nprobe.argtypes = [vp, sz]
    L.ref_set_opt_level.argtypes = [vp, C.c_int]
    L.ref_add.argtypes = [vp, sz, fp]
    L.ref_list_size.argtypes = [vp, sz, C.POINTER(C.c_size_t)]
    L.ref_get_list.argtypes = [vp, sz, ip64, fp, fp]
    L.ref_search_original.argtypes = [vp, sz, fp, sz, fp, ip64]
    L.ref_probes.argtypes = [vp, sz, fp, ip64]
    L.ref_warmup_tops.argtypes = [vp, sz, fp, sz, sz, sz, ip64, fp]
    L.ref_search_prune.argtypes = [vp, sz, fp, sz, ip64, fp, fp, ip64]
    L.ref_heap_topk.argtypes = [C.c_int, sz, fp, ip64, sz, fp, ip64]
    L.ref_search_group.argtypes = [vp, sz, fp, sz, C.c_int, C.c_int, C.c_int, C.c_int, sz, sz, C.c_int, C.c_int,
                                   C.c_char_p, fp, ip64, C.POINTER(C.c_double)]
    L.ref_save.argtypes = [vp, C.c_char_p]
    L.ref_load.argtypes = [vp, C.c_char_p]
    L.ref_info.argtypes = [vp] + [C.POINTER(C.c_size_t)] * 3 + [C.POINTER(C.c_int)]
    L.ref_xvecs_info.argtypes = [C.c_char_p, C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
    L.ref_load_xvecs.argtypes = [C.c_char_p, C.c_int, C.c_int, fp, sz, C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
    L.ref_write_results.argtypes = [ip64, fp, sz, sz, C.c_char_p]
    L.ref_load_results.argtypes = [C.c_char_p, ip64, fp, sz, sz]
    L.ref_recall.argtypes = [C.c_int, ip64, fp, ip64, fp, sz, sz, C.c_int, sz, C.POINTER(C.c_float)]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference oracle: " + load().ref_last_error().decode())


def set_threads(n):
    load().ref_set_threads(int(n))


def heap_topk(metric, vals, ids, k):
    vals = np.ascontiguousarray(vals, np.float32)
    ids = np.ascontiguousarray(ids, np.int64)
    ov = np.empty(k, np.float32)
    oi = np.empty(k, np.int64)
    _check(load().ref_heap_topk(metric, vals.size, _p(vals), _p(ids), k, _p(ov), _p(oi)))
    return ov, oi


class RefIndex:
    """The reference's harmony::Index, driven in-process."""

    def __init__(self, d, nlist, nprobe, metric=1):
        self.L = load()
        h = C.c_void_p()
        _check(self.L.ref_index_new(d, nlist, nprobe, metric, C.byref(h)))
        self.h = h
        self.d, self.nlist, self.nprobe, self.metric = d, nlist, nprobe, metric

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_index_free(self.h)
            self.h = None

    def train(self, x, lite=False):
        x = np.ascontiguousarray(x, np.float32)
        _check(self.L.ref_train(self.h, x.shape[0], _p(x), int(lite)))

    def set_centroids(self, c):
        c = np.ascontiguousarray(c, np.float32)
        assert c.shape == (self.nlist, self.d)
        _check(self.L.ref_set_centroids(self.h, _p(c)))

    def centroids(self):
        c = np.empty((self.nlist, self.d), np.float32)
        _check(self.L.ref_get_centroids(self.h, _p(c)))
        return c

    def set_nprobe(self, nprobe):
        self.nprobe = nprobe
        _check(self.L.ref_set_nprobe(self.h, nprobe))

    def set_opt_level(self, opt_level):
        _check(self.L.ref_set_opt_level(self.h, int(opt_level)))

    def add(self, x):
        x = np.ascontiguousarray(x, np.float32)
        _check(self.L.ref_add(self.h, x.shape[0], _p(x)))

    def list_size(self, l):
        s = C.c_size_t()
        _check(self.L.ref_list_size(self.h, l, C.byref(s)))
        return s.value

    def get_list(self, l):
        n = self.list_size(l)
        ids = np.empty(n, np.int64)
        codes = np.empty((n, self.d), np.float32)
        norms = np.empty(n, np.float32)
        if n:
            _check(self.L.ref_get_list(self.h, l, _p(ids), _p(codes), _p(norms)))
        return ids, codes, norms

    def search(self, q, k):
        q = np.ascontiguousarray(q, np.float32)
        D = np.empty((q.shape[0], k), np.float32)
        I = np.empty((q.shape[0], k), np.int64)
        _check(self.L.ref_search_original(self.h, q.shape[0], _p(q), k, _p(D), _p(I)))
        return D, I

    def search_group(self, q, k, workers=4, group=2, team=2, block=4, warmup_list=10, warmup_list_size=None,
                     cut=True, threads_per_rank=None, scratch_path=None):
        """The reference's GROUP mode with pruning (its default distributed
        mode), 1 master + `workers` ranks run as threads of this process.
        Returns (D, I, seconds of the master's search).  The reference needs
        nq <= 10000, divisible by group * block, and k <= 100."""
        import os
        import tempfile
        q = np.ascontiguousarray(q, np.float32)
        if warmup_list_size is None:
            warmup_list_size = k
        if threads_per_rank is None:
            threads_per_rank = max(1, (os.cpu_count() or 1) // (workers + 1))
        D = np.empty((q.shape[0], k), np.float32)
        I = np.empty((q.shape[0], k), np.int64)
        secs = C.c_double()
        with tempfile.TemporaryDirectory() as tmp:
            path = scratch_path or os.path.join(tmp, "group.index")
            _check(self.L.ref_search_group(self.h, q.shape[0], _p(q), k, workers, group, team, block, warmup_list,
                                           warmup_list_size, int(cut), threads_per_rank, path.encode(), _p(D), _p(I),
                                           C.byref(secs)))
        return D, I, secs.value

    def probes(self, q):
        q = np.ascontiguousarray(q, np.float32)
        npb = min(self.nprobe, self.nlist)
        P = np.empty((q.shape[0], npb), np.int64)
        _check(self.L.ref_probes(self.h, q.shape[0], _p(q), _p(P)))
        return P

    def warmup_tops(self, q, k, probes, warmup_list=10, warmup_list_size=None):
        q = np.ascontiguousarray(q, np.float32)
        probes = np.ascontiguousarray(probes, np.int64)
        if warmup_list_size is None:
            warmup_list_size = k
        t = np.empty(q.shape[0], np.float32)
        _check(self.L.ref_warmup_tops(self.h, q.shape[0], _p(q), k, warmup_list, warmup_list_size, _p(probes), _p(t)))
        return t

    def search_prune(self, q, k, probes, tops):
        q = np.ascontiguousarray(q, np.float32)
        probes = np.ascontiguousarray(probes, np.int64)
        tops = np.ascontiguousarray(tops, np.float32)
        D = np.empty((q.shape[0], k), np.float32)
        I = np.empty((q.shape[0], k), np.int64)
        _check(self.L.ref_search_prune(self.h, q.shape[0], _p(q), k, _p(probes), _p(tops), _p(D), _p(I)))
        return D, I

    def save(self, path):
        _check(self.L.ref_save(self.h, str(path).encode()))

    def load(self, path):
        _check(self.L.ref_load(self.h, str(path).encode()))
        d, nl, npb, m = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_int()
        _check(self.L.ref_info(self.h, C.byref(d), C.byref(nl), C.byref(npb), C.byref(m)))
        self.d, self.nlist, self.metric = d.value, nl.value, m.value


# The reference's dataset / result-file readers and recall metrics
# (src/utils.h), for the golden fixtures of harmonyclient_b200/datafiles.py.
def xvecs_info(path):
    n, d = C.c_size_t(), C.c_int()
    _check(load().ref_xvecs_info(str(path).encode(), C.byref(n), C.byref(d)))
    return n.value, d.value


def load_xvecs(path, a=1, b=0, cap=1 << 20):
    out = np.zeros(cap, np.float32)
    n, d = C.c_size_t(), C.c_int()
    _check(load().ref_load_xvecs(str(path).encode(), a, b, _p(out), cap, C.byref(n), C.byref(d)))
    return out[:n.value * d.value].reshape(n.value, d.value).copy()


def write_results(labels, distances, path):
    labels = np.ascontiguousarray(labels, np.int64)
    distances = np.ascontiguousarray(distances, np.float32)
    nq, k = labels.shape
    _check(load().ref_write_results(_p(labels), _p(distances), nq, k, str(path).encode()))


def load_results(path, nq, k):
    labels = np.zeros((nq, k), np.int64)
    dist = np.zeros((nq, k), np.float32)
    _check(load().ref_load_results(str(path).encode(), _p(labels), _p(dist), nq, k))
    return labels, dist


def recall(which, I, D, GT, GD, nq, k, metric, gt_k=0):
    I, GT = np.ascontiguousarray(I, np.int64), np.ascontiguousarray(GT, np.int64)
    D, GD = np.ascontiguousarray(D, np.float32), np.ascontiguousarray(GD, np.float32)
    out = C.c_float()
    _check(load().ref_recall(which, _p(I), _p(D), _p(GT), _p(GD), nq, k, metric, gt_k, C.byref(out)))
    return out.value
