"""Python mirror of Harmony's ``harmony::Index`` (src/Index.h:13-149) over the
CUDA engine.  Method names and argument meanings follow the reference:

* ``Index(d, nlist, nprobe, metric, opt_level, sub_k, sub_nlist, sub_nprobe,
  verbose, edge_device_enabled)`` — the reference constructor
  (src/Index.h:15-25); ``dim_blocks`` and ``device`` are additions;
* ``train(codes, faiss=False, lite=False)`` — src/Index.cpp:381-425;
* ``add(codes)`` — src/Index.cpp:581-697 (rebuilds the lists);
* ``search(queries, k)`` -> ``(distances, labels)`` — src/Index.cpp:1638-1706;
* ``preSearch(..., warmUpSearchList, warmUpSearchListSize, ...)`` —
  src/Index.h:90, the warm-up threshold parameters;
* ``save_index(path)`` / ``load_index(path)`` — src/Index.cpp:1708-1770;
* ``centroid_codes`` (read/write) and ``lists`` access via ``get_list``.

Errors raise ``HyError`` (a RuntimeError), as the reference throws
std::runtime_error.  All work runs on the GPU through libhy.so.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import HyError, IndexInfo, SearchStats, check

METRIC_IP, METRIC_L2 = 0, 1
OPT_NONE, OPT_TRIANGLE, OPT_SUBNN_L2, OPT_SUBNN_IP = 0, 1, 2, 4
OPT_TRI_SUBNN_L2, OPT_TRI_SUBNN_IP, OPT_SUBNN_ONLY, OPT_ALL = 3, 5, 6, 7
EDGEDEVIVE_ENABLED, EDGEDEVIVE_DISABLED = 0, 1


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f32(a, d=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if d is not None and (a.ndim != 2 or a.shape[1] != d):
        raise HyError(_lib.HY_ERR_ARG, f"expected an (n, {d}) float32 array, got shape {a.shape}")
    return a


class Index:
    def __init__(self, d=0, nlist=0, nprobe=0, metric=METRIC_L2, opt_level=OPT_NONE, sub_k=0, sub_nlist=1,
                 sub_nprobe=1, verbose=False, edge_device_enabled=EDGEDEVIVE_DISABLED, dim_blocks=4, device=0):
        self._L = _lib.load()
        h = C.c_void_p()
        check(self._L.hy_index_create(d, nlist, nprobe, int(metric), int(opt_level), dim_blocks, device, C.byref(h)))
        self._h = h
        self.verbose = verbose
        self.sub_k, self.sub_nlist, self.sub_nprobe = sub_k, sub_nlist, sub_nprobe

    def close(self):
        if getattr(self, "_h", None):
            self._L.hy_index_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # -- attributes of the reference class
    def info(self):
        inf = IndexInfo()
        check(self._L.hy_index_info(self._h, C.byref(inf)))
        return inf

    @property
    def d(self):
        return self.info().d

    @property
    def nlist(self):
        return self.info().nlist

    @property
    def metric(self):
        return self.info().metric

    @property
    def ntotal(self):
        return self.info().ntotal

    @property
    def opt_level(self):
        return self.info().opt_level

    @opt_level.setter
    def opt_level(self, v):
        """OPT_TRIANGLE with inner product: the reference's cos-bound window
        (see include/hy.h, hy_index_set_opt_level)."""
        check(self._L.hy_index_set_opt_level(self._h, int(v)))

    @property
    def nprobe(self):
        return self.info().nprobe

    @nprobe.setter
    def nprobe(self, v):
        check(self._L.hy_index_set_nprobe(self._h, int(v)))

    @property
    def centroid_codes(self):
        inf = self.info()
        c = np.empty((inf.nlist, inf.d), np.float32)
        check(self._L.hy_index_get_centroids(self._h, _p(c)))
        return c

    @centroid_codes.setter
    def centroid_codes(self, c):
        inf = self.info()
        c = _f32(c, inf.d)
        if c.shape[0] != inf.nlist:
            raise HyError(_lib.HY_ERR_ARG, f"centroids must be ({inf.nlist}, {inf.d})")
        check(self._L.hy_index_set_centroids(self._h, _p(c)))

    # -- reference methods
    def train(self, codes, faiss=False, lite=False):
        if faiss:
            raise HyError(_lib.HY_ERR_UNSUPPORTED, "faiss training is not part of this engine")
        x = _f32(codes, self.d)
        check(self._L.hy_index_train(self._h, x.shape[0], _p(x), int(bool(lite))))

    def add(self, codes):
        x = _f32(codes, self.d)
        check(self._L.hy_index_add(self._h, x.shape[0], _p(x)))

    def preSearch(self, nb=0, workerCount=0, blockCount=0, warmUpSearchList=0, warmUpSearchListSize=0, param=None,
                  path=""):
        """Sets the warm-up threshold parameters; the worker/block counts of
        the reference's MPI modes have no meaning on one GPU."""
        check(self._L.hy_index_presearch(self._h, int(warmUpSearchList), int(warmUpSearchListSize)))

    def set_form(self, form):
        """'plain' (exact FP32 scan), 'bf16' (batched tensor-core scan with
        exact FP32 re-rank) or 'fp8' (the same on e4m3 codes with per-list
        scales and an oversampled exact re-rank)."""
        f = {"plain": _lib.HY_FORM_PLAIN, "bf16": _lib.HY_FORM_BF16, "fp8": _lib.HY_FORM_FP8}.get(form, form)
        check(self._L.hy_index_set_form(self._h, int(f)))

    def set_plain_scan(self, mode):
        """The plain form's scan: 'auto' (default: list-major when the batch
        has at least 4 queries per list on average), 'query' (one CTA per
        query streams its probed lists) or 'list' (queries probing a list
        share one pass over it).  All give the same answer."""
        m = {"auto": _lib.HY_PLAIN_AUTO, "query": _lib.HY_PLAIN_QUERY_MAJOR,
             "list": _lib.HY_PLAIN_LIST_MAJOR}.get(mode, mode)
        check(self._L.hy_index_set_plain_scan(self._h, int(m)))

    def set_coarse(self, mode):
        """The bf16 form's coarse step: 'tensor' (default; bf16 tensor-core
        scores with error bounds, exact FP32 scores only for the centroids
        that can reach the nprobe best) or 'exact' (exact FP32 scores of every
        centroid).  Both give the same probe lists."""
        m = {"exact": _lib.HY_COARSE_EXACT, "tensor": _lib.HY_COARSE_TENSOR}.get(mode, mode)
        check(self._L.hy_index_set_coarse(self._h, int(m)))

    def set_batch_params(self, capq=0, oversample=0, row_slice=0):
        check(self._L.hy_index_set_batch_params(self._h, int(capq), int(oversample), int(row_slice)))

    def set_group_size(self, qg=0):
        """Queries per group of the tensor-core forms' search passes (32, 64
        or 128; 0 picks per pass by the expected queries per list)."""
        check(self._L.hy_index_set_group_size(self._h, int(qg)))

    def search(self, queries, k):
        q = _f32(queries, self.d)
        n = q.shape[0]
        D = np.empty((n, k), np.float32)
        I = np.empty((n, k), np.int64)
        check(self._L.hy_index_search(self._h, n, _p(q), int(k), _p(D), _p(I)))
        return D, I

    def autotune(self, queries, k, reps=3):
        """Pick the bf16 form's work shape on sample queries; returns the
        timings as a list of (row_slice, capq, ms, same_answer)."""
        q = _f32(queries, self.d)
        rep = np.zeros(18, np.float32)
        check(self._L.hy_index_autotune(self._h, q.shape[0], _p(q), int(k), int(reps), _p(rep)))
        return [(int(rep[3 * i]), int(rep[3 * i + 1]), abs(float(rep[3 * i + 2])), bool(rep[3 * i + 2] >= 0))
                for i in range(6)]

    def batch_params(self):
        inf = self.info()
        return {"capq": int(inf.capq), "row_slice": int(inf.row_slice)}

    def set_list_range(self, lo, hi):
        """Hold only lists [lo, hi) from the next add() on (list partition
        across GPUs; see harmonyclient_b200.parallel)."""
        check(self._L.hy_index_set_list_range(self._h, int(lo), int(hi)))

    def set_graph(self, enabled=True):
        """Graph mode for the device-pointer searches (CUDA graph replay)."""
        check(self._L.hy_index_set_graph(self._h, int(bool(enabled))))

    def search_nprobes(self, queries, k, nprobes):
        """Search with a per-query nprobe (int array, one per query)."""
        q = _f32(queries, self.d)
        npq = np.ascontiguousarray(nprobes, dtype=np.int32)
        if npq.shape != (q.shape[0],):
            raise ValueError("nprobes must hold one value per query")
        D = np.empty((q.shape[0], k), np.float32)
        I = np.empty((q.shape[0], k), np.int64)
        check(self._L.hy_index_search_nprobes(self._h, q.shape[0], _p(q), int(k), _p(npq), _p(D), _p(I)))
        return D, I

    def search_nprobes_device(self, n, q_ptr, k, nprobes_ptr, max_nprobe, d_ptr, i_ptr, stream=0):
        check(self._L.hy_index_search_nprobes_device(self._h, int(n), C.c_void_p(q_ptr), int(k),
                                                     C.c_void_p(nprobes_ptr), int(max_nprobe), C.c_void_p(d_ptr),
                                                     C.c_void_p(i_ptr), C.c_void_p(stream)))

    def search_preassigned(self, queries, k, probes):
        q = _f32(queries, self.d)
        P = np.ascontiguousarray(probes, np.int64)
        n = q.shape[0]
        D = np.empty((n, k), np.float32)
        I = np.empty((n, k), np.int64)
        check(self._L.hy_index_search_preassigned(self._h, n, _p(q), int(k), P.shape[1], _p(P), _p(D), _p(I)))
        return D, I

    def search_device(self, n, q_ptr, k, d_ptr, i_ptr, stream=0):
        """Device-pointer search: q (n x d float32), D (n x k float32), I
        (n x k int64) are CUDA device addresses; enqueued on `stream`."""
        check(self._L.hy_index_search_device(self._h, int(n), C.c_void_p(q_ptr), int(k), C.c_void_p(d_ptr),
                                             C.c_void_p(i_ptr), C.c_void_p(stream)))

    def probes(self, queries):
        q = _f32(queries, self.d)
        inf = self.info()
        P = np.empty((q.shape[0], min(inf.nprobe, inf.nlist)), np.int64)
        check(self._L.hy_index_probes(self._h, q.shape[0], _p(q), _p(P)))
        return P

    def warmup_tops(self, queries, k, probes, warmup_list=10, warmup_list_size=0):
        q = _f32(queries, self.d)
        P = np.ascontiguousarray(probes, np.int64)
        t = np.empty(q.shape[0], np.float32)
        check(self._L.hy_index_warmup_tops(self._h, q.shape[0], _p(q), int(k), P.shape[1], _p(P), int(warmup_list),
                                           int(warmup_list_size), _p(t)))
        return t

    def last_stats(self):
        st = SearchStats()
        check(self._L.hy_index_last_stats(self._h, C.byref(st)))
        return st.as_dict()

    def train_probe_model(self, queries, max_nprobe=64, k_label=10, epochs=30, lr=1e-3, coverage=0.97):
        """Train the learned probe predictor on sample queries (labels come
        from the exact scan at max_nprobe).  Returns the held-out report."""
        q = _f32(queries, self.d)
        rep = np.zeros(4, np.float32)
        check(self._L.hy_index_train_probe_model(self._h, q.shape[0], _p(q), int(max_nprobe), int(k_label),
                                                  int(epochs), float(lr), float(coverage), _p(rep)))
        return {"loss": float(rep[0]), "coverage": float(rep[1]), "mean_nprobe": float(rep[2]),
                "mean_label": float(rep[3])}

    def set_learned(self, enabled=True, judge_fraction=0.01, judge_recall=0.95):
        check(self._L.hy_index_set_learned(self._h, int(bool(enabled)), float(judge_fraction), float(judge_recall)))

    def get_probe_model(self):
        m = np.zeros(self._L.hy_probe_model_size(), np.float32)
        check(self._L.hy_index_get_probe_model(self._h, _p(m)))
        return m

    def set_probe_model(self, model):
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.size != self._L.hy_probe_model_size():
            raise ValueError("probe model has the wrong size")
        check(self._L.hy_index_set_probe_model(self._h, _p(m)))

    def list_size(self, l):
        s = C.c_size_t()
        check(self._L.hy_index_list_size(self._h, int(l), C.byref(s)))
        return s.value

    def get_list(self, l):
        n = self.list_size(l)
        d = self.d
        ids = np.empty(n, np.int64)
        codes = np.empty((n, d), np.float32)
        norms = np.empty(n, np.float32)
        if n:
            check(self._L.hy_index_get_list(self._h, int(l), _p(ids), _p(codes), _p(norms)))
        return ids, codes, norms

    def save_index(self, path):
        check(self._L.hy_index_save(self._h, str(path).encode()))

    def load_index(self, path):
        check(self._L.hy_index_load(self._h, str(path).encode()))


def file_inspect(path):
    """Header and list table of a reference .index file (no GPU needed)."""
    L = _lib.load()
    d, nl, ne, nt = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_size_t()
    m, o = C.c_int(), C.c_int()
    check(L.hy_file_inspect(str(path).encode(), C.byref(d), C.byref(nl), C.byref(m), C.byref(o), C.byref(ne),
                            C.byref(nt)))
    return {"d": d.value, "nlist": nl.value, "metric": m.value, "opt_level": o.value, "nonempty_lists": ne.value,
            "ntotal": nt.value}
