"""ctypes binding of libhy.so, the CUDA engine (C-ABI in include/hy.h).

Importing this module loads the in-tree library; if it has not been built the
import fails loudly — there is no CPU fallback for any operation.
"""
import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhy.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "hy.h")

HY_OK, HY_ERR_ARG, HY_ERR_OOM, HY_ERR_CUDA, HY_ERR_TIMEOUT, HY_ERR_STATE, HY_ERR_IO, HY_ERR_UNSUPPORTED = range(8)
HY_FORM_PLAIN, HY_FORM_BF16, HY_FORM_FP8 = 0, 1, 2
HY_COARSE_EXACT, HY_COARSE_TENSOR = 0, 1
HY_PLAIN_AUTO, HY_PLAIN_QUERY_MAJOR, HY_PLAIN_LIST_MAJOR = 0, 1, 2
HY_MAX_K = 256


class HyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hy error {code}: {msg}")
        self.code = code


class IndexInfo(C.Structure):
    _fields_ = [("d", C.c_size_t), ("nlist", C.c_size_t), ("nprobe", C.c_size_t), ("metric", C.c_int),
                ("opt_level", C.c_int), ("dim_blocks", C.c_size_t), ("ntotal", C.c_size_t),
                ("arena_rows", C.c_size_t), ("trained", C.c_int), ("device", C.c_int), ("form", C.c_int),
                ("learned", C.c_int), ("capq", C.c_size_t), ("row_slice", C.c_size_t)]


class SearchStats(C.Structure):
    _fields_ = [("nq", C.c_uint64), ("pairs", C.c_uint64), ("rows", C.c_uint64), ("tile_blocks", C.c_uint64),
                ("tile_blocks_max", C.c_uint64), ("coarse_ms", C.c_double), ("scan_ms", C.c_double),
                ("merge_ms", C.c_double), ("launches", C.c_uint64), ("fallback_queries", C.c_uint64),
                ("mean_nprobe", C.c_double), ("judge_recall", C.c_double), ("learned_fallback", C.c_uint64),
                ("kernel_ms", C.c_double), ("kernel_launches", C.c_uint64), ("graph_replayed", C.c_uint64),
                ("seg_sums", C.c_uint64), ("seg_sums_max", C.c_uint64), ("list_major", C.c_uint64),
                ("chunk_queries", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def declared_symbols():
    """Names of every function include/hy.h declares."""
    with open(HEADER) as f:
        txt = f.read()
    return sorted(set(re.findall(r"HY_API\s+[\w\s\*]+?\b(hy_\w+)\s*\(", txt)))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libhy.so is not built ({LIB_PATH}); run: python -m harmonyclient_b200.build")
    L = C.CDLL(LIB_PATH)
    sz, vp, i = C.c_size_t, C.c_void_p, C.c_int
    H = C.c_void_p
    L.hy_last_error.restype = C.c_char_p
    L.hy_version.restype = C.c_char_p
    L.hy_index_create.argtypes = [sz, sz, sz, i, i, sz, i, C.POINTER(C.c_void_p)]
    L.hy_index_destroy.argtypes = [H]
    L.hy_index_info.argtypes = [H, C.POINTER(IndexInfo)]
    L.hy_index_train.argtypes = [H, sz, vp, i]
    L.hy_index_train_device.argtypes = [H, sz, vp, i, vp]
    L.hy_index_set_centroids.argtypes = [H, vp]
    L.hy_index_get_centroids.argtypes = [H, vp]
    L.hy_index_add.argtypes = [H, sz, vp]
    L.hy_index_add_device.argtypes = [H, sz, vp, vp]
    L.hy_index_set_nprobe.argtypes = [H, sz]
    L.hy_index_set_opt_level.argtypes = [H, i]
    L.hy_index_presearch.argtypes = [H, sz, sz]
    L.hy_index_set_form.argtypes = [H, i]
    L.hy_index_set_plain_scan.argtypes = [H, i]
    L.hy_index_set_batch_params.argtypes = [H, sz, sz, sz]
    L.hy_index_set_group_size.argtypes = [H, C.c_int]
    L.hy_index_set_coarse.argtypes = [H, i]
    L.hy_index_search.argtypes = [H, sz, vp, sz, vp, vp]
    L.hy_index_search_device.argtypes = [H, sz, vp, sz, vp, vp, vp]
    L.hy_index_search_preassigned.argtypes = [H, sz, vp, sz, sz, vp, vp, vp]
    L.hy_index_probes.argtypes = [H, sz, vp, vp]
    L.hy_index_warmup_tops.argtypes = [H, sz, vp, sz, sz, vp, sz, sz, vp]
    L.hy_index_last_stats.argtypes = [H, C.POINTER(SearchStats)]
    L.hy_index_list_size.argtypes = [H, sz, C.POINTER(C.c_size_t)]
    L.hy_index_get_list.argtypes = [H, sz, vp, vp, vp]
    L.hy_index_save.argtypes = [H, C.c_char_p]
    L.hy_index_load.argtypes = [H, C.c_char_p]
    L.hy_file_inspect.argtypes = [C.c_char_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.hy_selftest_tcgen05.argtypes = [vp, vp, vp]
    L.hy_index_search_preassigned_noalloc.argtypes = [H, sz, vp, sz, sz, vp, vp, vp, vp]
    L.hy_index_set_graph.argtypes = [H, i]
    L.hy_index_set_list_range.argtypes = [H, sz, sz]
    L.hy_merge_topk.argtypes = [vp, vp, sz, sz, sz, i, vp, vp, vp]
    L.hy_selftest_tcgen05_e4m3.argtypes = [vp, vp, vp]
    L.hy_index_autotune.argtypes = [H, sz, vp, sz, i, vp]
    L.hy_index_search_nprobes.argtypes = [H, sz, vp, sz, vp, vp, vp]
    L.hy_index_search_nprobes_device.argtypes = [H, sz, vp, sz, vp, sz, vp, vp, vp]
    L.hy_index_train_probe_model.argtypes = [H, sz, vp, sz, sz, i, C.c_float, C.c_float, vp]
    L.hy_index_set_learned.argtypes = [H, i, C.c_float, C.c_float]
    L.hy_probe_model_size.restype = sz
    L.hy_index_get_probe_model.argtypes = [H, vp]
    L.hy_index_set_probe_model.argtypes = [H, vp]
    L.hy_mlp_loss_grad.argtypes = [vp, i, vp, vp, vp, vp]
    _lib = L
    return L


def check(rc):
    if rc != HY_OK:
        raise HyError(rc, load().hy_last_error().decode(errors="replace"))
