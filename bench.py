"""Benchmark of the IVF query hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form learned|bf16|plain] [--nprobe 64] [--nb 1000000] [--nq 10000]

Workload (one "step" = one batch search): 1,000,000 x 128 integer-valued
float32 vectors in [0,255] from a 4,096-component Gaussian mixture (seeded,
synthetic), nlist 1024 trained on the GPU, 10,000 queries from the same
mixture, k 100, nprobe 64; recall@10 against an FP64 brute force on a query
sample.  The list arena (~550 MB) is larger than L2, so no L2 flush is
needed between steps.

The headline form (--form learned) trains the probe network on 20,000 other
queries from the mixture, then searches with per-query nprobe on the bf16
tensor-core scan with the exact FP32 re-rank; the plain FP32 scan at the
fixed nprobe is timed in the same run ("plain_fp32", with its HBM roofline).

Prints one JSON line on rank 0.  Under torchrun each rank holds a replica of
the index and searches its own query batch (weak scaling, no collective on
the data path); `value` is the whole-job QPS, timed on the device as the
max over ranks.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS at recall@10>=0.95, 1 B200: learned+BF16 vs plain FP32 scan; scan HBM %"


# DRAM bytes (read + write) per launch of the dominant kernel, from ncu
# captures of this script (dram__bytes_read.sum + dram__bytes_write.sum),
# keyed by (workload, form, nb, nq, nprobe), with the capture each comes
# from (the summaries and commands are in profiles/).  A line whose
# configuration has no capture reports traffic null.
KNOWN_TRAFFIC = {
    ("c2", "plain", 1_000_000, 10_000, 64): 216_530_000_000,
    ("c2", "plain-lm", 1_000_000, 10_000, 64): 492_300_000,
    ("c2", "learned", 1_000_000, 10_000, 64): 261_650_000,
    ("c2", "bf16", 1_000_000, 10_000, 64): 292_800_000,
}
TRAFFIC_SOURCE = {
    "plain": "query-major scan_plain_kernel, 1,000-query ncu capture scaled x10 "
             "(profiles/scan_plain_kernel_c2_1M_nprobe64.md)",
    "plain-lm": "list_scan_kernel, average of the two passes of one 10,000-query search, ncu --set full "
                "(profiles/list_scan_kernel_c2_1M_nprobe64.md)",
    "learned": "batched_scan_kernel, average of the two passes of one 10,000-query search "
               "(profiles/batched_scan_kernel_c2_learned.md)",
    "bf16": "batched_scan_kernel, average of the two passes, nprobe 64 "
            "(profiles/batched_scan_kernel_c2_bf16_nprobe64.md)",
}


def peaks():
    """(HBM GB/s, dense bf16 TFLOP/s burst, which) from MEASURED_PEAKS.json,
    else the pool's earlier fallback measurement."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return j.get("hbm_gbs", 6650.0), j.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class Clocks:
    """Samples the GPU's SM clock and clock-event reasons during the timed
    region: through NVML every few milliseconds when it is available (timed
    regions here can be far shorter than nvidia-smi's 200 ms period), else
    through nvidia-smi.  Read-only."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device):
        self.device = device
        self.sm, self.reasons, self.max = [], set(), None
        self.stop = threading.Event()
        self.t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self.stop.is_set():
                    self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                    r = get_reasons(h)
                    for n, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(n)
                    time.sleep(0.002)

            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
        except Exception:
            self.t = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.t:
            self.t.join(timeout=2)

    def summary(self):
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.max,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml"}


# The measured workloads (seeded synthetic stand-ins of the named shapes).
WORKLOADS = {
    "c2": dict(gen="gmm_uint8", kw={}, d=128, nlist=1024, k=100, nb=1_000_000, nq=10_000, nprobe=64,
               desc="{nb} x 128 uint8-valued gmm (4096 components, sigma 20)",
               data="synthetic (seeded Gaussian mixture, integer-valued in [0,255])"),
    "c3": dict(gen="gmm_dense", kw={}, d=420, nlist=2048, k=10, nb=1_000_000, nq=10_000, nprobe=64,
               desc="{nb} x 420 float gmm (2048 components, per-dim mean U[-1,1], sigma 0.3)",
               data="synthetic (seeded Gaussian mixture, float32)"),
    # Zipf(1.1)-weighted components give skewed list sizes; every query has its
    # own nprobe drawn U[8,128] (seeded), searched through search_nprobes.
    "c4": dict(gen="gmm_uint8", kw={"ncomp": 16_384, "zipf": 1.1}, d=128, nlist=16_384, k=10, nb=10_000_000,
               nq=65_536, nprobe=128, per_query=(8, 128), cpu_ref=False,
               desc="{nb} x 128 uint8-valued gmm (16384 components weighted Zipf(1.1)), per-query nprobe U[8,128]",
               data="synthetic (seeded Zipf-weighted Gaussian mixture, integer-valued in [0,255])"),
    "c5": dict(gen="sparse_nonneg", kw={}, d=500, nlist=4096, k=10, nb=2_000_000, nq=20_000, nprobe=256, cpu_ref=False,
               desc="{nb} x 500 sparse non-negative L2-normalised (2048 components, 10% support, Exp(1))",
               data="synthetic (seeded sparse non-negative mixture, float32)"),
}


def queries(args, n, query_seed):
    """Another query set from the workload's mixture (file workloads: n rows
    of the base file, seeded)."""
    from harmonyclient_b200 import datasets
    W = WORKLOADS[args.workload]
    if W.get("files"):
        from harmonyclient_b200 import datafiles
        x = datafiles.load_xvecs(W["files"][0], (1, args.nb))
        pick = np.random.default_rng(query_seed).choice(x.shape[0], size=min(n, x.shape[0]), replace=False)
        return np.ascontiguousarray(x[np.sort(pick)], np.float32)
    return getattr(datasets, W["gen"])(0, n, seed=0, query_seed=query_seed, **W["kw"])[1]


def per_query_nprobe(args, nq):
    """The workload's per-query nprobe (None when it uses one nprobe)."""
    lo_hi = WORKLOADS[args.workload].get("per_query")
    if lo_hi is None:
        return None
    return np.random.default_rng(1).integers(lo_hi[0], lo_hi[1] + 1, size=nq).astype(np.int32)


def _bvecs_records(path):
    """The layout of a .bvecs file, told from its size: plain records (the
    public BIGANN files) or the reference loader's extra 4-byte header."""
    from harmonyclient_b200 import datafiles
    return str(path).endswith(".bvecs") and datafiles.bvecs_is_records(path)


def _file_info(path):
    """(rows, d) of a vector file, .bvecs counted in its own layout."""
    from harmonyclient_b200 import datafiles
    n, d = datafiles.load_xvecs_info(path)
    if str(path).endswith(".bvecs"):
        n = datafiles.bvecs_rows(path, _bvecs_records(path))
    return n, d


def file_workload(base_file, query_file, nb, nq):
    """Base and query rows from .fvecs / .bvecs / .txt files (the reference's
    readers, harmonyclient_b200.datafiles): the first nb / nq rows (0: all)."""
    from harmonyclient_b200 import datafiles
    x = datafiles.load_xvecs(base_file, (1, nb or 0), _bvecs_records(base_file))
    q = datafiles.load_xvecs(query_file, (1, nq or 0), _bvecs_records(query_file))
    if x.shape[1] != q.shape[1]:
        raise SystemExit(f"base d {x.shape[1]} != query d {q.shape[1]}")
    return np.ascontiguousarray(x, np.float32), np.ascontiguousarray(q, np.float32)


def workload(args, rank):
    from harmonyclient_b200 import datasets
    W = WORKLOADS[args.workload]
    if W.get("files"):
        # Every rank searches the file's queries.
        return file_workload(W["files"][0], W["files"][1], args.nb, args.nq)
    x, q = getattr(datasets, W["gen"])(args.nb, args.nq, seed=0, **W["kw"])
    if rank:
        # Other ranks search their own queries from the same mixture.
        q = queries(args, args.nq, 1000 + rank)
    return x, q


def cpu_baseline_ref(x, q, cent, nprobe, k, budget_s):
    """The reference's own ORIGINAL search (oracle/_ref) on the host cores, on
    a bounded query sample sized to ~budget_s seconds."""
    from oracle import ref
    if not ref.available():
        return None
    nt = os.cpu_count() or 1
    ref.set_threads(nt)
    R = ref.RefIndex(x.shape[1], cent.shape[0], nprobe)
    R.set_centroids(cent)
    R.add(x)
    m = max(nt, 64)
    t0 = time.perf_counter()
    R.search(q[:m], k)
    dt = time.perf_counter() - t0
    m2 = int(min(q.shape[0], max(m, m * budget_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    Dr, Ir = R.search(q[:m2], k)
    dt = time.perf_counter() - t0
    info = {"value": m2 / dt, "unit": "queries/s", "cores": nt, "kind": "reference",
            "sample": f"{m2} of {q.shape[0]} queries, reference Index::search ORIGINAL mode, OpenMP x{nt}"}
    info["group"] = cpu_baseline_group(R, q[:m2], k, Dr, Ir, nt)
    return info, Dr, Ir


def cpu_baseline_group(R, q, k, Dr, Ir, cores):
    """The reference's default distributed mode (GROUP with pruning,
    src/Index.cpp:1053-1187, src/node.cpp:679-1203) in its documented
    configuration (--group 2 --team 2 --block 4 on 5 MPI ranks), the ranks
    run as threads of this process (oracle/ref_mpi_threads.cpp) with the host
    cores split between them; timed as the reference times it (the master's
    Index::search), with every row compared to the ORIGINAL search's."""
    from tests.topk_check import row_agree
    workers, group, team, block = 4, 2, 2, 4
    m = min(q.shape[0], 10_000) // (group * block) * (group * block)
    if m == 0 or k > 100:
        return {"unavailable": "GROUP mode needs k <= 100 and nq divisible by group x block"}
    try:
        import psutil
        if psutil.virtual_memory().available < 48 << 30:
            return {"unavailable": "GROUP mode's per-worker distance buffers need ~20 GB of host memory here"}
    except ImportError:
        pass
    tpr = max(1, cores // (workers + 1))
    D, I, secs = R.search_group(q[:m], k, workers=workers, group=group, team=team, block=block,
                                threads_per_rank=tpr)
    eq = sum(1 for r in range(m) if row_agree(Dr[r], Ir[r], D[r], I[r], 0.0)[0])
    return {"value": round(m / secs, 2), "unit": "queries/s", "cores": tpr * (workers + 1),
            "ranks": workers + 1, "config": "group 2, team 2, block 4, pruning on, warm-up 10 lists x k rows",
            "ranks_as": "threads of one process (no MPI on this host)", "queries": m,
            "rows_equal_to_original": eq}


def parity_block(Dr, Ir, answers, q, cent, nprobe, k, integral):
    """Row-by-row comparison of the GPU forms' answers with the reference's
    Index::search on the same centroids (tests/topk_check.py rules): on
    integer-valued data distances bit-equal (rtol 0), else within 1e-5
    relative; ids equal below the k-th distance; queries whose nprobe-th and
    (nprobe+1)-th centroid distances tie within 1e-5 in FP64 are skipped."""
    from tests.topk_check import probe_tied_rows, row_agree
    m = Dr.shape[0]
    tied = probe_tied_rows(q[:m], cent, np.zeros((1, nprobe)), 1)
    rtol = 0.0 if integral else 1e-5
    out = {"vs": "reference Index::search, ORIGINAL mode (oracle/_ref), same centroids and lists",
           "queries": m, "nprobe": nprobe, "k": k, "rtol": rtol, "probe_tied_skipped": len(tied)}
    for name, (D, I) in answers.items():
        eq = sum(1 for r in range(m) if r not in tied and row_agree(Dr[r], Ir[r], D[r], I[r], rtol)[0])
        out[name] = {"rows_compared": m - len(tied), "rows_equal": eq}
    return out


def _search(idx, dq, dD, dI, k, ts, npq=None):
    """One device-pointer search on stream ts; npq = (device per-query
    nprobe tensor, its maximum) for the per-query workloads."""
    if npq is None:
        idx.search_device(dq.shape[0], dq.data_ptr(), k, dD.data_ptr(), dI.data_ptr(), ts.cuda_stream)
    else:
        idx.search_nprobes_device(dq.shape[0], dq.data_ptr(), k, npq[0].data_ptr(), npq[1], dD.data_ptr(),
                                  dI.data_ptr(), ts.cuda_stream)


def _time_device(idx, dq, dD, dI, k, steps, ts, dist, dev, npq=None):
    """Device-timed loop of `steps` batch searches (CUDA events on the
    launching stream `ts`, max over ranks); the last step's stats come back."""
    import torch
    n = dq.shape[0]
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")  # profilers select the timed launches by this range
        e0.record(ts)
        for _ in range(steps):
            _search(idx, dq, dD, dI, k, ts, npq)
        e1.record(ts)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    st = idx.last_stats()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item()), st, clk.summary()


def _kernel_ms(idx, dq, dD, dI, k, reps, ts, npq=None):
    """Average duration of the dominant scan kernel's launches: every
    launch is bracketed by CUDA events on its own stream inside the library;
    `reps` further searches, each read back."""
    import torch
    tot, launches = 0.0, 0
    for _ in range(reps):
        _search(idx, dq, dD, dI, k, ts, npq)
        st = idx.last_stats()
        tot += st["kernel_ms"]
        launches += st["kernel_launches"]
    torch.cuda.synchronize()
    return tot / max(launches, 1), launches / max(reps, 1)


def _score(x, q, D, I, ns, truth):
    """recall@10 and distance errors against the float64 GPU brute force on
    the first ns queries (0: all); the exact top-10 is computed once."""
    from oracle import gpu_bruteforce as gb
    ns = q.shape[0] if ns <= 0 else min(ns, q.shape[0])
    if "It" not in truth:
        truth["Dt"], truth["It"] = gb.topk(x, q[:ns], 10)
    return gb.score(D[:ns], I[:ns], truth["Dt"], truth["It"], x, q[:ns], at=10), ns


def run_ours(args, rank, world, dist):
    import ctypes as C

    import torch

    import harmonyclient_b200 as hb
    from harmonyclient_b200 import _lib, datasets

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    x, q = workload(args, rank)
    W = WORKLOADS[args.workload]
    nlist, k, d = W["nlist"], W["k"], W["d"]
    idx = hb.Index(d, nlist, args.nprobe, hb.METRIC_L2, device=dev)
    t0 = time.perf_counter()
    idx.train(x)
    idx.add(x)
    # Warm-up thresholds as the reference's default run uses them
    # (--warmup_list 10, warmup_list_size = k; src/query.cpp:845-847).
    idx.preSearch(warmUpSearchList=args.warmup_list, warmUpSearchListSize=k)
    build_s = time.perf_counter() - t0
    learned = args.form == "learned"
    probe_report, train_s = None, 0.0
    if learned:
        # The probe network is trained on its own query sample from the same
        # mixture (labels from the exact scan at the index's nprobe).
        tq = queries(args, args.train_queries, 777)
        t0 = time.perf_counter()
        probe_report = idx.train_probe_model(tq, max_nprobe=args.nprobe, k_label=10, epochs=args.epochs,
                                             lr=1e-3, coverage=args.coverage)
        train_s = time.perf_counter() - t0
        idx.set_learned(True, judge_fraction=args.judge_fraction, judge_recall=0.95)
    base = args.base if learned else args.form
    idx.set_form(base)
    tune = None
    if base == "fp8":
        idx.set_batch_params(oversample=args.oversample)
    if base != "plain" and args.group_size:
        idx.set_group_size(args.group_size)
    if base != "plain" and args.autotune:
        # Work shape picked on this batch (every shape gives the same answer).
        tune = idx.autotune(q, k, reps=2)

    stream = torch.cuda.Stream()  # the launching stream of every timed search
    dq = torch.from_numpy(q).cuda()
    npq_host = per_query_nprobe(args, q.shape[0])
    npq = None if npq_host is None else (torch.from_numpy(npq_host).cuda(), int(npq_host.max()))
    dD = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")
    idx.set_graph(args.graph)
    for _ in range(args.warmup):
        _search(idx, dq, dD, dI, k, stream, npq)
    torch.cuda.synchronize()
    ms_max, st_dev, clocks = _time_device(idx, dq, dD, dI, k, args.steps, stream, dist, dev, npq)
    value = world * q.shape[0] * args.steps / (ms_max / 1e3)
    I_main = dI.cpu().numpy()
    D_main = dD.cpu().numpy()
    kern_ms, kern_per_search = _kernel_ms(idx, dq, dD, dI, k, 3, stream, npq)
    kern_chunk = int(idx.last_stats()["chunk_queries"]) or q.shape[0]  # queries the timed launches cover

    # End to end through the public host API: pinned host queries in, results
    # back to pinned host memory, every step (with the learned form this
    # includes the recall judge's fixed-nprobe search of 1% of the batch).
    hq = torch.from_numpy(q).pin_memory()
    hD = torch.empty((q.shape[0], k), dtype=torch.float32).pin_memory()
    hI = torch.empty((q.shape[0], k), dtype=torch.int64).pin_memory()
    L = _lib.load()

    def e2e_step():
        if npq_host is None:
            _lib.check(L.hy_index_search(idx._h, q.shape[0], C.c_void_p(hq.data_ptr()), k, C.c_void_p(hD.data_ptr()),
                                         C.c_void_p(hI.data_ptr())))
        else:
            _lib.check(L.hy_index_search_nprobes(idx._h, q.shape[0], C.c_void_p(hq.data_ptr()), k,
                                                 C.c_void_p(npq_host.ctypes.data), C.c_void_p(hD.data_ptr()),
                                                 C.c_void_p(hI.data_ptr())))

    e2e_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    launches, fallback, judge, learned_fb, mean_np = 0, 0, [], 0, []
    for _ in range(args.steps):
        e2e_step()
        st = idx.last_stats()
        launches = st["launches"]
        fallback = max(fallback, st["fallback_queries"])
        judge.append(st["judge_recall"])
        learned_fb += st["learned_fallback"]
        mean_np.append(st["mean_nprobe"])
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], device="cuda")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * q.shape[0] * args.steps / float(te.item())

    # The plain FP32 scan on the same index and queries (fixed nprobe), the
    # comparison the headline metric names; it also gives the scan's HBM
    # fraction.
    plain = None
    P_main = idx.probes(q)
    if npq_host is not None:
        P_main[np.arange(P_main.shape[1])[None, :] >= npq_host[:, None]] = -1
    if base != "plain" and args.plain_steps > 0:
        if learned:
            idx.set_learned(False)
        idx.set_form("plain")
        _search(idx, dq, dD, dI, k, stream, npq)
        pms, pst, pclk = _time_device(idx, dq, dD, dI, k, args.plain_steps, stream, dist, dev, npq)
        pk_ms, pk_launches = _kernel_ms(idx, dq, dD, dI, k, 1, stream, npq)
        plain = {"ms": pms, "kernel_ms": pk_ms, "launches": pk_launches, "stats": idx.last_stats(),
                 "I": dI.cpu().numpy(), "D": dD.cpu().numpy(), "clocks": pclk}
        idx.set_form(base)
        if learned:
            idx.set_learned(True, judge_fraction=args.judge_fraction, judge_recall=0.95)

    if rank != 0:
        return None

    sizes = np.array([idx.list_size(l) for l in range(nlist)], np.int64)

    def pair_rows(P):
        return int(np.where(P >= 0, sizes[np.maximum(P, 0)], 0).sum())

    hbm_peak, tc_peak, peak_kind = peaks()
    learned_probes = int((P_main >= 0).sum())
    rows_main = pair_rows(P_main)
    if base == "plain":
        alg = rows_main * d * 4 + q.shape[0] * d * 4 + q.shape[0] * k * 12
        roof = plain_roofline(idx.last_stats(), kern_ms * kern_per_search, kern_per_search, alg, clocks, args,
                              hbm_peak, peak_kind)
    else:
        # One batched-scan launch does a 2d-flop bf16 inner product per
        # (query, probed row) pair of its pass and reads each list that some
        # query probes in that pass once, as bf16 rows (d x 2 bytes).  The
        # bound is whichever of the two takes longer at the measured peaks.
        # kern_ms covers the launches of the search's last query chunk, so
        # the work counted is that chunk's (the last kern_chunk queries).
        P_last = P_main[P_main.shape[0] - kern_chunk:]
        flops = pair_rows(P_last) * 2 * d / kern_per_search
        distinct = 0
        for j0, j1 in ((0, 1), (1, P_last.shape[1])):
            cols = P_last[:, j0:j1]
            used = np.unique(cols[cols >= 0])
            distinct += int(sizes[used].sum())
        lbytes = distinct * d * (1 if base == "fp8" else 2) / kern_per_search
        t_tc, t_hbm = flops / (tc_peak * 1e12), lbytes / (hbm_peak * 1e9)
        if t_tc >= t_hbm:
            ach = flops / (kern_ms / 1e3) / 1e12
            roof = {"bound": "tensor", "achieved": round(ach, 2), "peak": tc_peak, "unit": "TFLOP/s",
                    "frac": round(ach / tc_peak, 4)}
        else:
            ach = lbytes / (kern_ms / 1e3) / 1e9
            roof = {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm_peak, "unit": "GB/s",
                    "frac": round(ach / hbm_peak, 4)}
        roof.update({"traffic": KNOWN_TRAFFIC.get((args.workload, args.form, args.nb, args.nq, args.nprobe)),
                     "traffic_source": TRAFFIC_SOURCE.get(args.form),
                     "peak_kind": peak_kind, "kernel": "batched_scan_kernel", "kernel_ms": round(kern_ms, 4),
                     "algorithmic_flops": int(flops), "algorithmic_bytes": int(lbytes),
                     "launches_per_search": kern_per_search})

    truth = {}
    sc_main, ns = _score(x, q, D_main, I_main, args.recall_sample, truth)
    plain_line = None
    if plain is not None:
        if learned:
            idx.set_learned(False)
        P_plain = idx.probes(q)
        if npq_host is not None:
            P_plain[np.arange(P_plain.shape[1])[None, :] >= npq_host[:, None]] = -1
        prow = pair_rows(P_plain)
        palg = prow * d * 4 + q.shape[0] * d * 4 + q.shape[0] * k * 12
        pst = plain["stats"]
        scan_ms = plain["kernel_ms"] * plain["launches"]  # every scan launch of one search
        sc_plain, _ = _score(x, q, plain["D"], plain["I"], args.recall_sample, truth)
        pv = world * q.shape[0] * args.plain_steps / (plain["ms"] / 1e3)
        proof = plain_roofline(pst, scan_ms, plain["launches"], palg, plain["clocks"], args, hbm_peak, peak_kind)
        plain_line = {"value": round(pv, 1), "unit": "queries/s", "steps": args.plain_steps,
                      "ms_per_step": round(plain["ms"] / args.plain_steps, 3),
                      "recall_at_10": round(sc_plain["recall"], 4),
                      "dist_rel_err_max": sc_plain["dist_rel_err_max"],
                      "nprobe": args.nprobe, "speedup_of_headline": round(value / pv, 2),
                      "roofline": proof, "fallback_queries": pst.get("fallback_queries", 0),
                      "clocks": plain["clocks"]}

    parity = None
    if W.get("cpu_ref", True) and npq_host is None:
        got = cpu_baseline_ref(x, q, idx.centroid_codes, args.nprobe, k, args.cpu_budget)
        cpu = got[0] if got else None
        if got:
            # The GPU forms at the reference's fixed nprobe, on the same queries.
            answers = {}
            if plain is not None:
                answers["plain_fp32"] = (plain["D"], plain["I"])
            if learned:
                idx.set_learned(False)
            if base != "plain":
                Db, Ib = idx.search(q[:got[1].shape[0]], k)
                answers[f"{base}_fixed_nprobe"] = (Db, Ib)
            else:
                answers["plain_fp32"] = (D_main, I_main)
            if learned:
                idx.set_learned(True, judge_fraction=args.judge_fraction, judge_recall=0.95)
            integral = bool(np.all(x == np.rint(x)) and np.all(q == np.rint(q)) and np.abs(x).max() <= 255)
            parity = parity_block(got[1], got[2], answers, q, idx.centroid_codes, args.nprobe, k, integral)
    elif W.get("cpu_ref", True):
        cpu = None
    else:
        cpu = {"value": None, "unit": "queries/s", "cores": os.cpu_count(), "kind": "reference",
               "unavailable": "the reference's host add() of this base (nearest of nlist centroids for every row) "
                              "alone takes far longer than the bench's time bound on the host cores"}
    h2d = q.nbytes
    d2h = q.shape[0] * k * 12
    scan_name = {"bf16": "bf16 tcgen05 scan + exact FP32 re-rank",
                 "fp8": f"e4m3 tcgen05 scan (per-list scales) + exact FP32 re-rank of <= {args.oversample} x k",
                 "plain": "plain FP32 scan"}[base]
    form_name = f"learned probes + {scan_name}" if learned else scan_name
    line = {
        "metric": METRIC,
        "value": round(value, 1),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"plain": "f32", "bf16": "bf16", "fp8": "e4m3"}[base],
        "data": W["data"],
        "form": form_name,
        "config": {"workload": W["desc"].format(nb=args.nb) + f", nlist {nlist}, nprobe {args.nprobe}, k {k}, "
                               f"{q.shape[0]} queries per step per GPU",
                   "name": args.workload,
                   "nb": args.nb, "d": d, "nlist": nlist, "nprobe": args.nprobe, "k": k, "nq": q.shape[0],
                   "l2_flush": "not needed: list arena larger than L2", "parallelism": f"replicas x{world}"},
        "recall_at_10": round(sc_main["recall"], 4),
        "recall_vs": f"FP64 brute force on the GPU, {ns} queries",
        "dist_rel_err": {"max": sc_main["dist_rel_err_max"], "mean": sc_main["dist_rel_err_mean"]},
        "mean_nprobe": round(learned_probes / q.shape[0], 3),
        "roofline": roof,
        "e2e": {"value": round(e2e_value, 1), "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(st_dev["launches"]) * args.steps,
        "graph": {"enabled": bool(args.graph), "replayed": bool(st_dev["graph_replayed"])},
        "work_shape": {**idx.batch_params(), "autotune": tune},
        "plain_fp32": plain_line,
        "warmup_list": args.warmup_list,
        "fallback_queries": fallback,
        "parity": parity,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "build_s": round(build_s, 2),
    }
    if args.extras and world == 1:
        # The main index's other nprobes, then two other workloads (each
        # failure is recorded in the line rather than losing it).
        extras = {}
        for name, fn in (("c2_nprobe", lambda: extra_nprobe_sweep(idx, x, q, k, (16, 64, 256), 3, stream, dev,
                                                                     args.nprobe)),
                         (f"c2_sigma{args.hard_sigma:g}", lambda: extra_c2_hard(args, stream, dev, 3,
                                                                                 args.hard_sigma)),
                         ("c3", lambda: extra_c3(args, stream, dev, 3))):
            t0 = time.perf_counter()
            try:
                extras[name] = fn()
            except Exception as e:  # noqa: BLE001 - reported in the line
                extras[name] = {"error": f"{type(e).__name__}: {e}"}
            extras[name]["wall_s"] = round(time.perf_counter() - t0, 1)
        line["extras"] = extras
    if learned:
        line["probe_model"] = {"train_queries": args.train_queries, "epochs": args.epochs,
                               "coverage_target": args.coverage, "train_s": round(train_s, 2),
                               "heldout": {kk: round(v, 4) for kk, v in probe_report.items()},
                               "judge_fraction": args.judge_fraction,
                               "judge_recall_min": round(min(judge), 4) if judge else None,
                               "judge_fallbacks": learned_fb}
    return line


# ---------------------------------------------------------------------------
# Extra measurements of the one-GPU line: the other nprobes of the 1M x 128
# workload, a harder mixture on which the learned predictor has work to do,
# and the 1M x 420 precision workload at k 10 and 100.  Each is timed with
# CUDA events on the device-pointer API (graph mode) and scored against a
# float64 brute force over every query.
def plain_roofline(st, scan_ms, launches, palg, clocks, args, hbm_peak, peak_kind):
    """Roofline of the plain form's scan over one search (scan_ms: every scan
    launch of the search's last query chunk, the launches the library's
    kernel events time).  List-major: executed FP32 operations (3 x 32 x 16
    per executed (query, 32-row tile, 16-dimension segment) partial sum,
    `seg_sums`) against 148 SMs x 128 FP32 lanes x the SM clock measured
    during the run; the lists are read once per group of 32 queries, mostly
    from L2, so the pair bytes are reported beside it, not as a fraction.
    Query-major: pair bytes (every probed row of every query, d x 4 bytes,
    plus queries and results) against the measured copy bandwidth."""
    if st.get("list_major"):
        # The counters and kernel_ms cover the search's last query chunk; its
        # pair bytes are the unpruned segment sums' rows (32 rows x 16
        # dimensions x 4 bytes each, tiles padded to 32 rows).
        ops = st["seg_sums"] * 32 * 16 * 3
        palg = st["seg_sums_max"] * 32 * 16 * 4
        sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
        fpeak = 148 * 128 * sm_mhz * 1e6 / 1e12
        fach = ops / (scan_ms / 1e3) / 1e12
        return {"bound": "fp32", "achieved": round(fach, 2), "peak": round(fpeak, 2), "unit": "TFLOP/s",
                "frac": round(fach / fpeak, 4),
                "peak_kind": "nominal FP32 issue (148 SMs x 128 lanes x measured SM clock)",
                "kernel": "list_scan_kernel", "kernel_ms": round(scan_ms, 4), "launches_per_search": launches,
                "executed_ops": int(ops), "seg_sums_executed": round(st["seg_sums"] / max(st["seg_sums_max"], 1), 4),
                "pair_bytes": palg, "pair_bytes_rate_gbs": round(palg / (scan_ms / 1e3) / 1e9, 1),
                "traffic": KNOWN_TRAFFIC.get((args.workload, "plain-lm", args.nb, args.nq, args.nprobe)),
                "traffic_source": TRAFFIC_SOURCE["plain-lm"]}
    pach = palg / (scan_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": round(pach, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(pach / hbm_peak, 4), "peak_kind": peak_kind,
            "traffic": KNOWN_TRAFFIC.get((args.workload, "plain", args.nb, args.nq, args.nprobe)),
            "traffic_source": TRAFFIC_SOURCE["plain"],
            "kernel": "scan_plain_kernel", "kernel_ms": round(scan_ms, 4), "algorithmic_bytes": palg}


def _device_qps(idx, q, k, steps, ts, dev):
    """queries/s of `steps` device-pointer searches after two untimed ones,
    with the last answer, the stats of the last search and ms per step."""
    import torch
    dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    dD = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")
    for _ in range(2):
        _search(idx, dq, dD, dI, k, ts)
    torch.cuda.synchronize()
    ms, st, _ = _time_device(idx, dq, dD, dI, k, steps, ts, None, dev)
    kern_ms, launches = _kernel_ms(idx, dq, dD, dI, k, 1, ts)
    st = idx.last_stats()
    return {"qps": round(q.shape[0] * steps / (ms / 1e3), 1), "ms_per_step": round(ms / steps, 4),
            "kernel_ms": round(kern_ms * launches, 4)}, dD.cpu().numpy(), dI.cpu().numpy(), st


def _scored(x, q, D, I, truth, at, metric=1):
    from oracle import gpu_bruteforce as gb
    sc = gb.score(D, I, truth["D"], truth["I"], x, q, at=at, metric=metric)
    return {"recall_at_%d" % at: round(sc["recall"], 4), "dist_rel_err_max": sc["dist_rel_err_max"]}


def _plain_work(st):
    """The list-major plain scan's executed share of its unpruned block sums."""
    if st.get("list_major") and st.get("seg_sums_max"):
        return {"scan": "list-major", "seg_sums_executed": round(st["seg_sums"] / st["seg_sums_max"], 4)}
    return {"scan": "query-major"}


def extra_nprobe_sweep(idx, x, q, k, nprobes, steps, ts, dev, main_nprobe):
    """bf16 (fixed nprobe) and plain FP32 at each nprobe on the main index."""
    from oracle import gpu_bruteforce as gb
    truth = {}
    truth["D"], truth["I"] = gb.topk(x, q, 10)
    out = {}
    idx.set_learned(False)
    for npb in nprobes:
        idx.nprobe = npb
        row = {}
        for form in ("bf16", "plain"):
            idx.set_form(form)
            r, D, I, st = _device_qps(idx, q, k, steps, ts, dev)
            r.update(_scored(x, q, D, I, truth, 10))
            if form == "plain":
                r.update(_plain_work(st))
            row[form] = r
        row["bf16_over_plain"] = round(row["bf16"]["qps"] / row["plain"]["qps"], 2)
        out[str(npb)] = row
    idx.nprobe = main_nprobe
    return out


def extra_c2_hard(args, ts, dev, steps, sigma):
    """1M x 128 integer-valued mixture with a larger sigma (neighbours
    straddle lists, so nprobe 1 misses much of the top-10): the bf16 form at
    fixed nprobe 1..64, the learned probes + bf16 trained at several coverage
    targets (each a recall / speed trade-off), and the plain FP32 scan at the
    smallest fixed nprobe reaching recall@10 0.95.  Speed-ups compare the
    fastest configuration of each kind that reaches recall@10 0.95."""
    import harmonyclient_b200 as hb
    from harmonyclient_b200 import datasets
    from oracle import gpu_bruteforce as gb
    nb = args.nb
    x, q = datasets.gmm_uint8(nb, args.nq, sigma=sigma, seed=0)
    tq = datasets.gmm_uint8(0, args.train_queries, sigma=sigma, seed=0, query_seed=777)[1]
    k = 10
    max_np = 256
    idx = hb.Index(128, 1024, max_np, hb.METRIC_L2, device=dev)
    idx.train(x)
    idx.add(x)
    idx.preSearch(warmUpSearchList=args.warmup_list, warmUpSearchListSize=k)
    truth = {}
    truth["D"], truth["I"] = gb.topk(x, q, 10)
    idx.set_form("bf16")
    sweep = {}
    for npb in (1, 2, 4, 8, 16, 32, 64, 128, 256):
        idx.nprobe = npb
        r, D, I, _ = _device_qps(idx, q, k, steps, ts, dev)
        r.update(_scored(x, q, D, I, truth, 10))
        sweep[str(npb)] = r
    idx.nprobe = max_np
    learned = {}
    for cov in (0.5, 0.7, 0.8, 0.9, 0.97):
        t0 = time.perf_counter()
        rep = idx.train_probe_model(tq, max_nprobe=max_np, k_label=10, epochs=args.epochs, lr=1e-3, coverage=cov)
        train_s = time.perf_counter() - t0
        idx.set_learned(True, judge_fraction=args.judge_fraction, judge_recall=0.95)
        r, D, I, _ = _device_qps(idx, q, k, steps, ts, dev)
        r.update(_scored(x, q, D, I, truth, 10))
        r["mean_nprobe"] = round(float((idx.probes(q) >= 0).sum()) / q.shape[0], 3)
        r["train_s"] = round(train_s, 2)
        r["heldout"] = {kk: round(v, 4) for kk, v in rep.items()}
        idx.set_learned(False)
        learned[str(cov)] = r

    def best(rows):
        ok = [(r["qps"], key) for key, r in rows.items() if r["recall_at_10"] >= 0.95]
        return max(ok) if ok else (None, None)

    fq, fkey = best(sweep)
    lq, lkey = best(learned)
    target = int(fkey) if fkey else 64
    idx.nprobe = target
    idx.set_form("plain")
    plain, D, I, st = _device_qps(idx, q, k, max(1, steps // 2), ts, dev)
    plain.update(_scored(x, q, D, I, truth, 10))
    plain.update(_plain_work(st))
    plain["nprobe"] = target
    return {
        "workload": f"{nb} x 128 uint8-valued gmm (4096 components, sigma {sigma:g}), nlist 1024, k 10, "
                    f"{q.shape[0]} queries; probe network (max nprobe {max_np}) trained on {tq.shape[0]} other "
                    f"queries",
        "bf16_fixed_nprobe": sweep,
        "learned_bf16_by_coverage": learned,
        "fastest_fixed_at_recall_0.95": {"nprobe": fkey, "qps": fq},
        "fastest_learned_at_recall_0.95": {"coverage": lkey, "qps": lq},
        "learned_speedup_at_recall_0.95": round(lq / fq, 3) if lq and fq else None,
        "plain_fp32_at_fixed_nprobe": plain,
    }


def extra_c3(args, ts, dev, steps):
    """1M x 420 float mixture (nlist 2048, nprobe 64): the e4m3 form (4 x k
    exact re-rank), the bf16 form and the plain FP32 scan at k 10 and 100."""
    import harmonyclient_b200 as hb
    from harmonyclient_b200 import datasets
    from oracle import gpu_bruteforce as gb
    nb = args.nb
    x, q = datasets.gmm_dense(nb, args.nq, seed=0)
    idx = hb.Index(420, 2048, 64, hb.METRIC_L2, device=dev)
    idx.train(x)
    idx.add(x)
    truth = {}
    truth["D"], truth["I"] = gb.topk(x, q, 100)
    out = {"workload": f"{nb} x 420 float gmm (2048 components, per-dim mean U[-1,1], sigma 0.3), nlist 2048, "
                       f"nprobe 64, {q.shape[0]} queries"}
    for k in (10, 100):
        idx.preSearch(warmUpSearchList=args.warmup_list, warmUpSearchListSize=k)
        row = {}
        for form in ("fp8", "bf16", "plain"):
            idx.set_form(form)
            if form == "fp8":
                idx.set_batch_params(oversample=4)
            r, D, I, st = _device_qps(idx, q, k, steps if form != "plain" else max(1, steps // 2), ts, dev)
            r.update(_scored(x, q, D, I, truth, 10))
            if k > 10:
                r.update(_scored(x, q, D, I, truth, k))
            if form == "plain":
                r.update(_plain_work(st))
            row[form] = r
        out[f"k{k}"] = row
    return out


def run_lists(args, rank, world, dist):
    """--parallelism lists: one index partitioned by lists over the N ranks
    (harmonyclient_b200.parallel); every rank searches the same query batch
    over its own lists, then one all-gather and the device merge.  `value` is
    the batch's queries/s (strong scaling: the index is fixed, its lists are
    split), timed with CUDA events on the current stream, max over ranks."""
    import torch

    from harmonyclient_b200.parallel import ListShardedIndex

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    W = WORKLOADS[args.workload]
    x, q = workload(args, 0)  # every rank: the same base and queries
    k = W["k"]
    sh = ListShardedIndex(W["d"], W["nlist"], args.nprobe, device=dev)
    sh.train(x)
    sh.add(x)
    sh.index.preSearch(warmUpSearchList=args.warmup_list, warmUpSearchListSize=k)
    base = "bf16" if args.form == "learned" else args.form
    sh.index.set_form(base)
    dq = torch.from_numpy(q).cuda()
    for _ in range(args.warmup):
        sh.search_device(dq, k)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        e0.record()
        for _ in range(args.steps):
            Dm, Im = sh.search_device(dq, k)
        e1.record()
        torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    if rank != 0:
        return None
    sc, ns = _score(x, q, Dm.cpu().numpy(), Im.cpu().numpy(), args.recall_sample, {})
    return {
        "metric": METRIC, "value": round(q.shape[0] * args.steps / (ms / 1e3), 1), "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": {"plain": "f32", "bf16": "bf16", "fp8": "e4m3"}[base], "data": W["data"],
        "config": {"workload": W["desc"].format(nb=args.nb) + f", nlist {W['nlist']}, nprobe {args.nprobe}, k {k}, "
                               f"{q.shape[0]} queries per step, lists split over {world} GPUs",
                   "name": args.workload, "parallelism": f"lists x{world}"},
        "recall_at_10": round(sc["recall"], 4), "recall_vs": f"FP64 brute force on the GPU, {ns} queries",
        "clocks": clk.summary(),
    }


def run_reference(args, rank):
    """The reference's own CPU query path (Index::search, ORIGINAL mode,
    OpenMP over all host cores), compiled from the reference sources into
    oracle/_ref, on the same workload."""
    if rank != 0:
        return None
    from oracle import ref
    if not ref.available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref not built"}
    if not WORKLOADS[args.workload].get("cpu_ref", True):
        return {"impl": "reference", "unavailable": f"workload {args.workload}: the reference's host add() of this "
                                                    "base takes far longer than the bench's time bound"}
    x, q = workload(args, 0)
    nt = os.cpu_count() or 1
    ref.set_threads(nt)
    W = WORKLOADS[args.workload]
    nlist, k = W["nlist"], W["k"]
    R = ref.RefIndex(W["d"], nlist, args.nprobe)
    R.train(x)
    R.add(x)
    m = max(nt, 64)
    t0 = time.perf_counter()
    R.search(q[:m], k)
    dt = time.perf_counter() - t0
    per_step = int(min(q.shape[0], max(m, m * args.ref_step_s / max(dt, 1e-6))))
    for _ in range(args.warmup):
        R.search(q[:per_step], k)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R.search(q[:per_step], k)
    dt = time.perf_counter() - t0
    v = per_step * args.steps / dt
    return {
        "metric": METRIC, "value": round(v, 2), "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": W["data"],
        "impl": "reference",
        "config": {"workload": W["desc"].format(nb=args.nb) + f", nlist {nlist}, nprobe {args.nprobe}, k {k}",
                   "name": args.workload, "queries_per_step": per_step},
        "cpu_baseline": {"value": round(v, 2), "unit": "queries/s", "cores": nt, "kind": "reference",
                         "sample": f"{per_step} queries per step of the {q.shape[0]}-query batch"},
        "e2e": {"value": round(v, 2), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nprobe", type=int, default=None, help="default: the workload's (c4: the per-query maximum)")
    ap.add_argument("--warmup-list", type=int, default=10)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--parallelism", default="replicas", choices=["replicas", "lists"],
                    help="N > 1: replicas (each GPU its own query batch) or one index split by lists")
    ap.add_argument("--form", default="learned", choices=["learned", "bf16", "fp8", "plain"])
    ap.add_argument("--base", default="bf16", choices=["bf16", "fp8", "plain"],
                    help="scan form under the learned probes")
    ap.add_argument("--oversample", type=int, default=4, help="e4m3 form: re-rank at most oversample x k")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--group-size", type=int, default=0, choices=[0, 32, 64, 128],
                    help="queries per group of the tensor-core passes (0: per pass by queries per list)")
    ap.add_argument("--train-queries", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--coverage", type=float, default=0.97)
    ap.add_argument("--judge-fraction", type=float, default=0.01)
    ap.add_argument("--no-graph", dest="graph", action="store_false")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--hard-sigma", type=float, default=80.0,
                    help="sigma of the extra 1M x 128 mixture on which the learned probes are compared")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the other nprobes, the sigma-60 mixture and the 1M x 420 workload")
    ap.add_argument("--nb", type=int, default=None, help="default: the workload's")
    ap.add_argument("--nq", type=int, default=None, help="default: the workload's")
    ap.add_argument("--recall-sample", type=int, default=0, help="queries scored for recall (0: all)")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--ref-step-s", type=float, default=5.0)
    ap.add_argument("--base-file", default=None,
                    help="base vectors (.fvecs / .bvecs / .txt) instead of the workload's synthetic data; the "
                         "workload keeps its nlist, nprobe and k")
    ap.add_argument("--query-file", default=None, help="query vectors for --base-file")
    args = ap.parse_args()
    if args.base_file:
        if not args.query_file:
            raise SystemExit("--base-file needs --query-file")
        nb_f, d_f = _file_info(args.base_file)
        nq_f, _ = _file_info(args.query_file)
        args.nb = min(args.nb or nb_f, nb_f)
        args.nq = min(args.nq or nq_f, nq_f)
        name = f"{os.path.basename(args.base_file)} / {os.path.basename(args.query_file)}"
        WORKLOADS[args.workload] = {**WORKLOADS[args.workload], "files": (args.base_file, args.query_file),
                                    "d": d_f, "desc": "{nb} x " + f"{d_f} vectors of {name}",
                                    "data": f"file: {name}", "per_query": None}
    W = WORKLOADS[args.workload]
    args.nb = W["nb"] if args.nb is None else args.nb
    args.nq = W["nq"] if args.nq is None else args.nq
    args.nprobe = W["nprobe"] if args.nprobe is None else args.nprobe
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if args.parallelism == "lists" and world > 1:
        line = run_lists(args, rank, world, dist)
    else:
        line = run_ours(args, rank, world, dist)
    if line is not None:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
