"""Benchmark of the IVF query hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--nprobe 64] [--nb 1000000] [--nq 10000]

Workload (one "step" = one batch search): 1,000,000 x 128 integer-valued
float32 vectors in [0,255] from a 4,096-component Gaussian mixture (seeded,
synthetic), nlist 1024 trained on the GPU, 10,000 queries from the same
mixture, k 100, nprobe 64 (recall@10 against an FP64 brute force is reported
for the first 10 of the 100).  The list arena (~550 MB) is larger than L2,
so no L2 flush is needed between steps.

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


def workload(args, rank):
    from harmonyclient_b200 import datasets
    x, q = datasets.gmm_uint8(args.nb, args.nq, seed=0)
    if rank:
        _, q = datasets.gmm_uint8(args.nb, args.nq, seed=1000 + rank)
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
    R.search(q[:m2], k)
    dt = time.perf_counter() - t0
    return {"value": m2 / dt, "unit": "queries/s", "cores": nt, "kind": "reference",
            "sample": f"{m2} of {q.shape[0]} queries, reference Index::search ORIGINAL mode, OpenMP x{nt}"}


def run_ours(args, rank, world, dist):
    import torch

    import harmonyclient_b200 as hb
    from harmonyclient_b200 import _lib

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    x, q = workload(args, rank)
    nlist, k = 1024, 100
    idx = hb.Index(128, nlist, args.nprobe, hb.METRIC_L2, device=dev)
    t0 = time.perf_counter()
    idx.train(x)
    idx.add(x)
    # Warm-up thresholds as the reference's default run uses them
    # (--warmup_list 10, warmup_list_size = k; src/query.cpp:845-847).
    idx.preSearch(warmUpSearchList=args.warmup_list, warmUpSearchListSize=k)
    idx.set_form(args.form)
    build_s = time.perf_counter() - t0
    cent = idx.centroid_codes

    stream = torch.cuda.current_stream().cuda_stream
    dq = torch.from_numpy(q).cuda()
    dD = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")

    def step():
        idx.search_device(q.shape[0], dq.data_ptr(), k, dD.data_ptr(), dI.data_ptr(), stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * q.shape[0] * args.steps / (ms_max / 1e3)

    # End to end through the public host API: pinned host queries in, results
    # back to pinned host memory, every step.
    hq = torch.from_numpy(q).pin_memory()
    hD = torch.empty((q.shape[0], k), dtype=torch.float32).pin_memory()
    hI = torch.empty((q.shape[0], k), dtype=torch.int64).pin_memory()
    L = _lib.load()
    import ctypes as C

    def e2e_step():
        _lib.check(L.hy_index_search(idx._h, q.shape[0], C.c_void_p(hq.data_ptr()), k, C.c_void_p(hD.data_ptr()),
                                     C.c_void_p(hI.data_ptr())))

    e2e_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    scan_ms, loaded, possible, launches, fallback = [], 0, 0, 0, 0
    for _ in range(args.steps):
        e2e_step()
        st = idx.last_stats()
        scan_ms.append(st["scan_ms"])
        loaded, possible, launches = st["tile_blocks"], st["tile_blocks_max"], st["launches"]
        fallback = max(fallback, st["fallback_queries"])
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], device="cuda")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * q.shape[0] * args.steps / float(te.item())

    if rank != 0:
        return None

    # Roofline of the dominant kernel (the list scan): algorithmic bytes are
    # the pair bytes sum_q sum_{l in probes(q)} |l| * d * 4 plus query and
    # result bytes; the bytes the kernel actually loads after pruning are
    # reported beside them.
    P = idx.probes(q)
    sizes = np.array([idx.list_size(l) for l in range(nlist)], np.int64)
    pair_rows = int(sizes[P].sum())
    alg_bytes = pair_rows * 128 * 4 + q.shape[0] * 128 * 4 + q.shape[0] * k * 12
    scan_avg = statistics.mean(scan_ms)
    hbm_peak, tc_peak, peak_kind = peaks()
    if args.form == "plain":
        achieved = alg_bytes / (scan_avg / 1e3) / 1e9
        loaded_bytes = loaded * 32 * 32 * 4
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(achieved / hbm_peak, 4), "traffic": None, "peak_kind": peak_kind,
                "kernel": "scan_plain_kernel", "kernel_ms": round(scan_avg, 4), "algorithmic_bytes": alg_bytes,
                "loaded_bytes": loaded_bytes, "loaded_frac_of_unpruned": round(loaded / max(possible, 1), 4)}
    else:
        # Algorithmic work of the batched scan: one 2*d-flop inner product per
        # (query, probed row) pair, on the bf16 tensor cores.
        alg_flops = pair_rows * 2 * 128
        achieved = alg_flops / (scan_avg / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": round(achieved, 2), "peak": tc_peak, "unit": "TFLOP/s",
                "frac": round(achieved / tc_peak, 4), "traffic": None, "peak_kind": peak_kind,
                "kernel": "batched_scan_kernel", "kernel_ms": round(scan_avg, 4), "algorithmic_flops": alg_flops,
                "pair_bytes_fp32": alg_bytes}

    # recall@10 against FP64 brute force on a query sample
    from oracle import port
    ns = min(args.recall_sample, q.shape[0])
    Dt, It = port.bruteforce_f64(x, q[:ns], 10)
    I_ours = dI[:ns, :10].cpu().numpy()
    recall10 = float(np.mean([len(set(a) & set(b)) / 10 for a, b in zip(I_ours.tolist(), It.tolist())]))

    cpu = cpu_baseline_ref(x, q, cent, args.nprobe, k, args.cpu_budget)

    h2d = q.nbytes
    d2h = q.shape[0] * k * 12
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
        "dtype": "f32",
        "data": "synthetic (seeded Gaussian mixture, integer-valued in [0,255])",
        "form": args.form,
        "config": {"workload": f"{args.nb} x 128 uint8-valued gmm, nlist {nlist}, nprobe {args.nprobe}, "
                               f"k {k}, {q.shape[0]} queries per step per GPU",
                   "nb": args.nb, "d": 128, "nlist": nlist, "nprobe": args.nprobe, "k": k, "nq": q.shape[0],
                   "l2_flush": "not needed: list arena larger than L2", "parallelism": f"replicas x{world}"},
        "recall_at_10": round(recall10, 4),
        "recall_sample": ns,
        "roofline": roof,
        "e2e": {"value": round(e2e_value, 1), "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches) * args.steps,
        "warmup_list": args.warmup_list,
        "fallback_queries": fallback,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "build_s": round(build_s, 2),
    }
    return line


def run_reference(args, rank):
    """The reference's own CPU query path (Index::search, ORIGINAL mode,
    OpenMP over all host cores), compiled from the reference sources into
    oracle/_ref, on the same workload."""
    if rank != 0:
        return None
    from oracle import ref
    if not ref.available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref not built"}
    x, q = workload(args, 0)
    nt = os.cpu_count() or 1
    ref.set_threads(nt)
    nlist, k = 1024, 100
    R = ref.RefIndex(128, nlist, args.nprobe)
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
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"{args.nb} x 128 uint8-valued gmm, nlist {nlist}, nprobe {args.nprobe}, k {k}",
                   "queries_per_step": per_step},
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
    ap.add_argument("--nprobe", type=int, default=64)
    ap.add_argument("--warmup-list", type=int, default=10)
    ap.add_argument("--form", default="bf16", choices=["plain", "bf16"])
    ap.add_argument("--nb", type=int, default=1_000_000)
    ap.add_argument("--nq", type=int, default=10_000)
    ap.add_argument("--recall-sample", type=int, default=200)
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--ref-step-s", type=float, default=5.0)
    args = ap.parse_args()
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
    line = run_ours(args, rank, world, dist)
    if line is not None:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
