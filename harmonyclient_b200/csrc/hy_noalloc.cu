// Search entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they serve queries: a process whose
// device memory is owned by another allocator (a framework's caching pool or a
// fixed arena reserved at start-up) must not grab memory behind that
// allocator's back, and cudaMalloc can synchronise the device and fail under
// memory pressure in the middle of serving.  hy_index_search_preassigned_noalloc
// serves them: the caller passes device buffers for the queries, probe lists
// and results, and every temporary the scan needs lives in one file-scope
// __device__ array of fixed size (NOALLOC_SCRATCH_BYTES), which each GPU that
// loads the library holds until the process exits.
//
// The array is shared by all calls on a device and keeps the last call's
// contents; the entry point clears what must start at zero (status word,
// counters, per-query thresholds) at the start of each call.  Calls whose GPU
// work overlaps (two host threads, or two streams) race on the array and must
// be serialised by the caller.  A call holds the index's call lock from its
// first read of the index until its work has completed on the device, so
// add / load / reset on the same index from another thread wait for it.
#include <mutex>

#include "../../include/hy.h"
#include "hy_kernels.cuh"

namespace hy {
struct IndexView {
    ArenaLayout L;
    const float* codes;
    const int64_t* list_off;
    const int32_t* list_size;
    const int64_t* ids;
    int metric;
    size_t d, nlist;
    int device;
    bool trained, has_lists;
};
int index_view(const hy_index* h, IndexView* v);
int set_error(int code, const char* msg);
std::mutex& index_mutex(hy_index* h);
}  // namespace hy

namespace {

// Fixed scratch: 8 MiB per device.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(8) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch for each device, looked up once per
// device with that device current (the host-side symbol is only a stand-in,
// not a device address).
constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_scratch_ptr[MAX_DEVICES] = {};

int scratch_for_device(int device, unsigned char** out) {
    if (device < 0 || device >= MAX_DEVICES) return hy::set_error(HY_ERR_ARG, "noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return hy::set_error(HY_ERR_CUDA, "noalloc: cudaGetSymbolAddress of the scratch array failed");
        g_scratch_ptr[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
    return HY_OK;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Copy of the probe lists with every id outside [-1, nlist) replaced by -1;
// such an id raises the status word (reported as HY_ERR_ARG).
__global__ void sanitize_probes_kernel(const int64_t* __restrict__ in, int64_t n, int64_t nlist,
                                       int64_t* __restrict__ out, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t l = in[i];
        const bool ok = l >= -1 && l < nlist;
        out[i] = ok ? l : -1;
        if (!ok) atomicExch(bad, 1);
    }
}

}  // namespace

// See include/hy.h.  The first call on a device looks up the scratch array's
// device address; make that first call before any stream capture.
extern "C" int hy_index_search_preassigned_noalloc(hy_index* h, size_t n, const float* dq, size_t k, size_t nprobe,
                                                   const int64_t* dprobes, float* dD, int64_t* dI, void* stream) {
    if (!h || (n > 0 && (!dq || !dprobes || !dD || !dI)))
        return hy::set_error(HY_ERR_ARG, "search_preassigned_noalloc: NULL argument");
    if (n == 0) return HY_OK;
    if (k < 1 || k > HY_MAX_K) return hy::set_error(HY_ERR_ARG, "search_preassigned_noalloc: k must be in [1, 256]");
    if (nprobe < 1) return hy::set_error(HY_ERR_ARG, "search_preassigned_noalloc: nprobe must be >= 1");
    // Held until the final synchronisation: the scan and merge read the
    // index's arena, list tables and ids, which add / load / reset replace.
    std::lock_guard<std::mutex> index_lock(hy::index_mutex(h));
    hy::IndexView v;
    int rc = hy::index_view(h, &v);
    if (rc != HY_OK) return rc;
    if (!v.trained || !v.has_lists) return hy::set_error(HY_ERR_STATE, "search_preassigned_noalloc: index has no lists");
    if (cudaSetDevice(v.device) != cudaSuccess) return hy::set_error(HY_ERR_CUDA, "search_preassigned_noalloc: cudaSetDevice");
    unsigned char* base = nullptr;
    rc = scratch_for_device(v.device, &base);
    if (rc != HY_OK) return rc;

    // Same split of the probe lists over CTAs as the allocating entry points.
    const int kp = k <= 32 ? 32 : k <= 64 ? 64 : k <= 128 ? 128 : 256;
    int nsplit = 1;
    const size_t target_ctas = 2 * 148;
    if (n < target_ctas) nsplit = (int)std::min<size_t>((target_ctas + n - 1) / n, nprobe);
    while ((nprobe + nsplit - 1) / nsplit > 2048) ++nsplit;

    // Scratch layout: status word, counters, thresholds, probes, parts.
    const size_t off_err = 0, off_cnt = 256, off_thr = 512;
    const size_t off_probes = off_thr + align256(n * sizeof(uint32_t));
    const size_t off_parts = off_probes + align256(n * nprobe * sizeof(int64_t));
    const size_t need = off_parts + n * (size_t)nsplit * kp * sizeof(uint64_t);
    if (need > NOALLOC_SCRATCH_BYTES)
        return hy::set_error(HY_ERR_ARG,
                             "search_preassigned_noalloc: the batch needs more than the 8 MiB scratch "
                             "(n * nprobe * 8 + n * nsplit * K' * 8 bytes); search fewer queries per call");
    int* err = reinterpret_cast<int*>(base + off_err);
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(base + off_cnt);
    uint32_t* gthr = reinterpret_cast<uint32_t*>(base + off_thr);
    int64_t* probes = reinterpret_cast<int64_t*>(base + off_probes);
    uint64_t* parts = reinterpret_cast<uint64_t*>(base + off_parts);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(gthr, 0xff, n * sizeof(uint32_t), s) != cudaSuccess)
        return hy::set_error(HY_ERR_CUDA, "search_preassigned_noalloc: clearing the scratch failed");
    const int64_t np = (int64_t)(n * nprobe);
    sanitize_probes_kernel<<<(int)std::min<int64_t>((np + 255) / 256, 1 << 20), 256, 0, s>>>(dprobes, np,
                                                                                          (int64_t)v.nlist, probes, err);
    hy::ScanParams p;
    p.L = v.L;
    p.codes = v.codes;
    p.list_off = v.list_off;
    p.list_size = v.list_size;
    p.q = dq;
    p.probes = probes;
    p.init_thr = nullptr;
    p.g_thr = nsplit > 1 ? gthr : nullptr;
    p.out = parts;
    p.counters = counters;
    p.err = err;
    p.nq = (int)n;
    p.nprobe = (int)nprobe;
    p.nsplit = nsplit;
    p.k = (int)k;
    p.metric = v.metric;
    p.prune = 1;
    int smem = 0;
    if (hy::launch_scan_plain(p, &smem, s) != cudaSuccess)
        return hy::set_error(HY_ERR_CUDA, "search_preassigned_noalloc: scan launch failed");
    if (hy::launch_merge(parts, (int)n, nsplit, kp, (int)k, v.metric, v.ids, dD, dI, s) != cudaSuccess)
        return hy::set_error(HY_ERR_CUDA, "search_preassigned_noalloc: merge launch failed");
    int herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return hy::set_error(HY_ERR_CUDA, "search_preassigned_noalloc: the search failed on the device");
    if (herr == 1) return hy::set_error(HY_ERR_ARG, "search_preassigned_noalloc: probe list id outside [-1, nlist)");
    if (herr != 0) return hy::set_error(HY_ERR_TIMEOUT, "search_preassigned_noalloc: a device-side wait gave up");
    return HY_OK;
}
