// noalloc.cu — an exact top-k entry point that allocates no device memory.
//
// Who needs it: callers that must not allocate on the device while they
// serve queries. cudaMalloc synchronizes the whole device, so a serving
// loop with a latency budget cannot afford one per call, and hosts that run
// inside a framework owning the device's memory (a caching allocator or a
// fixed memory pool) may forbid raw cudaMalloc altogether. The regular
// fv_gpu_brute_batch keeps grow-only scratch buffers that it allocates on
// first use and whenever a larger batch arrives; this variant takes its
// scratch from one fixed array linked into the library instead.
//
// The scratch is a file-scope __device__ array of PV_NOALLOC_SCRATCH_BYTES
// (2 MiB); every GPU that loads the library holds it until the process
// exits. Host code cannot use the array's name as a device address (in
// host code it names a host-side stand-in), so the first call on each
// device looks up the real address with cudaGetSymbolAddress and caches it;
// that first call should therefore come before any stream capture.
// All calls share the one array and it keeps the previous call's contents:
// everything that must start at a known value is reset by each call, and
// calls that overlap on the GPU (two host threads, two indexes on one
// device) race on it, so callers must serialize them.
#include <string.h>

#include <mutex>

#include "paves_ext.h"
#include "pv_internal.h"

namespace {

constexpr size_t PV_NOALLOC_SCRATCH_BYTES = 2u << 20;
__device__ __align__(256) unsigned char pv_noalloc_scratch[PV_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_mu;
void *g_scratch[NOALLOC_MAX_DEVICES];  // per-device address of the array

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device address of the scratch array on the current device (set up once).
void *scratch_for(int device, char *errbuf, size_t errlen) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
        snprintf(errbuf, errlen, "gpu: device %d out of range", device);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, pv_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            snprintf(errbuf, errlen, "gpu: cudaGetSymbolAddress failed: %s",
                     cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch[device] = p;
    }
    return g_scratch[device];
}

}  // namespace

using namespace pv;

extern "C" int pv_brute_batch_noalloc(FvGpuIndex *g, int nq, const float *d_queries,
                                      uint32_t topb, FvHit *d_out, uint32_t *d_cnt,
                                      char *errbuf, size_t errlen) {
    char dummy[8];
    if (!errbuf || !errlen) {
        errbuf = dummy;
        errlen = sizeof(dummy);
    }
    if (!g || !d_queries || !d_out || !d_cnt) {
        snprintf(errbuf, errlen, "gpu: null argument");
        return -1;
    }
    if (nq < 1 || nq > PV_NOALLOC_MAX_BATCH || topb < 1 || topb > PV_NOALLOC_MAX_TOPB) {
        snprintf(errbuf, errlen,
                 "gpu: no-alloc batch limited to nq <= %d and topb <= %d (got nq=%d topb=%u)",
                 PV_NOALLOC_MAX_BATCH, PV_NOALLOC_MAX_TOPB, nq, topb);
        return -1;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    unsigned char *base = (unsigned char *)scratch_for(g->device, errbuf, errlen);
    if (!base) return -1;

    ScanPlan pl;
    if (!plan_scan_f32(g->count, g->dpad, nq, (int)topb, g->sm_count, pl)) {
        snprintf(errbuf, errlen, "gpu: dimension %d not supported by the scan", g->dim);
        return -1;
    }
    // at most one CTA group per SM: bounds the partial lists to
    // nq * sm_count * topb keys
    int grow = g->sm_count / pl.qtiles;
    if (grow < 1) grow = 1;
    if (grow < pl.grow) {
        uint64_t rpc = (g->count + grow - 1) / grow;
        rpc = (rpc + 31) & ~31ull;
        pl.rows_per_cta = rpc;
        pl.grow = (int)((g->count + rpc - 1) / rpc);
        pl.merge_smem = (size_t)pl.M * 8 + (size_t)pl.grow * 8;
    }

    // carve the scratch: padded queries, per-query program ids (-1), bound,
    // partial lists and their counts
    const size_t off_q = 0;
    const size_t off_prog = off_q + al256((size_t)nq * g->dpad * 4);
    const size_t off_tau = off_prog + al256((size_t)nq * 4);
    const size_t off_part = off_tau + al256((size_t)nq * 8);
    const size_t off_pcnt = off_part + al256((size_t)nq * pl.grow * topb * 8);
    const size_t off_pop = off_pcnt + al256((size_t)nq * pl.grow * 4);
    const size_t need = off_pop + 256;
    if (need > PV_NOALLOC_SCRATCH_BYTES) {
        snprintf(errbuf, errlen, "gpu: no-alloc scratch too small (%zu > %zu bytes)", need,
                 PV_NOALLOC_SCRATCH_BYTES);
        return -1;
    }
    float *q = (float *)(base + off_q);
    int32_t *qprog = (int32_t *)(base + off_prog);
    unsigned long long *tau = (unsigned long long *)(base + off_tau);
    uint64_t *part = (uint64_t *)(base + off_part);
    uint32_t *pcnt = (uint32_t *)(base + off_pcnt);
    unsigned long long *pop = (unsigned long long *)(base + off_pop);
    uint8_t *trunc = (uint8_t *)(pop + 1);

    cudaStream_t st = g->stream;
    // queries: [nq][dim] -> [nq][dpad] rows with zero padding
    if (g->dpad == g->dim) {
        PV_CUDA_OK(cudaMemcpyAsync(q, d_queries, (size_t)nq * g->dim * 4,
                                   cudaMemcpyDeviceToDevice, st),
                   errbuf, errlen);
    } else {
        PV_CUDA_OK(cudaMemsetAsync(q, 0, (size_t)nq * g->dpad * 4, st), errbuf, errlen);
        PV_CUDA_OK(cudaMemcpy2DAsync(q, (size_t)g->dpad * 4, d_queries, (size_t)g->dim * 4,
                                     (size_t)g->dim * 4, nq, cudaMemcpyDeviceToDevice, st),
                   errbuf, errlen);
    }
    // no predicate (-1), bounds start at the largest key
    PV_CUDA_OK(cudaMemsetAsync(qprog, 0xFF, (size_t)nq * 4, st), errbuf, errlen);
    PV_CUDA_OK(cudaMemsetAsync(tau, 0xFF, (size_t)nq * 8, st), errbuf, errlen);

    ScanF32Args a;
    a.vecs = g->d_vecs;
    a.nrows = g->count;
    a.dpad = g->dpad;
    a.queries = q;
    a.nq = nq;
    a.bitmaps = nullptr;
    a.bm_words = (g->count + 31) / 32;
    a.qprog = qprog;
    a.K = (int)topb;
    a.S = pl.S;
    a.CB = pl.CB;
    a.rows_per_cta = pl.rows_per_cta;
    a.grow = pl.grow;
    a.qtiles = pl.qtiles;
    a.tau = tau;
    a.part = part;
    a.part_cnt = pcnt;
    PV_CUDA_OK(launch_scan_f32(a, pl, st), errbuf, errlen);
    PV_CUDA_OK(launch_merge(part, pcnt, pl.grow, (int)topb, pl, tau, qprog, pop, g->count, nq,
                            d_out, d_cnt, trunc, st),
               errbuf, errlen);
    PV_CUDA_OK(cudaStreamSynchronize(st), errbuf, errlen);
    return 0;
}
