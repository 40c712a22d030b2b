// index.cu — device-resident index: upload, layout conversion, release.
//
// Replaces fv_gpu_index_upload / fv_gpu_index_free / pick_device
// (gpu_engine.cu:1518-1773). The resident layout differs from the
// reference's on purpose:
//  * exact rows stay FP32 with the row stride rounded to 16 bytes, so a
//    warp fetches a 128-dim row in one 16-byte-per-lane load;
//  * reduced precision (BF16 / FP8-E4M3 with a per-row scale) is an extra
//    copy beside the FP32 rows, which the exact re-rank reads; the row
//    stride is padded to a multiple of 64 elements (128 B for BF16) for the
//    tensor-core scan; per-row squared norms of the stored representation
//    feed the norm-form distance;
//  * the level-0 graph ([cnt, neigh...] rows of stride 2M+1) becomes a
//    fixed-width adjacency of deg_cap = 2M u32 slots padded with
//    UINT32_MAX plus a u16 degree array: 128-byte aligned neighbour rows;
//  * attribute columns stay f64 (predicate semantics are f64 compares).
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "index.h"
#include "paves_ext.h"
#include "pv_internal.h"

namespace pv {

// fp32 rows -> bf16 rows (zero padded to kpad) + squared norm of the bf16 row
__global__ void to_bf16_kernel(const float *__restrict__ src, int dpad, int dim,
                               uint64_t nrows, __nv_bfloat16 *__restrict__ dst, int kpad,
                               float *__restrict__ norm) {
    const int lane = threadIdx.x & 31;
    uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (row >= nrows) return;
    float acc = 0.f;
    for (int j = lane; j < kpad; j += 32) {
        float v = j < dim ? src[row * dpad + j] : 0.f;
        __nv_bfloat16 b = __float2bfloat16_rn(v);
        dst[row * kpad + j] = b;
        float r = __bfloat162float(b);
        acc = fmaf(r, r, acc);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) norm[row] = acc;
}

// ||x||^2 of the f32 rows (one warp per row) and their maximum (the bits
// of non-negative floats order like the floats)
__global__ void norm32_kernel(const float *__restrict__ src, int dpad, uint64_t nrows,
                              float *__restrict__ norm, unsigned *__restrict__ nmax) {
    const int lane = threadIdx.x & 31;
    uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (row >= nrows) return;
    float acc = 0.f;
    for (int j = lane; j < dpad; j += 32) {
        const float v = src[row * dpad + j];
        acc = fmaf(v, v, acc);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        norm[row] = acc;
        atomicMax(nmax, __float_as_uint(acc));
    }
}

// fp32 rows -> fp8-e4m3 rows with one scale per row (absmax / 448), plus
// the squared norm of the dequantized row.
__global__ void to_fp8_kernel(const float *__restrict__ src, int dpad, int dim,
                              uint64_t nrows, __nv_fp8_e4m3 *__restrict__ dst, int kpad,
                              float *__restrict__ scale, float *__restrict__ norm) {
    const int lane = threadIdx.x & 31;
    uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (row >= nrows) return;
    float amax = 0.f;
    for (int j = lane; j < dim; j += 32) amax = fmaxf(amax, fabsf(src[row * dpad + j]));
    for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const float s = amax > 0.f ? amax / 448.f : 1.f;
    const float inv = 1.f / s;
    float acc = 0.f;
    for (int j = lane; j < kpad; j += 32) {
        float v = j < dim ? src[row * dpad + j] * inv : 0.f;
        __nv_fp8_e4m3 b(v);
        dst[row * kpad + j] = b;
        float r = float(b) * s;
        acc = fmaf(r, r, acc);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        norm[row] = acc;
        scale[row] = s;
    }
}

// [cnt, n0, n1, ...] rows of stride l0_stride -> fixed-width adjacency.
// Out-of-range neighbour ids are dropped (they would otherwise be followed).
__global__ void adj_kernel(const uint32_t *__restrict__ l0, uint32_t l0_stride,
                           uint64_t nrows, int deg_cap, uint32_t *__restrict__ adj,
                           uint16_t *__restrict__ deg) {
    uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const uint32_t *src = l0 + row * l0_stride;
    uint32_t cnt = src[0];
    if (cnt > l0_stride - 1) cnt = l0_stride - 1;
    int n = 0;
    for (uint32_t i = 0; i < cnt && n < deg_cap; i++) {
        uint32_t v = src[1 + i];
        if (v < nrows) adj[row * deg_cap + n++] = v;
    }
    deg[row] = (uint16_t)n;
    for (int i = n; i < deg_cap; i++) adj[row * deg_cap + i] = 0xFFFFFFFFu;
}

static int pick_device(size_t need) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        (void)cudaGetLastError();
        return -1;
    }
    int best = -1;
    size_t bestfree = 0;
    int cur = 0;
    cudaGetDevice(&cur);
    for (int i = 0; i < n; i++) {
        if (cudaSetDevice(i) != cudaSuccess) continue;
        size_t f = 0, t = 0;
        if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
            (void)cudaGetLastError();
            continue;
        }
        if (f > bestfree && f > need + (512ull << 20)) {
            bestfree = f;
            best = i;
        }
    }
    cudaSetDevice(best >= 0 ? best : cur);
    (void)cudaGetLastError();
    return best;
}

}  // namespace pv

// Largest |value| of an array if every value is an integer of magnitude
// <= 256 (exactly representable in bf16), else -1.
float pv_integral_amax(const float *v, uint64_t n) {
    float amax = 0.f;
    for (uint64_t i = 0; i < n; i++) {
        const float x = v[i];
        if (x != floorf(x)) return -1.f;
        const float a = fabsf(x);
        if (a > amax) amax = a;
        if (amax > 256.f) return -1.f;
    }
    return amax;
}

// True when bf16 tensor-core distances are exact for rows with integral
// max row_amax and queries with integral max q_amax: the norm form's
// largest intermediate, ||x||^2 + ||q||^2 <= dim * (row_amax^2 + q_amax^2),
// and every partial dot product stay below 2^24.
bool pv_bf16_exact(int dim, float row_amax, float q_amax) {
    if (row_amax < 0.f || q_amax < 0.f) return false;
    const double worst = (double)dim * ((double)row_amax * row_amax + (double)q_amax * q_amax);
    return worst < 16777216.0;
}

namespace pv {

// The dynamic shared-memory limit is a per-function, per-device attribute
// that every launch must fit, including kernel nodes of CUDA graphs captured
// earlier. Launch sites therefore only ever raise it: a graph captured with
// a large size stays launchable after a later call asks for a smaller one.
cudaError_t raise_smem_limit(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t &cur = limit[{fn, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

}  // namespace pv

using namespace pv;

extern "C" int fv_gpu_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return n > 0;
}

extern "C" int fv_gpu_index_device(const FvGpuIndex *g) { return g ? g->device : -1; }
extern "C" int fv_gpu_index_precision(const FvGpuIndex *g) { return g ? g->precision : -1; }

extern "C" void fv_gpu_index_free(FvGpuIndex *g) {
    if (!g) return;
    if (g->device >= 0) cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (!g->view) {  // a view borrows the device data of its parent
        cudaFree(g->d_vecs);
        cudaFree(g->d_cols);
        cudaFree(g->d_prows);
        cudaFree(g->d_adj);
        cudaFree(g->d_deg);
        cudaFree(g->d_vlow);
        cudaFree(g->d_vscale);
        cudaFree(g->d_norm);
        cudaFree(g->d_norm32);
    }
    Buf *bufs[] = {&g->scan.stage_h, &g->scan.stage_d, &g->scan.bitmaps, &g->scan.popcnt,
                   &g->scan.tau, &g->scan.part, &g->scan.part_cnt, &g->scan.cand,
                   &g->scan.out_d, &g->scan.out_h, &g->scan.sparse, &g->graph.visited, &g->graph.res,
                   &g->graph.stats, &g->graph.route, &g->graph.route_h, &g->graph.gout};
    for (Buf *b : bufs) b->release();
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    for (cudaEvent_t e : g->rev)
        if (e) cudaEventDestroy(e);
    if (g->stream) cudaStreamDestroy(g->stream);
    if (g->stream2) cudaStreamDestroy(g->stream2);
    delete g;
}

namespace {

// Low-precision rows, norms and scales made by an earlier upload (read back
// with pv_index_export and stored beside the index file).
struct Prepared {
    const void *vlow;
    const float *norm;
    const float *scale;  // FP8 only
    float row_amax;
};

FvGpuIndex *upload_impl(const float *vectors, const double *cols, const uint32_t *post_rows,
                        const uint32_t *l0, uint32_t l0_stride, uint64_t count, int dim,
                        int ncols, int device, int precision, const Prepared *prep,
                        char *errbuf, size_t errlen) {
    auto fail = [&](const char *what, cudaError_t e) -> FvGpuIndex * {
        if (errbuf && errlen)
            snprintf(errbuf, errlen, "gpu: index upload: %s%s%s", what, e ? ": " : "",
                     e ? cudaGetErrorString(e) : "");
        return nullptr;
    };
    if (!vectors || count == 0 || dim <= 0) return fail("empty index", cudaSuccess);
    if (count >= 0xFFFFFFFFull) return fail("too many rows (row ids are u32)", cudaSuccess);
    if (ncols < 0 || ncols > 32) return fail("ncols out of range", cudaSuccess);
    if (ncols > 0 && (!cols || !post_rows)) return fail("columns missing", cudaSuccess);
    if (precision < FV_GPU_PREC_FP32 || precision > FV_GPU_PREC_FP8)
        return fail("unknown precision", cudaSuccess);
    if (l0 && l0_stride < 2) return fail("bad l0 stride", cudaSuccess);
    if (prep && (precision == FV_GPU_PREC_FP32 || !prep->vlow || !prep->norm ||
                 (precision == FV_GPU_PREC_FP8 && !prep->scale)))
        return fail("prepared arrays missing for this precision", cudaSuccess);

    const int dpad = (dim + 3) & ~3;
    // low-precision row stride: whole 128-byte swizzle rows
    const int kpad = precision == FV_GPU_PREC_FP8 ? (dim + 127) & ~127 : (dim + 63) & ~63;
    const uint64_t rows_pad = (count + 127) & ~127ull;  // norms/scales per 128-row tile
    size_t need = count * (size_t)dpad * 4 + count * (size_t)ncols * 12;
    if (l0) need += count * (size_t)(l0_stride - 1) * 4 + count * 2;
    if (precision != FV_GPU_PREC_FP32) need += count * (size_t)kpad * 2 + count * 8;
    if (device < 0) device = pick_device(need);
    if (device < 0) return fail("no CUDA device with enough free memory", cudaSuccess);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail("cudaSetDevice", e);

    FvGpuIndex *g = new FvGpuIndex();
    g->device = device;
    g->precision = precision;
    g->count = count;
    g->dim = dim;
    g->ncols = ncols;
    g->l0_stride = l0 ? l0_stride : 0;
    g->dpad = dpad;
    g->kpad = kpad;
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, device);
    auto bail = [&](const char *what, cudaError_t err) -> FvGpuIndex * {
        fail(what, err);
        fv_gpu_index_free(g);
        return nullptr;
    };
    if ((e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail("stream", e);
    if ((e = cudaStreamCreateWithFlags(&g->stream2, cudaStreamNonBlocking)) != cudaSuccess)
        return bail("stream", e);
    cudaEventCreate(&g->ev0);
    cudaEventCreate(&g->ev1);

    // every copy and fill of the upload runs on g->stream, in order with the
    // conversion kernels (the library's streams do not wait for the legacy
    // default stream, and a fill of device memory returns before it runs)
    if ((e = cudaMalloc(&g->d_vecs, count * (size_t)dpad * 4)) != cudaSuccess)
        return bail("rows", e);
    if (dpad == dim) {
        e = cudaMemcpyAsync(g->d_vecs, vectors, count * (size_t)dim * 4, cudaMemcpyHostToDevice,
                            g->stream);
    } else {
        if ((e = cudaMemsetAsync(g->d_vecs, 0, count * (size_t)dpad * 4, g->stream)) == cudaSuccess)
            e = cudaMemcpy2DAsync(g->d_vecs, (size_t)dpad * 4, vectors, (size_t)dim * 4,
                                  (size_t)dim * 4, count, cudaMemcpyHostToDevice, g->stream);
    }
    if (e != cudaSuccess) return bail("rows copy", e);

    if (ncols > 0) {
        if ((e = cudaMalloc(&g->d_cols, count * (size_t)ncols * 8)) != cudaSuccess)
            return bail("columns", e);
        if ((e = cudaMemcpyAsync(g->d_cols, cols, count * (size_t)ncols * 8,
                                 cudaMemcpyHostToDevice, g->stream)) != cudaSuccess)
            return bail("columns copy", e);
        if ((e = cudaMalloc(&g->d_prows, count * (size_t)ncols * 4)) != cudaSuccess)
            return bail("postings", e);
        if ((e = cudaMemcpyAsync(g->d_prows, post_rows, count * (size_t)ncols * 4,
                                 cudaMemcpyHostToDevice, g->stream)) != cudaSuccess)
            return bail("postings copy", e);
        pv::build_sorted_cols(g, cols, post_rows);
    }

    if (l0) {
        g->deg_cap = (int)l0_stride - 1;
        uint32_t *d_l0 = nullptr;
        if ((e = cudaMalloc(&d_l0, count * (size_t)l0_stride * 4)) != cudaSuccess)
            return bail("graph staging", e);
        e = cudaMemcpyAsync(d_l0, l0, count * (size_t)l0_stride * 4, cudaMemcpyHostToDevice,
                            g->stream);
        if (e == cudaSuccess) e = cudaMalloc(&g->d_adj, count * (size_t)g->deg_cap * 4);
        if (e == cudaSuccess) e = cudaMalloc(&g->d_deg, count * 2);
        if (e == cudaSuccess) {
            adj_kernel<<<(unsigned)((count + 255) / 256), 256, 0, g->stream>>>(
                d_l0, l0_stride, count, g->deg_cap, g->d_adj, g->d_deg);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        cudaFree(d_l0);
        if (e != cudaSuccess) return bail("graph", e);
    }

    // the BF16 exactness certificate's input: scanned here, or stored
    g->row_amax = prep ? prep->row_amax : pv_integral_amax(vectors, count * (uint64_t)dim);

    // f32 row norms for the exact mode's tensor-core scan (padded to whole
    // 128-row tiles, then the maximum's word)
    {
        const size_t rows_pad32 = (size_t)((count + 127) / 128) * 128;
        if ((e = cudaMalloc(&g->d_norm32, rows_pad32 * 4 + 16)) != cudaSuccess)
            return bail("f32 norms", e);
        unsigned *d_max = (unsigned *)(g->d_norm32 + rows_pad32);
        unsigned h_max = 0;
        if ((e = cudaMemsetAsync(g->d_norm32, 0, rows_pad32 * 4 + 16, g->stream)) != cudaSuccess)
            return bail("f32 norms", e);
        norm32_kernel<<<(unsigned)((count + 7) / 8), 256, 0, g->stream>>>(g->d_vecs, dpad, count,
                                                                         g->d_norm32, d_max);
        if ((e = cudaGetLastError()) != cudaSuccess) return bail("f32 norms", e);
        if ((e = cudaMemcpyAsync(&h_max, d_max, 4, cudaMemcpyDeviceToHost, g->stream)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(g->stream)) != cudaSuccess)
            return bail("f32 norms", e);
        memcpy(&g->norm32_max, &h_max, 4);
    }

    if (precision != FV_GPU_PREC_FP32) {
        const bool f8 = precision == FV_GPU_PREC_FP8;
        const size_t esz = f8 ? 1 : 2;
        if ((e = cudaMalloc(&g->d_vlow, count * (size_t)kpad * esz)) != cudaSuccess)
            return bail("low-precision rows", e);
        if ((e = cudaMalloc(&g->d_norm, rows_pad * 4)) != cudaSuccess) return bail("norms", e);
        if ((e = cudaMemsetAsync(g->d_norm, 0, rows_pad * 4, g->stream)) != cudaSuccess)
            return bail("norms", e);
        unsigned blocks = (unsigned)((count + 7) / 8);
        if (prep) {
            // straight copies of the stored device layout
            e = cudaMemcpyAsync(g->d_vlow, prep->vlow, count * (size_t)kpad * esz,
                                cudaMemcpyHostToDevice, g->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(g->d_norm, prep->norm, count * 4, cudaMemcpyHostToDevice,
                                    g->stream);
            if (e == cudaSuccess && f8) {
                if ((e = cudaMalloc(&g->d_vscale, rows_pad * 4)) == cudaSuccess &&
                    (e = cudaMemsetAsync(g->d_vscale, 0, rows_pad * 4, g->stream)) == cudaSuccess)
                    e = cudaMemcpyAsync(g->d_vscale, prep->scale, count * 4,
                                        cudaMemcpyHostToDevice, g->stream);
            }
            if (e != cudaSuccess) return bail("prepared rows", e);
        } else if (f8) {
            if ((e = cudaMalloc(&g->d_vscale, rows_pad * 4)) != cudaSuccess)
                return bail("scales", e);
            if ((e = cudaMemsetAsync(g->d_vscale, 0, rows_pad * 4, g->stream)) != cudaSuccess)
                return bail("scales", e);
            to_fp8_kernel<<<blocks, 256, 0, g->stream>>>(g->d_vecs, dpad, dim, count,
                                                         (__nv_fp8_e4m3 *)g->d_vlow, kpad,
                                                         g->d_vscale, g->d_norm);
        } else {
            to_bf16_kernel<<<blocks, 256, 0, g->stream>>>(g->d_vecs, dpad, dim, count,
                                                          (__nv_bfloat16 *)g->d_vlow, kpad,
                                                          g->d_norm);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return bail("convert", e);
    }
    // the caller's arrays may go once this returns
    if ((e = cudaStreamSynchronize(g->stream)) != cudaSuccess) return bail("upload", e);
    return g;
}

}  // namespace

extern "C" FvGpuIndex *fv_gpu_index_upload(const float *vectors, const double *cols,
                                           const uint32_t *post_rows, const uint32_t *l0,
                                           uint32_t l0_stride, uint64_t count, int dim,
                                           int ncols, int device, int precision,
                                           char *errbuf, size_t errlen) {
    return upload_impl(vectors, cols, post_rows, l0, l0_stride, count, dim, ncols, device,
                       precision, nullptr, errbuf, errlen);
}

extern "C" FvGpuIndex *pv_index_upload_prepared(const float *vectors, const double *cols,
                                                const uint32_t *post_rows, const uint32_t *l0,
                                                uint32_t l0_stride, uint64_t count, int dim,
                                                int ncols, int device, int precision,
                                                const void *vlow, const float *norms,
                                                const float *scales, float row_amax,
                                                char *errbuf, size_t errlen) {
    const Prepared p{vlow, norms, scales, row_amax};
    return upload_impl(vectors, cols, post_rows, l0, l0_stride, count, dim, ncols, device,
                       precision, &p, errbuf, errlen);
}

extern "C" int64_t pv_index_part_bytes(const FvGpuIndex *g, int part) {
    if (!g || g->precision == FV_GPU_PREC_FP32 || !g->d_vlow) return -1;
    const size_t esz = g->precision == FV_GPU_PREC_FP8 ? 1 : 2;
    switch (part) {
        case PV_PART_LOWP_ROWS: return (int64_t)(g->count * (size_t)g->kpad * esz);
        case PV_PART_NORMS: return (int64_t)(g->count * 4);
        case PV_PART_SCALES: return g->precision == FV_GPU_PREC_FP8 ? (int64_t)(g->count * 4) : -1;
    }
    return -1;
}

extern "C" int pv_index_export(FvGpuIndex *g, int part, void *dst, uint64_t bytes,
                               float *row_amax, char *errbuf, size_t errlen) {
    const int64_t need = pv_index_part_bytes(g, part);
    if (need < 0 || !dst || bytes != (uint64_t)need) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "export: no such part or wrong size");
        return -1;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    const void *src = part == PV_PART_LOWP_ROWS ? g->d_vlow
                      : part == PV_PART_NORMS  ? (const void *)g->d_norm
                                               : (const void *)g->d_vscale;
    PV_CUDA_OK(cudaMemcpyAsync(dst, src, (size_t)need, cudaMemcpyDeviceToHost, g->stream), errbuf,
               errlen);
    PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
    if (row_amax) *row_amax = g->row_amax;
    return 0;
}

extern "C" int fv_gpu_mem_probe(uint64_t *free_bytes, uint64_t *total_bytes) {
    static int probed = -2;
    if (probed == -2) probed = pick_device(0);
    if (probed < 0) return -1;
    size_t f = 0, t = 0;
    if (cudaSetDevice(probed) != cudaSuccess || cudaMemGetInfo(&f, &t) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1;
    }
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return probed;
}

namespace pv {

// A handle that shares g's device data and owns its own stream, events and
// scratch: work captured into CUDA graphs on the view keeps fixed scratch
// addresses whatever other calls do on g. Freed with fv_gpu_index_free
// (scratch only); must not outlive g.
FvGpuIndex *index_view(const FvGpuIndex *g) {
    FvGpuIndex *v = new FvGpuIndex();
    v->device = g->device;
    v->precision = g->precision;
    v->count = g->count;
    v->dim = g->dim;
    v->ncols = g->ncols;
    v->l0_stride = g->l0_stride;
    v->dpad = g->dpad;
    v->d_vecs = g->d_vecs;
    v->d_cols = g->d_cols;
    v->d_prows = g->d_prows;
    v->d_adj = g->d_adj;
    v->d_deg = g->d_deg;
    v->deg_cap = g->deg_cap;
    v->kpad = g->kpad;
    v->d_vlow = g->d_vlow;
    v->d_vscale = g->d_vscale;
    v->d_norm = g->d_norm;
    v->d_norm32 = g->d_norm32;
    v->norm32_max = g->norm32_max;
    v->exact_tc = g->exact_tc;
    v->row_amax = g->row_amax;
    v->sorted_cols = g->sorted_cols;
    v->sm_count = g->sm_count;
    v->view = true;
    if (cudaSetDevice(v->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&v->stream2, cudaStreamNonBlocking) != cudaSuccess) {
        if (v->stream) cudaStreamDestroy(v->stream);
        delete v;
        return nullptr;
    }
    cudaEventCreate(&v->ev0);
    cudaEventCreate(&v->ev1);
    return v;
}

}  // namespace pv
