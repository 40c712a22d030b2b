// scan_f32t.cu — exact FP32 filtered L2 scan for query tiles of 32 or 64
// queries: the register-blocked form of the exact scan (scan_f32.cu keeps
// the small tiles, where the scan is bandwidth-bound).
//
// Same results as scan_f32_kernel: squared L2 in the difference form
// (x - q)^2 summed in FP32 (the CPU cursor's l2sq, engine.cpp:43-90), the
// predicate as one bitmap bit, canonical (dist, id) keys, per-CTA top-K
// lists for merge_kernel. Different organisation: a CTA holds its query
// tile in shared memory and streams row tiles of 128 rows through shared
// memory in chunks of 32 dims (cp.async, three chunks in flight); each
// thread owns 8 rows x (QT / 16) queries and accumulates their distances
// in registers with packed FP32 pairs (sub.rn.f32x2 / fma.rn.f32x2: two
// dims per instruction, each lane's rounding identical to sub / fma.rn).
// Per 4 dims a thread issues 8 + QT/16 shared loads for 8 * QT/16 * 4
// packed operations, so the FP32 pipe, not the issue slots or shared
// memory, bounds the kernel: 2 FP32 operations per (row, query, dim).
// After a tile, each (row, query) distance that beats its query's bound
// and passes its filter bit joins the query's candidate buffer
// (topk.cuh), flushed by a bitonic sort when it may overflow.
#include "common.cuh"
#include "pv_internal.h"
#include "sm100.cuh"
#include "topk.cuh"

namespace pv {

constexpr int FT_RT = 128;         // rows per tile
constexpr int FT_CH = 32;          // dims per staged chunk
constexpr int FT_XS = FT_CH + 4;   // padded row stride of a staged chunk (floats)
constexpr int FT_NSTG = 3;         // chunks in flight
constexpr int FT_RPT = 8;          // rows per thread (rows tr + 16 i)
constexpr int FT_CB = 192;         // candidate buffer per query
constexpr int FT_S = 256;          // region per query: K (<= 64) + buffer

__device__ __forceinline__ uint64_t f2_pack(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float f2_sum(uint64_t v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return lo + hi;
}
// acc += (x - q) * (x - q) on both halves of the pairs
__device__ __forceinline__ void f2_sqdiff_acc(uint64_t &acc, uint64_t x, uint64_t q) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(q));
    asm("fma.rn.f32x2 %0, %1, %1, %0;" : "+l"(acc) : "l"(d));
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sm100::smem_u32(dst)),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

size_t scan_f32t_smem(int qt, int dp) {
    const size_t qs = (size_t)qt * (dp + 4) * 4;
    const size_t xs = (size_t)FT_NSTG * FT_RT * FT_XS * 4;
    const size_t reg = (size_t)qt * FT_S * 8;
    return qs + xs + reg + (size_t)qt * 8 + (size_t)qt * 4 * 4 + (size_t)(3 * qt + 1) * 4 +
           (size_t)qt * 4 + 16;
}

template <int QT, int DP>
__global__ void __launch_bounds__(256, 1) scan_f32t_kernel(ScanF32Args a) {
    constexpr int QJ = QT / 16;       // queries per thread (tq + 16 j)
    constexpr int NCH = DP / FT_CH;   // chunks per row
    constexpr int QS = DP + 4;        // padded query stride (floats)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = a.K;
    float *sQ = (float *)smem_raw;                      // [QT][QS]
    float *sX = sQ + QT * QS;                           // [NSTG][RT][XS]
    TopkSmem t;
    t.region = (uint64_t *)(sX + FT_NSTG * FT_RT * FT_XS);  // [QT][S]
    t.tau = (unsigned long long *)(t.region + (size_t)QT * FT_S);
    uint32_t *s_bw = (uint32_t *)(t.tau + QT);          // [QT][4] words of the tile
    t.nb = (int *)(s_bw + QT * 4);
    t.nt = t.nb + QT;
    t.flush_list = t.nt + QT;
    int *s_prog = t.flush_list + QT + 1;

    const int tid = threadIdx.x, tq = tid & 15, tr = tid >> 4;
    const int qtile = blockIdx.x % a.qtiles;
    const int rblk = blockIdx.x / a.qtiles;
    const int qt0 = qtile * QT;
    const int dpad = a.dpad;

    for (int i = tid; i < QT * FT_S; i += blockDim.x) t.region[i] = KEY_MAX;
    if (tid < QT) {
        t.nb[tid] = 0;
        t.nt[tid] = 0;
        t.tau[tid] = KEY_MAX;
        const int qg = qt0 + tid;
        s_prog[tid] = qg < a.nq ? a.qprog[qg] : -1;
    }
    // the query tile, zero past dpad and past the batch
    for (int i = tid; i < QT * (DP / 4); i += blockDim.x) {
        const int qq = i / (DP / 4), c4 = i - qq * (DP / 4);
        const int qg = qt0 + qq;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (qg < a.nq && c4 * 4 < dpad)
            v = __ldg((const float4 *)(a.queries + (size_t)qg * dpad + c4 * 4));
        *(float4 *)(sQ + qq * QS + c4 * 4) = v;
    }

    const uint64_t r0 = (uint64_t)rblk * a.rows_per_cta;
    uint64_t r1 = r0 + a.rows_per_cta;
    if (r1 > a.nrows) r1 = a.nrows;
    const int ntile = r1 > r0 ? (int)((r1 - r0 + FT_RT - 1) / FT_RT) : 0;
    const int total = ntile * NCH;

    // the filter words of tile tt (4 words of 32 rows per query)
    auto load_words = [&](int tt) {
        if (tid < QT * 4) {
            const int qq = tid >> 2, w = tid & 3;
            const int pg = s_prog[qq];
            const uint64_t word = ((r0 + (uint64_t)tt * FT_RT) >> 5) + w;
            uint32_t v = 0xFFFFFFFFu;
            if (pg >= 0) v = word < a.bm_words ? __ldg(a.bitmaps + (uint64_t)pg * a.bm_words + word) : 0u;
            s_bw[tid] = v;
        }
    };
    // chunk s = (tile s / NCH, dims (s % NCH) * 32 ..): 128 rows x 32 dims,
    // four 16-byte copies per thread; rows past the range and dims past
    // dpad are zero-filled
    auto issue = [&](int s) {
        const int tt = s / NCH, c = s - tt * NCH;
        float *dst = sX + (s % FT_NSTG) * (FT_RT * FT_XS);
        const uint64_t rb = r0 + (uint64_t)tt * FT_RT;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int f = tid + 256 * u;
            const int row = f >> 3, c4 = f & 7;
            const int dim = c * FT_CH + c4 * 4;
            const uint64_t gr = rb + row;
            const bool ok = gr < r1 && dim < dpad;
            const float *src = ok ? a.vecs + gr * (uint64_t)dpad + dim : a.vecs;
            cp_async16(dst + row * FT_XS + c4 * 4, src, ok ? 16 : 0);
        }
        cp_async_commit();
    };

    __syncthreads();  // s_prog, queries
    load_words(0);
#pragma unroll
    for (int s = 0; s < FT_NSTG - 1; s++) {
        if (s < total) issue(s);
        else cp_async_commit();
    }

    uint64_t acc[FT_RPT][QJ];
    for (int s = 0; s < total; s++) {
        cp_async_wait<FT_NSTG - 2>();
        __syncthreads();  // chunk s visible; chunk s - 1's stage free
        if (s + FT_NSTG - 1 < total) issue(s + FT_NSTG - 1);
        else cp_async_commit();
        const int tt = s / NCH, c = s - tt * NCH;
        if (c == 0) {
#pragma unroll
            for (int i = 0; i < FT_RPT; i++)
#pragma unroll
                for (int j = 0; j < QJ; j++) acc[i][j] = 0ull;
        }
        const float *xs = sX + (s % FT_NSTG) * (FT_RT * FT_XS) + tr * FT_XS;
        const float *qs = sQ + tq * QS + c * FT_CH;
#pragma unroll
        for (int kk = 0; kk < FT_CH; kk += 4) {
            uint64_t qa[QJ], qb[QJ];
#pragma unroll
            for (int j = 0; j < QJ; j++) {
                const float4 q = *(const float4 *)(qs + j * 16 * QS + kk);
                qa[j] = f2_pack(q.x, q.y);
                qb[j] = f2_pack(q.z, q.w);
            }
#pragma unroll
            for (int i = 0; i < FT_RPT; i++) {
                const float4 x = *(const float4 *)(xs + i * 16 * FT_XS + kk);
                const uint64_t xa = f2_pack(x.x, x.y), xb = f2_pack(x.z, x.w);
#pragma unroll
                for (int j = 0; j < QJ; j++) {
                    f2_sqdiff_acc(acc[i][j], xa, qa[j]);
                    f2_sqdiff_acc(acc[i][j], xb, qb[j]);
                }
            }
        }
        if (c != NCH - 1) continue;
        // ---- tile tt complete: candidates
        const uint64_t rb = r0 + (uint64_t)tt * FT_RT;
#pragma unroll
        for (int i = 0; i < FT_RPT; i++) {
            const int lr = tr + 16 * i;
            const uint64_t row = rb + lr;
#pragma unroll
            for (int j = 0; j < QJ; j++) {
                const int qq = tq + 16 * j;
                if (row >= r1 || qt0 + qq >= a.nq) continue;
                if (!((s_bw[qq * 4 + (lr >> 5)] >> (lr & 31)) & 1u)) continue;
                const uint64_t key = make_key(f2_sum(acc[i][j]), (uint32_t)row);
                if (key < t.tau[qq]) {
                    const int pos = atomicAdd(&t.nb[qq], 1);
                    t.region[(size_t)qq * FT_S + K + pos] = key;
                }
            }
        }
        __syncthreads();
        const bool last = tt == ntile - 1;
        if (tid == 0) {
            // flush when the next tile could overflow a buffer, at the end,
            // or as soon as a query without a full list has K keys
            int n = 0;
            for (int qq = 0; qq < QT; qq++)
                if (t.nb[qq] > 0 && (last || t.nb[qq] > FT_CB - FT_RT ||
                                     (t.nt[qq] < K && t.nb[qq] >= K)))
                    t.flush_list[1 + n++] = qq;
            t.flush_list[0] = n;
        }
        // bounds published by other CTAs
        if (tid < QT && qt0 + tid < a.nq) {
            const unsigned long long g = *((volatile unsigned long long *)(a.tau + qt0 + tid));
            if (g < t.tau[tid]) t.tau[tid] = g;
        }
        __syncthreads();
        topk_flush(t, FT_S, K, FT_CB, qt0, a.nq, a.tau);
        if (!last) load_words(tt + 1);  // read after the next tile's barriers
    }
    cp_async_wait<0>();
    __syncthreads();

    // per-CTA results
    for (int qq = 0; qq < QT; qq++) {
        const int qg = qt0 + qq;
        if (qg >= a.nq) break;
        uint64_t *dst = a.part + ((uint64_t)qg * a.grow + rblk) * K;
        const int n = t.nt[qq];
        for (int i = tid; i < n; i += blockDim.x) dst[i] = t.region[(size_t)qq * FT_S + i];
        if (tid == 0) a.part_cnt[(uint64_t)qg * a.grow + rblk] = (uint32_t)n;
    }
}

// Plan for the register-blocked scan: query tiles of 64 (dpad <= 128) or
// 32 (dpad <= 256) for batches of at least 24 queries and K <= 64; false
// when the batch belongs to the small-tile kernel.
bool plan_scan_f32t(uint64_t nrows, int dpad, int nq, int K, int sm_count, ScanPlan &pl) {
    if (nq < 24 || K > 64 || dpad > 256) return false;
    const int dp = (dpad + 31) & ~31;
    pl.QT = (dp <= 128 && nq > 32) ? 64 : 32;
    pl.DCH = dp;  // the padded row length (a template argument)
    pl.CB = FT_CB;
    pl.S = FT_S;
    pl.smem = scan_f32t_smem(pl.QT, dp <= 128 ? 128 : 256);
    pl.qtiles = (nq + pl.QT - 1) / pl.QT;
    int grow = sm_count / pl.qtiles;
    if (grow < 1) grow = 1;
    // at least 8 tiles per CTA: a CTA's set-up (query tile, first bound)
    // amortizes over its rows
    const uint64_t max_grow = (nrows + 8 * FT_RT - 1) / (8 * FT_RT);
    if ((uint64_t)grow > max_grow) grow = (int)(max_grow ? max_grow : 1);
    uint64_t rpc = (nrows + grow - 1) / grow;
    rpc = (rpc + 31) & ~31ull;  // whole filter words per CTA
    pl.rows_per_cta = rpc;
    pl.grow = (int)((nrows + rpc - 1) / rpc);
    if (pl.grow < 1) pl.grow = 1;
    pl.M = 4096;
    pl.merge_smem = (size_t)pl.M * 8 + (size_t)pl.grow * 8;
    return true;
}

template <int QT, int DP>
static cudaError_t launch_t(const ScanF32Args &a, const ScanPlan &pl, cudaStream_t st) {
    auto kern = scan_f32t_kernel<QT, DP>;
    cudaError_t e = raise_smem_limit((const void *)kern, pl.smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)(pl.grow * pl.qtiles), 256, pl.smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_scan_f32t(const ScanF32Args &a, const ScanPlan &pl, cudaStream_t st) {
    const int dp = pl.DCH <= 128 ? 128 : 256;
    if (pl.QT == 64 && dp == 128) return launch_t<64, 128>(a, pl, st);
    if (pl.QT == 32 && dp == 128) return launch_t<32, 128>(a, pl, st);
    if (pl.QT == 32 && dp == 256) return launch_t<32, 256>(a, pl, st);
    return cudaErrorInvalidValue;
}

}  // namespace pv
