// scan_f32.cu — exact FP32 filtered L2 scan with fused top-K selection.
//
// Replaces the reference's tiled scan + merge pair (fv_brute_tile_kernel,
// gpu_engine.cu:474-610, and fv_brute_merge_kernel, :1003-1065) and its
// legacy per-query kernel (:348-418). Design:
//  * rows stream from HBM once per query tile with coalesced 16-byte loads:
//    lane L of a warp owns dims [4L, 4L+4) of every 128-dim chunk, so one
//    warp-wide load instruction fetches one 512-byte row;
//  * the query tile (QT queries) lives in registers for the whole kernel;
//  * distances are (x - q)^2 summed in FP32 (difference form, like the CPU
//    cursor's l2sq, engine.cpp:43-90), reduced across lanes by a
//    transposing butterfly: R = 32/QT rows x QT queries = 32 partial sums
//    per lane collapse in 31 shuffles so lane L ends with pair L;
//  * the predicate is one bit of a per-batch bitmap, read only for
//    candidates that already beat the threshold;
//  * survivors go to per-query shared-memory buffers (topk.cuh), and a
//    grid-wide per-query bound in global memory lets CTAs prune with each
//    other's K-th key;
//  * a merge kernel reduces the per-CTA lists of a query to its final
//    ascending top-K and writes FvHit records directly.
#include "common.cuh"
#include "pv_internal.h"
#include "topk.cuh"

namespace pv {


template <int QT>
struct ScanShape {
    static constexpr int R = 32 / QT;           // rows per warp iteration
    // rows per step (between block barriers); long steps for the small,
    // bandwidth-bound tiles keep more loads in flight per warp
    static constexpr int RPS = (QT >= 8) ? 128 : (QT >= 4 ? 256 : 1024);
    static constexpr int U = RPS / (8 * R);     // iterations per warp per step
    static constexpr int CB = 2 * RPS;
};

// Transposing butterfly: 32 partial sums per lane -> lane L holds total L.
__device__ __forceinline__ float butterfly32(float (&p)[32], int lane) {
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = (lane & s) != 0;
#pragma unroll
        for (int j = 0; j < s; j++) {
            const float send = upper ? p[j] : p[j + s];
            const float keep = upper ? p[j + s] : p[j];
            p[j] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    return p[0];
}

template <int QT, int DCH>
__global__ void __launch_bounds__(256, 2) scan_f32_kernel(ScanF32Args a) {
    using SH = ScanShape<QT>;
    constexpr int R = SH::R;
    constexpr int U = SH::U;
    constexpr int RPS = SH::RPS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int S = a.S, K = a.K, CB = a.CB;
    TopkSmem t;
    t.region = (uint64_t *)smem_raw;
    t.tau = (unsigned long long *)(t.region + (size_t)QT * S);
    t.nb = (int *)(t.tau + QT);
    t.nt = t.nb + QT;
    t.flush_list = t.nt + QT;
    int *s_prog = t.flush_list + QT + 1;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int qtile = blockIdx.x % a.qtiles;
    const int rblk = blockIdx.x / a.qtiles;
    const int qt0 = qtile * QT;

    for (int i = tid; i < QT * S; i += blockDim.x) t.region[i] = KEY_MAX;
    if (tid < QT) {
        t.nb[tid] = 0;
        t.nt[tid] = 0;
        t.tau[tid] = KEY_MAX;
        const int qg = qt0 + tid;
        s_prog[tid] = qg < a.nq ? a.qprog[qg] : -1;
    }

    // query tile in registers
    float4 qr[QT][DCH];
#pragma unroll
    for (int qq = 0; qq < QT; qq++) {
        const int qg = qt0 + qq;
#pragma unroll
        for (int c = 0; c < DCH; c++) {
            const int j = c * 128 + lane * 4;
            qr[qq][c] = (qg < a.nq && j < a.dpad)
                            ? __ldg((const float4 *)(a.queries + (size_t)qg * a.dpad + j))
                            : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    __syncthreads();

    const uint64_t r0 = (uint64_t)rblk * a.rows_per_cta;
    uint64_t r1 = r0 + a.rows_per_cta;
    if (r1 > a.nrows) r1 = a.nrows;

    // pair owned by this lane after the butterfly
    const int my_r = lane / QT;
    const int my_q = lane % QT;
    const int my_qg = qt0 + my_q;

    // The first step is one warp iteration (8 * R rows) so every query's
    // threshold exists early; later steps are RPS rows.
    int us = 1;
    for (uint64_t sb = r0; sb < r1; sb += (uint64_t)8 * R * us, us = U) {
#pragma unroll 1
        for (int u = 0; u < us; u++) {
            const uint64_t rb = sb + (uint64_t)(warp * us + u) * R;
            if (rb >= r1) break;
            // predicate word of this lane's (row, query) pair, fetched with
            // the rows so the filter never waits on a dependent load (the R
            // rows of an iteration lie in one 32-row word)
            const int my_pg = s_prog[my_q];
            const uint32_t pword =
                my_pg >= 0 ? __ldg(a.bitmaps + (uint64_t)my_pg * a.bm_words + (rb >> 5))
                           : 0xFFFFFFFFu;
            float p[32];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const uint64_t row = rb + r;
                const bool ok = row < r1;
                float4 x[DCH];
#pragma unroll
                for (int c = 0; c < DCH; c++) {
                    const int j = c * 128 + lane * 4;
                    x[c] = (ok && j < a.dpad)
                               ? __ldg((const float4 *)(a.vecs + row * (uint64_t)a.dpad + j))
                               : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int qq = 0; qq < QT; qq++) {
                    float s = 0.f;
#pragma unroll
                    for (int c = 0; c < DCH; c++) {
                        float d0 = x[c].x - qr[qq][c].x;
                        float d1 = x[c].y - qr[qq][c].y;
                        float d2 = x[c].z - qr[qq][c].z;
                        float d3 = x[c].w - qr[qq][c].w;
                        s = fmaf(d0, d0, s);
                        s = fmaf(d1, d1, s);
                        s = fmaf(d2, d2, s);
                        s = fmaf(d3, d3, s);
                    }
                    p[r * QT + qq] = s;
                }
            }
            const float dist = butterfly32(p, lane);
            const uint64_t row = rb + my_r;
            if (row < r1 && my_qg < a.nq && ((pword >> (row & 31)) & 1u)) {
                const uint64_t key = make_key(dist, (uint32_t)row);
                if (key < t.tau[my_q]) {
                    const int pos = atomicAdd(&t.nb[my_q], 1);
                    t.region[(size_t)my_q * S + K + pos] = key;
                }
            }
        }
        __syncthreads();
        const bool last = sb + (uint64_t)8 * R * us >= r1;
        if (tid == 0) {
            // flush when the next step could overflow the buffer, at the
            // end, or as soon as a query without a full list has K keys
            // (that sets its threshold)
            int n = 0;
            for (int qq = 0; qq < QT; qq++)
                if (t.nb[qq] > 0 && (last || t.nb[qq] > CB - RPS ||
                                     (t.nt[qq] < K && t.nb[qq] >= K)))
                    t.flush_list[1 + n++] = qq;
            t.flush_list[0] = n;
        }
        // pick up bounds published by other CTAs
        if (tid < QT && qt0 + tid < a.nq) {
            const unsigned long long g = *((volatile unsigned long long *)(a.tau + qt0 + tid));
            if (g < t.tau[tid]) t.tau[tid] = g;
        }
        __syncthreads();
        topk_flush(t, S, K, CB, qt0, a.nq, a.tau);
    }
    __syncthreads();

    // per-CTA results
    for (int qq = 0; qq < QT; qq++) {
        const int qg = qt0 + qq;
        if (qg >= a.nq) break;
        uint64_t *dst = a.part + ((uint64_t)qg * a.grow + rblk) * K;
        const int n = t.nt[qq];
        for (int i = tid; i < n; i += blockDim.x) dst[i] = t.region[(size_t)qq * S + i];
        if (tid == 0) a.part_cnt[(uint64_t)qg * a.grow + rblk] = (uint32_t)n;
    }
}

// Reduces the per-CTA lists of one query to its final top-K (one CTA per
// query). Only keys <= the grid-wide bound can be in the answer; lists are
// ascending so each contributes a prefix. A warp measures a list's prefix
// with one coalesced load + ballot per 32 entries, a warp scan turns the
// lengths into offsets, and the gathered prefixes are sorted with a bitonic
// network sized to their count. Prefixes that exceed the buffer are folded
// into the running top-K in further rounds (rare: the bound keeps the
// union near K).
__global__ void __launch_bounds__(256)
merge_kernel(const uint64_t *__restrict__ part, const uint32_t *__restrict__ part_cnt,
             int grow, int K, int M, const unsigned long long *__restrict__ tau,
             const int32_t *__restrict__ qprog,
             const unsigned long long *__restrict__ popcnt, uint64_t nrows,
             FvHit *__restrict__ out, uint32_t *__restrict__ out_cnt,
             uint8_t *__restrict__ trunc, unsigned long long *__restrict__ tau_out,
             int KO, uint8_t *__restrict__ unc, int KU) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *buf = (uint64_t *)smem_raw;   // [M]
    int *s_c = (int *)(buf + M);            // [grow] prefix lengths
    int *s_off = s_c + grow;                // [grow] offsets within a round
    __shared__ int s_gend, s_n;
    const int q = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nwarps = blockDim.x >> 5;
    const unsigned long long bound = tau[q];
    const uint64_t *lists = part + (uint64_t)q * grow * K;
    const uint32_t *cnts = part_cnt + (uint64_t)q * grow;

    // fast path: one coalesced pass over all list slots; survivors (slot
    // inside its list's count and key <= bound) are appended in any order,
    // then sorted. Taken whenever they fit the buffer (the usual case).
    for (int g = tid; g < grow; g += blockDim.x) {
        const uint32_t c = cnts[g];
        s_c[g] = c > (uint32_t)KU ? KU : (int)c;
    }
    if (tid == 0) s_n = 0;
    __syncthreads();
    {
        const uint64_t total = (uint64_t)grow * K;
        for (uint64_t i = tid; i < total; i += blockDim.x) {
            const int g = (int)(i / K), j = (int)(i - (uint64_t)g * K);
            if (j >= s_c[g]) continue;
            const uint64_t key = lists[i];
            if (key > bound) continue;
            const int pos = atomicAdd(&s_n, 1);
            if (pos < M) buf[pos] = key;
        }
    }
    __syncthreads();
    const int nfast = s_n;
    if (nfast <= M) {
        int n2 = 1;
        while (n2 < nfast) n2 <<= 1;
        for (int i = nfast + tid; i < n2; i += blockDim.x) buf[i] = KEY_MAX;
        __syncthreads();
        for (int k = 2; k <= n2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < (n2 >> 1); i += blockDim.x) {
                    const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                    const int hi = lo | j;
                    const uint64_t x = buf[lo], y = buf[hi];
                    if ((x > y) == ((lo & k) == 0)) {
                        buf[lo] = y;
                        buf[hi] = x;
                    }
                }
                __syncthreads();
            }
        }
        const int nt = nfast < KO ? nfast : KO;
        for (int i = nt + tid; i < KO; i += blockDim.x) buf[i] = KEY_MAX;
        __syncthreads();
    } else {
    // general path: measure each list's prefix, then fold in rounds
    for (int g = warp; g < grow; g += nwarps) {
        int c = (int)cnts[g];
        if (c > KU) c = KU;
        const uint64_t *L = lists + (uint64_t)g * K;
        int n = 0;
        for (int j0 = 0; j0 < c; j0 += 32) {
            const int j = j0 + lane;
            const uint64_t key = j < c ? L[j] : KEY_MAX;
            const uint32_t m = __ballot_sync(0xffffffffu, j < c && key <= bound);
            n += __popc(m);
            if (m != 0xffffffffu) break;
        }
        if (lane == 0) s_c[g] = n;
    }
    __syncthreads();

    int nt = 0;  // valid keys in buf[0, K) carried between rounds
    int g = 0;
    while (g < grow) {
        const int cap = M - nt;
        if (warp == 0) {
            // lists g.. in order while their prefixes fit (at least one list)
            int base = 0, ge = g;
            while (ge < grow) {
                const int i = ge + lane;
                const int c = i < grow ? s_c[i] : 0;
                int incl = c;
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const int excl = base + incl - c;
                const bool fits = i < grow && (excl + c <= cap || i == g);
                const uint32_t fm = __ballot_sync(0xffffffffu, fits);
                const int nfit = __ffs(~fm) ? __ffs(~fm) - 1 : 32;  // leading run
                if (lane < nfit) s_off[i] = nt + excl;
                base += __shfl_sync(0xffffffffu, incl, nfit > 0 ? nfit - 1 : 0) * (nfit > 0);
                ge += nfit;
                if (nfit < 32) break;
            }
            if (lane == 0) {
                s_gend = ge;
                s_n = nt + base;
            }
        }
        __syncthreads();
        const int gend = s_gend, n = s_n;
        for (int gg = g + warp; gg < gend; gg += nwarps) {
            const uint64_t *L = lists + (uint64_t)gg * K;
            const int c = s_c[gg], off = s_off[gg];
            for (int i = lane; i < c; i += 32) buf[off + i] = L[i];
        }
        int n2 = 1;
        while (n2 < n) n2 <<= 1;
        for (int i = n + tid; i < n2; i += blockDim.x) buf[i] = KEY_MAX;
        __syncthreads();
        for (int k = 2; k <= n2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < (n2 >> 1); i += blockDim.x) {
                    const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                    const int hi = lo | j;
                    const uint64_t x = buf[lo], y = buf[hi];
                    const bool up = (lo & k) == 0;
                    if ((x > y) == up) {
                        buf[lo] = y;
                        buf[hi] = x;
                    }
                }
                __syncthreads();
            }
        }
        __syncthreads();
        nt = n < KO ? n : KO;
        g = gend;
    }
    for (int i = nt + tid; i < KO; i += blockDim.x) buf[i] = KEY_MAX;
    __syncthreads();
    }  // general path
    for (int i = tid; i < KO; i += blockDim.x) {
        const uint64_t k = buf[i];
        if (k != KEY_MAX) {
            FvHit h;
            h.node = (uint64_t)key_row(k);
            h.dist = key_dist(k);
            out[(uint64_t)q * KO + i] = h;
        }
    }
    __shared__ int s_lo, s_unc;
    if (tid == 0) {
        int lo = 0, hi = KO;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (buf[mid] != KEY_MAX) lo = mid + 1; else hi = mid;
        }
        s_lo = lo;
        s_unc = 0;
        out_cnt[q] = (uint32_t)lo;
        const int pg = qprog[q];
        const unsigned long long passing = pg >= 0 ? popcnt[pg] : nrows;
        trunc[q] = passing > (unsigned long long)KO ? 1 : 0;
        // the KO-th merged key bounds the KO-th key of any superset of rows
        if (tau_out && lo == KO) tau_out[q] = buf[KO - 1];
    }
    if (unc) {
        // Lists shorter than the output: a full list whose last key is at
        // or below the output's last key (or below the bound while the
        // output is short) may have dropped a member of it.
        __syncthreads();
        const uint64_t lim = s_lo == KO ? buf[KO - 1] : bound;
        for (int g = tid; g < grow; g += blockDim.x)
            if (cnts[g] >= (uint32_t)K && lists[(uint64_t)g * K + K - 1] <= lim) s_unc = 1;
        __syncthreads();
        if (tid == 0) unc[q] = (uint8_t)s_unc;
    }
}

static inline int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

static int pick_dch(int dpad) {
    if (dpad <= 128) return 1;
    if (dpad <= 256) return 2;
    if (dpad <= 512) return 4;
    return 0;
}

int scan_f32_max_qt(int dim) {
    int dch = pick_dch((dim + 3) & ~3);
    if (dch == 0) return 0;
    return 16 / dch;
}

template <int QT>
static int cb_for() { return ScanShape<QT>::CB; }

static int cb_of(int qt) {
    switch (qt) {
        case 1: return cb_for<1>();
        case 2: return cb_for<2>();
        case 4: return cb_for<4>();
        case 8: return cb_for<8>();
        default: return cb_for<16>();
    }
}

bool plan_scan_f32(uint64_t nrows, int dpad, int nq, int K, int sm_count, ScanPlan &pl,
                   uint64_t min_rows) {
    pl.DCH = pick_dch(dpad);
    if (pl.DCH == 0) return false;
    int qt_cap = 16 / pl.DCH;
    int qt = 1;
    while (qt < qt_cap && qt < nq) qt <<= 1;
    // shared memory budget: QT regions of S keys
    for (;;) {
        int cb = cb_of(qt);
        int S = next_pow2(K + cb);
        size_t smem = (size_t)qt * S * 8 + qt * 8 + (3 * qt + 1) * 4 + qt * 4 + 16;
        if (smem <= 110 * 1024 || qt == 1) {
            pl.QT = qt;
            pl.CB = cb;
            pl.S = S;
            pl.smem = smem;
            break;
        }
        qt >>= 1;
    }
    pl.qtiles = (nq + pl.QT - 1) / pl.QT;
    // two resident CTAs per SM when the regions allow it
    int per_sm = pl.smem <= 100 * 1024 ? 2 : 1;
    int target = sm_count * per_sm;
    int grow = target / pl.qtiles;
    if (grow < 1) grow = 1;
    // rows per CTA at least min_rows (long streams amortize the flushes)
    uint64_t max_grow = (nrows + min_rows - 1) / min_rows;
    if (max_grow < 1) max_grow = 1;
    if ((uint64_t)grow > max_grow) grow = (int)max_grow;
    uint64_t rpc = (nrows + grow - 1) / grow;
    rpc = (rpc + 31) & ~31ull;
    if (rpc == 0) rpc = 32;
    pl.rows_per_cta = rpc;
    pl.grow = (int)((nrows + rpc - 1) / rpc);
    if (pl.grow < 1) pl.grow = 1;
    pl.M = next_pow2(2 * K) < 4096 ? 4096 : next_pow2(2 * K);
    pl.merge_smem = (size_t)pl.M * 8 + (size_t)pl.grow * 8;
    return true;
}

template <int QT, int DCH>
static cudaError_t launch_qt(const ScanF32Args &a, const ScanPlan &pl, cudaStream_t st) {
    auto kern = scan_f32_kernel<QT, DCH>;
    cudaError_t e = raise_smem_limit((const void *)kern, pl.smem);
    if (e != cudaSuccess) return e;
    unsigned grid = (unsigned)(pl.grow * pl.qtiles);
    kern<<<grid, 256, pl.smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_scan_f32(const ScanF32Args &a, const ScanPlan &pl, cudaStream_t st) {
#define PV_CASE(Q, D) \
    if (pl.QT == Q && pl.DCH == D) return launch_qt<Q, D>(a, pl, st);
    PV_CASE(1, 1) PV_CASE(2, 1) PV_CASE(4, 1) PV_CASE(8, 1) PV_CASE(16, 1)
    PV_CASE(1, 2) PV_CASE(2, 2) PV_CASE(4, 2) PV_CASE(8, 2)
    PV_CASE(1, 4) PV_CASE(2, 4) PV_CASE(4, 4)
#undef PV_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_merge(const uint64_t *part, const uint32_t *part_cnt, int grow, int K,
                         const ScanPlan &pl, const unsigned long long *tau,
                         const int32_t *qprog, const unsigned long long *popcnt,
                         uint64_t nrows, int nq, FvHit *out, uint32_t *out_cnt,
                         uint8_t *trunc, cudaStream_t st, unsigned long long *tau_out,
                         int kout, uint8_t *unc, int kuse) {
    if (kout <= 0) kout = K;
    if (kuse <= 0 || kuse > K) kuse = K;
    if (kout > pl.M) return cudaErrorInvalidValue;
    cudaError_t e = raise_smem_limit((const void *)merge_kernel, pl.merge_smem);
    if (e != cudaSuccess) return e;
    merge_kernel<<<nq, 256, pl.merge_smem, st>>>(part, part_cnt, grow, K, pl.M, tau, qprog,
                                                 popcnt, nrows, out, out_cnt, trunc, tau_out,
                                                 kout, unc, kuse);
    return cudaGetLastError();
}

}  // namespace pv
