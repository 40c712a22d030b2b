// sparse.cu — selective filters scan only their matching rows.
//
// The reference answers a selective filter through its posting-list
// driver: the spans of the sorted attribute values that can match bound
// the candidate rows (engine.cpp:464-599, fv_pred_estimate :640-643), and
// its GPU router sends a query to the span path when that total is small
// (gpu_engine.cu:2249-2260). Here the same bound decides the route:
//  * at upload each attribute column's values are kept sorted on the host
//    (from the posting rows), so a comparison or IN list is counted exactly
//    by binary search, and AND / OR / NOT combine lower / upper bounds;
//  * a batch whose queries share one filter bounded by a small count
//    compacts that filter's bitmap into a row-id list on the device and
//    either gathers those rows into a contiguous set for the tensor-core
//    scan (2048+ rows, when the batch's mode scans on the tensor cores),
//    or computes the exact FP32 distance of every (query, listed row) and
//    selects each query's top-k from those keys (a radix select).
// Results equal the full scan's: same rows, same FP32 distances.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pv_internal.h"

namespace pv {

void build_sorted_cols(FvGpuIndex *g, const double *cols, const uint32_t *post_rows) {
    g->sorted_cols.assign(g->ncols, {});
    for (int c = 0; c < g->ncols; c++) {
        std::vector<double> &v = g->sorted_cols[c];
        v.reserve(g->count);
        const double *col = cols + (uint64_t)c * g->count;
        const uint32_t *pr = post_rows + (uint64_t)c * g->count;
        for (uint64_t i = 0; i < g->count; i++) {
            const double x = col[pr[i] < g->count ? pr[i] : 0];
            if (x == x) v.push_back(x);  // NaN sorts last and matches nothing
        }
        // posting rows are ordered by value; keep the copy sorted regardless
        if (!std::is_sorted(v.begin(), v.end())) std::sort(v.begin(), v.end());
    }
}

namespace {

uint64_t count_cmp(const std::vector<double> &v, int op, double c) {
    const uint64_t n = v.size();
    if (c != c) return op == FV_CMP_NE ? n : 0;  // NaN constant
    const uint64_t lo = std::lower_bound(v.begin(), v.end(), c) - v.begin();
    const uint64_t hi = std::upper_bound(v.begin(), v.end(), c) - v.begin();
    switch (op) {
        case FV_CMP_LT: return lo;
        case FV_CMP_LE: return hi;
        case FV_CMP_EQ: return hi - lo;
        case FV_CMP_GE: return n - lo;
        case FV_CMP_GT: return n - hi;
        case FV_CMP_NE: return n - (hi - lo);
    }
    return n;
}

}  // namespace

// Estimated fraction of rows a range-form program passes: the product of
// its terms' exact fractions (independent columns); 0 for other programs or
// without sorted columns.
double prog_pass_estimate(const FvGpuIndex *g, const PredInsn *ins, int n, const double *consts) {
    if (n != 1 || ins[0].kind != PV_NODE_RANGE || g->count == 0 ||
        (int)g->sorted_cols.size() != g->ncols)
        return 0.0;
    const double N = (double)g->count;
    double f = 1.0;
    int ci = ins[0].val0;
    for (int k = 0; k < ins[0].n; k++) {
        const int meta = (int)consts[ci];
        const int col = meta & 0xFFFF;
        if (col >= g->ncols) return 0.0;
        const std::vector<double> &v = g->sorted_cols[col];
        uint64_t c = 0;
        if (meta & PV_TERM_MASK) {
            uint64_t bits;
            memcpy(&bits, &consts[ci + 1], 8);
            for (int b = 0; b < 64; b++)
                if ((bits >> b) & 1ull) c += count_cmp(v, FV_CMP_EQ, (double)b);
            ci += 2;
        } else {
            const double lo = consts[ci + 1], hi = consts[ci + 2];
            if (lo == lo && hi == hi) {
                const uint64_t a = std::lower_bound(v.begin(), v.end(), lo) - v.begin();
                const uint64_t b = std::upper_bound(v.begin(), v.end(), hi) - v.begin();
                c = b > a ? b - a : 0;
            }
            ci += 3;
        }
        f *= (double)c / N;
    }
    return f;
}

uint64_t prog_upper_bound(const FvGpuIndex *g, const PredInsn *ins, int n, const double *consts) {
    const uint64_t N = g->count;
    if ((int)g->sorted_cols.size() != g->ncols || g->ncols == 0) return N;
    struct B { uint64_t lo, hi; };
    std::vector<B> st;
    st.reserve(n);
    for (int i = 0; i < n; i++) {
        const PredInsn &in = ins[i];
        switch (in.kind) {
            case FV_NODE_CMP: {
                if (in.col < 0 || in.col >= g->ncols) return N;
                const uint64_t c = count_cmp(g->sorted_cols[in.col], in.op, in.value);
                st.push_back({c, c});
                break;
            }
            case FV_NODE_IN: {
                if (in.col < 0 || in.col >= g->ncols) return N;
                std::vector<double> vals(consts + in.val0, consts + in.val0 + in.n);
                std::sort(vals.begin(), vals.end());
                vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
                uint64_t c = 0;
                for (double x : vals) c += count_cmp(g->sorted_cols[in.col], FV_CMP_EQ, x);
                st.push_back({c, c});
                break;
            }
            case PV_NODE_RANGE: {
                // AND of exact per-term counts: at most the smallest, at
                // least what the terms' counts force to overlap
                uint64_t hi = N, lo_sum = 0;
                int ci = in.val0;
                for (int k = 0; k < in.n; k++) {
                    const int meta = (int)consts[ci];
                    const int col = meta & 0xFFFF;
                    if (col >= g->ncols) return N;
                    const std::vector<double> &v = g->sorted_cols[col];
                    uint64_t c = 0;
                    if (meta & PV_TERM_MASK) {
                        uint64_t bits;
                        memcpy(&bits, &consts[ci + 1], 8);
                        for (int b = 0; b < 64; b++)
                            if ((bits >> b) & 1ull) c += count_cmp(v, FV_CMP_EQ, (double)b);
                        ci += 2;
                    } else {
                        const double lo = consts[ci + 1], hi_v = consts[ci + 2];
                        if (lo == lo && hi_v == hi_v) {  // closed [lo, hi]
                            const uint64_t a = std::lower_bound(v.begin(), v.end(), lo) - v.begin();
                            const uint64_t b = std::upper_bound(v.begin(), v.end(), hi_v) - v.begin();
                            c = b > a ? b - a : 0;
                        }
                        ci += 3;
                    }
                    hi = std::min(hi, c);
                    lo_sum += c;
                }
                const uint64_t over = in.n > 1 ? (uint64_t)(in.n - 1) * N : 0;
                st.push_back({lo_sum > over ? lo_sum - over : 0, hi});
                break;
            }
            case FV_NODE_AND:
            case FV_NODE_OR: {
                if (in.n == 0) {
                    st.push_back(in.kind == FV_NODE_AND ? B{N, N} : B{0, 0});
                    break;
                }
                if (st.size() < 2) return N;
                const B b = st.back();
                st.pop_back();
                const B a = st.back();
                st.pop_back();
                if (in.kind == FV_NODE_AND)
                    st.push_back({a.lo + b.lo > N ? a.lo + b.lo - N : 0, std::min(a.hi, b.hi)});
                else
                    st.push_back({std::max(a.lo, b.lo), std::min(N, a.hi + b.hi)});
                break;
            }
            default: {  // NOT
                if (st.empty()) return N;
                const B a = st.back();
                st.back() = {N - a.hi, N - a.lo};
                break;
            }
        }
    }
    return st.size() == 1 ? st.back().hi : N;
}

// Bitmap -> ascending row ids within each block of words; blocks claim
// their output range with one atomic (the list's order across blocks does
// not matter: keys carry the row id).
__global__ void __launch_bounds__(256) compact_kernel(const uint32_t *__restrict__ bm,
                                                      uint64_t bm_words, uint64_t nrows,
                                                      uint32_t *__restrict__ ids,
                                                      unsigned long long *__restrict__ count,
                                                      uint64_t cap) {
    __shared__ int s_warp[8];
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint64_t w0 = (uint64_t)blockIdx.x * blockDim.x; w0 < bm_words;
         w0 += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t w = w0 + tid;
        uint32_t word = w < bm_words ? bm[w] : 0u;
        if (w == bm_words - 1 && (nrows & 31)) word &= (1u << (nrows & 31)) - 1u;
        const int c = __popc(word);
        int incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        int before = 0, total = 0;
        for (int i = 0; i < 8; i++) {
            if (i < warp) before += s_warp[i];
            total += s_warp[i];
        }
        if (tid == 0) s_base = atomicAdd(count, (unsigned long long)total);
        __syncthreads();
        uint64_t pos = s_base + before + incl - c;
        while (word) {
            const int b = __ffs(word) - 1;
            word &= word - 1;
            if (pos < cap) ids[pos] = (uint32_t)(w * 32 + b);
            pos++;
        }
        __syncthreads();
    }
}

// Exact FP32 distances of every listed row to every query of the batch:
// keys[q][i] = (||x_rowids[i] - q||^2, rowids[i]) for i < n = min(*count,
// cap), and dcnt[q] = n. grid (row blocks, query tiles of GD_QT); a warp
// takes one row at a time: lane L holds dims [4L, 4L+4) of each 128-dim
// chunk, the GD_QT partial sums are reduced with xor-shuffles.
constexpr int GD_QT = 8;

__global__ void __launch_bounds__(256)
gather_dist_kernel(const float *__restrict__ vecs, int dpad, const float *__restrict__ queries,
                   int nq, const uint32_t *__restrict__ rowids,
                   const unsigned long long *__restrict__ count, uint64_t cap,
                   uint64_t *__restrict__ keys, uint32_t *__restrict__ dcnt) {
    extern __shared__ __align__(16) float gd_q[];  // [GD_QT][dpad]
    const int q0 = blockIdx.y * GD_QT;
    const uint64_t n = min((unsigned long long)cap, *count);
    for (int i = threadIdx.x; i < GD_QT * dpad; i += blockDim.x) {
        const int j = i / dpad, d = i - j * dpad;
        gd_q[i] = q0 + j < nq ? queries[(size_t)(q0 + j) * dpad + d] : 0.f;
    }
    if (blockIdx.x == 0 && threadIdx.x < GD_QT && q0 + (int)threadIdx.x < nq)
        dcnt[q0 + threadIdx.x] = (uint32_t)n;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t r = (uint64_t)blockIdx.x * 8 + warp; r < n; r += (uint64_t)gridDim.x * 8) {
        const uint32_t row = __ldg(rowids + r);
        const float *x = vecs + (uint64_t)row * dpad;
        float acc[GD_QT];
#pragma unroll
        for (int j = 0; j < GD_QT; j++) acc[j] = 0.f;
        for (int c = lane * 4; c < dpad; c += 128) {
            const float4 v = __ldg((const float4 *)(x + c));
#pragma unroll
            for (int j = 0; j < GD_QT; j++) {
                const float4 w = *(const float4 *)(gd_q + j * dpad + c);
                const float d0 = v.x - w.x, d1 = v.y - w.y, d2 = v.z - w.z, d3 = v.w - w.w;
                acc[j] = fmaf(d0, d0, acc[j]);
                acc[j] = fmaf(d1, d1, acc[j]);
                acc[j] = fmaf(d2, d2, acc[j]);
                acc[j] = fmaf(d3, d3, acc[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < GD_QT; j++)
#pragma unroll
            for (int o = 16; o; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
        float mine = acc[0];
#pragma unroll
        for (int j = 1; j < GD_QT; j++)
            if (lane == j) mine = acc[j];
        if (lane < GD_QT && q0 + lane < nq)
            keys[(uint64_t)(q0 + lane) * cap + r] = make_key(mine, row);
    }
}

// The listed rows in the tensor-core scan's operand layout: compacted row i
// (i < min(*count, cap)) is index row ids[i] — its operand row (row_bytes,
// a multiple of 16), norm and fp8 scale; one warp per row, 16-byte copies.
// valid[w] marks the compacted rows [32w, 32w + 32) that exist.
__global__ void __launch_bounds__(256)
gather_rows_kernel(const unsigned char *__restrict__ src, size_t row_bytes,
                   const float *__restrict__ norms, const float *__restrict__ scales,
                   const uint32_t *__restrict__ ids, const unsigned long long *__restrict__ count,
                   uint64_t cap, unsigned char *__restrict__ dst, float *__restrict__ dnorm,
                   float *__restrict__ dscale, uint32_t *__restrict__ valid, uint64_t vwords) {
    const uint64_t n = min((unsigned long long)cap, *count);
    const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = gt; w < vwords; w += nthreads) {
        const uint64_t r0 = w * 32;
        valid[w] = r0 >= n ? 0u : n - r0 >= 32 ? 0xFFFFFFFFu : (1u << (n - r0)) - 1u;
    }
    const int lane = threadIdx.x & 31;
    const size_t n16 = row_bytes / 16;
    for (uint64_t i = gt >> 5; i < n; i += nthreads >> 5) {
        const uint32_t r = __ldg(ids + i);
        const uint4 *s4 = (const uint4 *)(src + (size_t)r * row_bytes);
        uint4 *d4 = (uint4 *)(dst + (size_t)i * row_bytes);
        for (size_t j = lane; j < n16; j += 32) d4[j] = __ldg(s4 + j);
        if (lane == 0) {
            dnorm[i] = __ldg(norms + r);
            if (dscale) dscale[i] = __ldg(scales + r);
        }
    }
}

// The sparse route on the tensor cores: the filter's bitmap is compacted to
// a row list, the listed rows are gathered into a contiguous set in the
// scan's operand layout (the upload's BF16 / FP8 rows, or the f32 rows read
// as TF32 for exact-mode batches), and the tensor-core scan runs over that
// set with the same supersets, certificates and re-rank as over the whole
// index; keys carry the index rows, so ties order as in the full scan.
int sparse_tc_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, uint64_t bound, bool tf32,
                     FvHit *d_out, uint32_t *d_cnt, uint8_t *d_trunc, cudaEvent_t *ev,
                     char *errbuf, size_t errlen) {
    const int nq = db.nq;
    char *d = db.stage_d->as<char>();
    const float *d_q = (const float *)(d + db.off_q);
    const int32_t *d_qprog = (const int32_t *)(d + db.off_qprog);
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;
    const bool fp8 = !tf32 && g->precision == FV_GPU_PREC_FP8;
    const size_t row_bytes = tf32 ? (size_t)g->dpad * 4 : (size_t)g->kpad * (fp8 ? 1 : 2);
    const uint64_t cap = std::max<uint64_t>(bound, 1);
    const uint64_t cap_pad = (cap + 127) & ~127ull;  // whole 128-row tiles
    const uint64_t vwords = cap_pad / 32;
    // scratch: [count u64][ids u32 x cap_pad][rows][norms][scales][valid words]
    auto al = [](size_t x, size_t a) { return (x + a - 1) & ~(a - 1); };
    const size_t off_ids = 256;
    const size_t off_rows = al(off_ids + cap_pad * 4, 1024);
    const size_t off_norm = al(off_rows + cap_pad * row_bytes, 1024);
    const size_t off_scale = al(off_norm + cap_pad * 4, 256);
    const size_t off_valid = al(off_scale + (fp8 ? cap_pad * 4 : 0), 256);
    PV_CUDA_OK(s.sparse.ensure(off_valid + vwords * 4 + 256), errbuf, errlen);
    char *sp = s.sparse.as<char>();
    unsigned long long *d_count = (unsigned long long *)sp;
    uint32_t *ids = (uint32_t *)(sp + off_ids);
    unsigned char *rows = (unsigned char *)(sp + off_rows);
    float *norms = (float *)(sp + off_norm);
    float *scales = fp8 ? (float *)(sp + off_scale) : nullptr;
    uint32_t *valid = (uint32_t *)(sp + off_valid);
    PV_CUDA_OK(cudaMemsetAsync(d_count, 0, 8, g->stream), errbuf, errlen);
    unsigned blocks = (unsigned)std::min<uint64_t>((bm_words + 255) / 256, (uint64_t)g->sm_count * 4);
    if (!blocks) blocks = 1;
    compact_kernel<<<blocks, 256, 0, g->stream>>>(s.bitmaps.as<uint32_t>(), bm_words, g->count,
                                                  ids, d_count, cap);
    PV_CUDA_OK(cudaGetLastError(), errbuf, errlen);
    const unsigned gblocks = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((cap + 7) / 8, (uint64_t)g->sm_count * 8));
    const unsigned char *src = tf32 ? (const unsigned char *)g->d_vecs
                                    : (const unsigned char *)g->d_vlow;
    gather_rows_kernel<<<gblocks, 256, 0, g->stream>>>(
        src, row_bytes, tf32 ? g->d_norm32 : g->d_norm, fp8 ? g->d_vscale : nullptr, ids, d_count,
        cap, rows, norms, scales, valid, vwords);
    PV_CUDA_OK(cudaGetLastError(), errbuf, errlen);
    g->launches += 2;  // compaction, gather
    const TcRowSet rs{rows, norms, scales, cap_pad, ids, d_count};
    return launch_scan_tc(g, nq, db.q_amax, d_q, d_qprog, valid, vwords,
                          s.popcnt.as<unsigned long long>(), topb, d_out, d_cnt, d_trunc, ev,
                          errbuf, errlen, nullptr, tf32, &rs);
}

// The sparse route of brute_launch: every query uses program 0, whose
// matches are at most `bound` rows. The bitmap is compacted to a row list,
// every (query, listed row) gets its exact FP32 key, and each query's
// top-topb is selected from its keys (launch_dense_merge).
int sparse_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, uint64_t bound, FvHit *d_out,
                  uint32_t *d_cnt, uint8_t *d_trunc, char *errbuf, size_t errlen) {
    const int nq = db.nq;
    char *d = db.stage_d->as<char>();
    const float *d_q = (const float *)(d + db.off_q);
    const int32_t *d_qprog = (const int32_t *)(d + db.off_qprog);
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;
    const uint64_t cap = std::max<uint64_t>(bound, 1);
    // scratch: [count u64][dcnt u32 x nq][ids u32 x cap][keys u64 x nq x cap]
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t off_dcnt = 256, off_ids = off_dcnt + al((size_t)nq * 4);
    const size_t off_keys = off_ids + al(cap * 4);
    PV_CUDA_OK(s.sparse.ensure(off_keys + (size_t)nq * cap * 8 + 256), errbuf, errlen);
    char *sp = s.sparse.as<char>();
    unsigned long long *d_count = (unsigned long long *)sp;
    uint32_t *dcnt = (uint32_t *)(sp + off_dcnt);
    uint32_t *ids = (uint32_t *)(sp + off_ids);
    uint64_t *keys = (uint64_t *)(sp + off_keys);
    PV_CUDA_OK(cudaMemsetAsync(d_count, 0, 8, g->stream), errbuf, errlen);
    unsigned blocks = (unsigned)std::min<uint64_t>((bm_words + 255) / 256, (uint64_t)g->sm_count * 4);
    if (!blocks) blocks = 1;
    compact_kernel<<<blocks, 256, 0, g->stream>>>(s.bitmaps.as<uint32_t>(), bm_words, g->count,
                                                  ids, d_count, cap);
    PV_CUDA_OK(cudaGetLastError(), errbuf, errlen);
    const int qtiles = (nq + GD_QT - 1) / GD_QT;
    const uint64_t bx = std::max<uint64_t>(
        1, std::min<uint64_t>((cap + 63) / 64, std::max(1, 4 * g->sm_count / qtiles)));
    const size_t smem = (size_t)GD_QT * g->dpad * 4;
    PV_CUDA_OK(raise_smem_limit((const void *)gather_dist_kernel, smem), errbuf, errlen);
    gather_dist_kernel<<<dim3((unsigned)bx, (unsigned)qtiles), 256, smem, g->stream>>>(
        g->d_vecs, g->dpad, d_q, nq, ids, d_count, cap, keys, dcnt);
    PV_CUDA_OK(cudaGetLastError(), errbuf, errlen);
    g->launches += 3;  // compaction, distances, selection
    // the truncation flag counts the filter's true matches
    PV_CUDA_OK(launch_dense_merge(keys, cap, dcnt, false, nullptr, nullptr, (int)topb, d_qprog,
                                  s.popcnt.as<unsigned long long>(), g->count, nq, d_out, d_cnt,
                                  d_trunc, nullptr, nullptr, g->stream),
               errbuf, errlen);
    return 0;
}

}  // namespace pv
