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
//    runs the exact FP32 scan over the listed rows only (the scan kernel
//    gathers rows through the list; keys keep the index's row ids).
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
                        if (lo == lo && hi_v == hi_v) {
                            const uint64_t a = (meta & PV_TERM_LO_OPEN)
                                                   ? std::upper_bound(v.begin(), v.end(), lo) - v.begin()
                                                   : std::lower_bound(v.begin(), v.end(), lo) - v.begin();
                            const uint64_t b = (meta & PV_TERM_HI_OPEN)
                                                   ? std::lower_bound(v.begin(), v.end(), hi_v) - v.begin()
                                                   : std::upper_bound(v.begin(), v.end(), hi_v) - v.begin();
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

// The sparse route of brute_launch: every query uses program 0 and its
// bound is at most `bound` rows. Exact FP32 scan over the compacted rows.
int sparse_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, uint64_t bound, FvHit *d_out,
                  uint32_t *d_cnt, uint8_t *d_trunc, char *errbuf, size_t errlen) {
    const int nq = db.nq;
    char *d = db.stage_d->as<char>();
    const float *d_q = (const float *)(d + db.off_q);
    const int32_t *d_qprog = (const int32_t *)(d + db.off_qprog);
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;
    const uint64_t cap = std::max<uint64_t>(bound, 1);
    ScanPlan pl;
    // few rows: short streams per CTA, so that the grid still fills the GPU
    if (!plan_scan_f32(cap, g->dpad, nq, (int)topb, g->sm_count, pl, 128)) {
        snprintf(errbuf, errlen, "gpu: dimension %d not supported by the scan", g->dim);
        return -1;
    }
    // scratch: [count u64][ids u32 cap][qprog -1 x nq]
    const size_t off_ids = 256, off_neg = off_ids + ((cap * 4 + 255) & ~(size_t)255);
    PV_CUDA_OK(s.sparse.ensure(off_neg + (size_t)nq * 4 + 256), errbuf, errlen);
    char *sp = s.sparse.as<char>();
    unsigned long long *d_count = (unsigned long long *)sp;
    uint32_t *ids = (uint32_t *)(sp + off_ids);
    int32_t *neg = (int32_t *)(sp + off_neg);
    PV_CUDA_OK(cudaMemsetAsync(d_count, 0, 8, g->stream), errbuf, errlen);
    PV_CUDA_OK(cudaMemsetAsync(neg, 0xFF, (size_t)nq * 4, g->stream), errbuf, errlen);
    unsigned blocks = (unsigned)std::min<uint64_t>((bm_words + 255) / 256, (uint64_t)g->sm_count * 4);
    if (!blocks) blocks = 1;
    compact_kernel<<<blocks, 256, 0, g->stream>>>(s.bitmaps.as<uint32_t>(), bm_words, g->count,
                                                  ids, d_count, cap);
    PV_CUDA_OK(cudaGetLastError(), errbuf, errlen);
    PV_CUDA_OK(s.tau.ensure((size_t)nq * 8), errbuf, errlen);
    PV_CUDA_OK(s.part.ensure((size_t)nq * pl.grow * topb * 8), errbuf, errlen);
    PV_CUDA_OK(s.part_cnt.ensure((size_t)nq * pl.grow * 4), errbuf, errlen);
    PV_CUDA_OK(cudaMemsetAsync(s.tau.p, 0xFF, (size_t)nq * 8, g->stream), errbuf, errlen);
    ScanF32Args a;
    a.vecs = g->d_vecs;
    a.nrows = cap;
    a.dpad = g->dpad;
    a.queries = d_q;
    a.nq = nq;
    a.bitmaps = s.bitmaps.as<uint32_t>();
    a.bm_words = bm_words;
    a.qprog = neg;  // every listed row passes
    a.K = (int)topb;
    a.S = pl.S;
    a.CB = pl.CB;
    a.rows_per_cta = pl.rows_per_cta;
    a.grow = pl.grow;
    a.qtiles = pl.qtiles;
    a.tau = s.tau.as<unsigned long long>();
    a.part = s.part.as<uint64_t>();
    a.part_cnt = s.part_cnt.as<uint32_t>();
    a.rowids = ids;
    a.nrows_dev = d_count;
    g->launches += 3;  // compaction, scan, merge
    PV_CUDA_OK(launch_scan_f32(a, pl, g->stream), errbuf, errlen);
    // the merge's truncation flag counts the filter's true matches
    PV_CUDA_OK(launch_merge(a.part, a.part_cnt, pl.grow, (int)topb, pl, a.tau, d_qprog,
                            s.popcnt.as<unsigned long long>(), g->count, nq, d_out, d_cnt,
                            d_trunc, g->stream),
               errbuf, errlen);
    return 0;
}

}  // namespace pv
