// bitmap.cu — predicate programs evaluated into packed row bitmaps.
//
// One bit per row per distinct predicate of a batch (N/8 bytes: 125 KB at
// 1M rows). Each thread evaluates one row; a warp ballot forms one 32-row
// word. Column reads are coalesced over the column-major f64 attribute
// array, so one pass costs ncols_used * N * 8 bytes of HBM, once per batch
// instead of once per candidate. The evaluation follows the reference's
// FvPred::eval_node (engine.cpp:397-431) and fv_eval_dev
// (gpu_engine.cu:238-279) exactly: IEEE compares on f64, NaN is false,
// NE is (v == v && v != c). Programs that are an AND of comparisons and IN
// lists arrive in range form (one instruction: per-column intervals and
// small-integer sets, compiled on the host) and cost a few instructions per
// row; others run on the bit-stack interpreter.
#include "bitmap_core.cuh"
#include "launch.cuh"

namespace pv {

__global__ void __launch_bounds__(256, BM_BLOCKS_PER_SM)
bitmap_multi_kernel(const double *__restrict__ cols, uint64_t nrows,
                    const PredInsn *__restrict__ insns, int ninsns,
                    const PredProg *__restrict__ progs, int P,
                    const double *__restrict__ consts, int nconsts,
                    const int *__restrict__ dcounts, int ncols,
                    uint32_t *__restrict__ bitmaps, uint64_t bm_words,
                    unsigned long long *__restrict__ popcnt) {
    pdl_wait();
    pdl_trigger();
    bitmap_work(blockIdx.x, gridDim.x, cols, nrows, insns, ninsns, progs, P, consts, nconsts,
                dcounts, ncols, bitmaps, bm_words, popcnt);
}

static cudaError_t launch_multi(const double *cols, uint64_t nrows, const PredInsn *insns,
                                const PredProg *progs, const double *consts, int P,
                                int ninsns, int nconsts, const int *dcounts, int ncols,
                                uint32_t *bitmaps, uint64_t bm_words,
                                unsigned long long *popcnt, int sm_count, cudaStream_t st) {
    const uint64_t groups = (bm_words + 3) / 4;
    const uint64_t nch = (uint64_t)(P + BM_PCH - 1) / BM_PCH;
    uint64_t blocks = nch * ((groups + 7) / 8);
    const uint64_t cap = (uint64_t)sm_count * BM_BLOCKS_PER_SM;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    return launch_pdl(bitmap_multi_kernel, dim3((unsigned)blocks), dim3(256), 0, st, cols, nrows,
                      insns, ninsns, progs, P, consts, nconsts, dcounts, ncols, bitmaps, bm_words,
                      popcnt);
}

// One program in range form (a batch sharing one filter that is an AND of
// per-column intervals and small-integer sets, every term's constants in
// the pool and its column in the table: checked on the host). A lean
// kernel: a warp evaluates 4 consecutive 32-row words, 4 rows per lane in
// flight, with few registers, so every word of the index is in flight in
// one wave (the general kernel holds 128 registers per thread for up to 4
// register columns x 8 programs and walks 3-4 row groups per warp). The
// tests are those of bitmap_work's range path: f64 compares, NaN fails,
// an IN-set term admits an integer b in [0, 64) with bit b of its mask.
__global__ void __launch_bounds__(256)
bitmap_range1_kernel(const double *__restrict__ cols, uint64_t nrows,
                     const PredInsn *__restrict__ insns, const PredProg *__restrict__ progs,
                     const double *__restrict__ consts, int nconsts,
                     uint32_t *__restrict__ bitmap, uint64_t bm_words,
                     unsigned long long *__restrict__ popcnt) {
    __shared__ unsigned int s_cnt;
    pdl_wait();
    pdl_trigger();
    if (threadIdx.x == 0) s_cnt = 0;
    const PredInsn r = insns[progs[0].insn0];
    const int nt = min(max(r.n, 0), PV_RANGE_MAX_TERMS);
    int tcol[PV_RANGE_MAX_TERMS];
    bool tmask[PV_RANGE_MAX_TERMS];
    double tlo[PV_RANGE_MAX_TERMS], thi[PV_RANGE_MAX_TERMS];
    unsigned long long tbits[PV_RANGE_MAX_TERMS];
    int ci = r.val0;
#pragma unroll
    for (int k = 0; k < PV_RANGE_MAX_TERMS; k++) {
        tcol[k] = 0;
        tmask[k] = false;
        tlo[k] = thi[k] = __longlong_as_double(0x7ff8000000000000ll);  // NaN: admits nothing
        tbits[k] = 0;
        if (k < nt && ci >= 0 && ci + 2 <= nconsts) {
            const int meta = (int)consts[ci];
            tcol[k] = meta & 0xFFFF;
            if (meta & PV_TERM_MASK) {
                tmask[k] = true;
                tbits[k] = (unsigned long long)__double_as_longlong(consts[ci + 1]);
                ci += 2;
            } else {
                if (ci + 3 <= nconsts) {
                    tlo[k] = consts[ci + 1];
                    thi[k] = consts[ci + 2];
                }
                ci += 3;
            }
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t w0 = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 4;
    uint64_t row[4];
    bool ok[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        row[j] = (w0 + j) * 32 + lane;
        ok[j] = row[j] < nrows;
    }
#pragma unroll
    for (int k = 0; k < PV_RANGE_MAX_TERMS; k++) {
        if (k >= nt) break;
        const double *c = cols + (uint64_t)tcol[k] * nrows;
        double v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = ok[j] ? __ldg(c + row[j]) : 0.0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (tmask[k]) {
                const bool in = v[j] >= 0.0 && v[j] < 64.0;
                const int b = in ? (int)v[j] : 64;
                const int code = (in && (double)b == v[j]) ? b : 64;
                ok[j] = ok[j] && code < 64 && ((tbits[k] >> (code & 63)) & 1ull);
            } else {
                ok[j] = ok[j] && v[j] >= tlo[k] && v[j] <= thi[k];
            }
        }
    }
    unsigned int cnt = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint32_t wd = __ballot_sync(0xffffffffu, ok[j]);
        if (lane == j && w0 + j < bm_words) bitmap[w0 + j] = wd;
        cnt += __popc(wd);
    }
    if (lane == 0 && cnt) atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt) atomicAdd(popcnt, (unsigned long long)s_cnt);
}

cudaError_t launch_bitmaps(const double *cols, uint64_t nrows, const PredInsn *insns,
                           const PredProg *progs, const double *consts, int P,
                           uint32_t *bitmaps, uint64_t bm_words,
                           unsigned long long *popcnt, int sm_count, cudaStream_t st,
                           int ninsns, int nconsts, int ncols, bool one_range) {
    if (P <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(popcnt, 0, sizeof(unsigned long long) * P, st);
    if (e != cudaSuccess) return e;
    if (one_range && P == 1) {
        const uint64_t blocks = (bm_words + 31) / 32;  // 8 warps x 4 words
        return launch_pdl(bitmap_range1_kernel, dim3((unsigned)(blocks ? blocks : 1)), dim3(256),
                          0, st, cols, nrows, insns, progs, consts, nconsts, bitmaps, bm_words,
                          popcnt);
    }
    return launch_multi(cols, nrows, insns, progs, consts, P, ninsns, nconsts, nullptr, ncols,
                        bitmaps, bm_words, popcnt, sm_count, st);
}

cudaError_t launch_bitmaps_capped(const double *cols, uint64_t nrows, const PredInsn *insns,
                                  const PredProg *progs, const double *consts,
                                  const int *dcounts, int P_cap, int insn_cap, int const_cap,
                                  uint32_t *bitmaps, uint64_t bm_words,
                                  unsigned long long *popcnt, int sm_count, cudaStream_t st,
                                  int ncols) {
    if (P_cap <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(popcnt, 0, sizeof(unsigned long long) * P_cap, st);
    if (e != cudaSuccess) return e;
    return launch_multi(cols, nrows, insns, progs, consts, P_cap, insn_cap, const_cap, dcounts, ncols,
                        bitmaps, bm_words, popcnt, sm_count, st);
}

}  // namespace pv
