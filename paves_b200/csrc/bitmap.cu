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

cudaError_t launch_bitmaps(const double *cols, uint64_t nrows, const PredInsn *insns,
                           const PredProg *progs, const double *consts, int P,
                           uint32_t *bitmaps, uint64_t bm_words,
                           unsigned long long *popcnt, int sm_count, cudaStream_t st,
                           int ninsns, int nconsts, int ncols) {
    if (P <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(popcnt, 0, sizeof(unsigned long long) * P, st);
    if (e != cudaSuccess) return e;
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
