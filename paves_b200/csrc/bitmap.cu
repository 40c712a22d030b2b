// bitmap.cu — predicate programs evaluated into packed row bitmaps.
//
// One bit per row per distinct predicate of a batch (N/8 bytes: 125 KB at
// 1M rows). Each thread evaluates one row; a warp ballot forms one 32-row
// word. Column reads are coalesced over the column-major f64 attribute
// array, so one pass costs ncols_used * N * 8 bytes of HBM, once per batch
// instead of once per candidate. The evaluation follows the reference's
// FvPred::eval_node (engine.cpp:397-431) and fv_eval_dev
// (gpu_engine.cu:238-279) exactly: IEEE compares on f64, NaN is false,
// NE is (v == v && v != c).
#include "common.cuh"

namespace pv {

__device__ __forceinline__ bool cmp_op(double v, int op, double c) {
    switch (op) {
        case FV_CMP_LT: return v < c;
        case FV_CMP_LE: return v <= c;
        case FV_CMP_EQ: return v == c;
        case FV_CMP_GE: return v >= c;
        case FV_CMP_GT: return v > c;
        case FV_CMP_NE: return v == v && v != c;
    }
    return false;
}

// Evaluates one program for one row with a bit stack (top = bit 0).
__device__ __forceinline__ bool eval_prog(const PredInsn *__restrict__ ins, int n,
                                          const double *__restrict__ consts,
                                          const double *__restrict__ cols,
                                          uint64_t nrows, uint64_t row) {
    uint64_t st = 0;
    for (int i = 0; i < n; i++) {
        const PredInsn in = ins[i];
        switch (in.kind) {
            case FV_NODE_CMP: {
                double v = __ldg(cols + (uint64_t)in.col * nrows + row);
                st = (st << 1) | (cmp_op(v, in.op, in.value) ? 1u : 0u);
                break;
            }
            case FV_NODE_IN: {
                double v = __ldg(cols + (uint64_t)in.col * nrows + row);
                bool b = false;
                for (int j = 0; j < in.n; j++) b |= (v == consts[in.val0 + j]);
                st = (st << 1) | (b ? 1u : 0u);
                break;
            }
            case FV_NODE_AND:
                if (in.n == 0) st = (st << 1) | 1u;
                else { uint64_t b = st & 3u; st = (st >> 2) << 1 | (b == 3u ? 1u : 0u); }
                break;
            case FV_NODE_OR:
                if (in.n == 0) st = st << 1;
                else { uint64_t b = st & 3u; st = (st >> 2) << 1 | (b != 0u ? 1u : 0u); }
                break;
            case FV_NODE_NOT:
                st ^= 1u;
                break;
        }
    }
    return st & 1u;
}

// grid: (ceil(words / 8), P); block 256 = 8 warps, one 32-row word per warp
// per grid-stride step. popcnt[p] receives the number of passing rows.
__global__ void __launch_bounds__(256)
bitmap_kernel(const double *__restrict__ cols, uint64_t nrows,
              const PredInsn *__restrict__ insns, const PredProg *__restrict__ progs,
              const double *__restrict__ consts, uint32_t *__restrict__ bitmaps,
              uint64_t bm_words, unsigned long long *__restrict__ popcnt) {
    __shared__ PredInsn s_ins[128];
    const int p = blockIdx.y;
    const PredProg pg = progs[p];
    const bool in_smem = pg.ninsn <= 128;
    if (in_smem)
        for (int i = threadIdx.x; i < pg.ninsn; i += blockDim.x) s_ins[i] = insns[pg.insn0 + i];
    __syncthreads();
    const PredInsn *ins = in_smem ? s_ins : insns + pg.insn0;
    const int lane = threadIdx.x & 31;
    const uint64_t warp0 = (uint64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const uint64_t wstride = (uint64_t)gridDim.x * 8;
    uint32_t mycount = 0;
    for (uint64_t w = warp0; w < bm_words; w += wstride) {
        uint64_t row = w * 32 + lane;
        bool b = row < nrows && eval_prog(ins, pg.ninsn, consts, cols, nrows, row);
        uint32_t word = __ballot_sync(0xffffffffu, b);
        if (lane == 0) {
            bitmaps[(uint64_t)p * bm_words + w] = word;
            mycount += __popc(word);
        }
    }
    __shared__ unsigned int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    if (lane == 0 && mycount) atomicAdd(&s_cnt, mycount);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt) atomicAdd(popcnt + p, (unsigned long long)s_cnt);
}

constexpr int BM_REG_COLS = 4;  // columns held in registers per row group

// All programs of a batch in one pass: a warp takes 4 consecutive 32-row
// words and evaluates every program on them, 4 rows per lane in flight, so
// a column's values are fetched from HBM once per batch and re-read from
// L1 by the other programs. Programs and constants live in shared memory
// (dynamic: up to the launch's capacities). dcounts, if given, holds the
// batch's {P, ninsns, nconsts} in device memory (each <= its capacity), so
// one launch shape serves batches of varying predicates.
__global__ void __launch_bounds__(256)
bitmap_multi_kernel(const double *__restrict__ cols, uint64_t nrows,
                    const PredInsn *__restrict__ insns, int ninsns,
                    const PredProg *__restrict__ progs, int P,
                    const double *__restrict__ consts, int nconsts,
                    const int *__restrict__ dcounts, int ncols,
                    uint32_t *__restrict__ bitmaps, uint64_t bm_words,
                    unsigned long long *__restrict__ popcnt) {
    extern __shared__ __align__(16) unsigned char bm_smem[];
    PredInsn *s_ins = (PredInsn *)bm_smem;                    // [ninsns cap]
    PredProg *s_prog = (PredProg *)(s_ins + ninsns);          // [P cap]
    double *s_const = (double *)(s_prog + P + (P & 1));       // [nconsts cap]
    unsigned int *s_cnt = (unsigned int *)(s_const + nconsts);  // [P cap]
    if (dcounts) {
        P = min(P, dcounts[0]);
        ninsns = min(ninsns, dcounts[1]);
        nconsts = min(nconsts, dcounts[2]);
    }
    for (int i = threadIdx.x; i < ninsns; i += blockDim.x) s_ins[i] = insns[i];
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        PredProg pg = progs[i];
        // a program reaching past the copied instructions evaluates to false
        if (pg.insn0 < 0 || pg.ninsn < 0 || pg.insn0 + pg.ninsn > ninsns) pg.ninsn = 0;
        s_prog[i] = pg;
        s_cnt[i] = 0;
    }
    for (int i = threadIdx.x; i < nconsts; i += blockDim.x) s_const[i] = consts[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t groups = (bm_words + 3) / 4;
    const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t grp = gw; grp < groups; grp += nw) {
        uint64_t row[4];
        bool live[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            row[j] = (grp * 4 + j) * 32 + lane;
            live[j] = row[j] < nrows;
        }
        // with few columns, each row's values are read once into registers
        // for all programs
        double cv[BM_REG_COLS][4];
        if (ncols <= BM_REG_COLS) {
#pragma unroll
            for (int cc = 0; cc < BM_REG_COLS; cc++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    cv[cc][j] = (cc < ncols && live[j]) ? __ldg(cols + (uint64_t)cc * nrows + row[j])
                                                         : 0.0;
        }
        for (int p = 0; p < P; p++) {
            const PredProg pg = s_prog[p];
            uint64_t st[4] = {0, 0, 0, 0};
            for (int i = 0; i < pg.ninsn; i++) {
                const PredInsn in = s_ins[pg.insn0 + i];
                if (in.kind == FV_NODE_CMP || in.kind == FV_NODE_IN) {
                    double v[4];
                    if (ncols <= BM_REG_COLS) {
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            double x = cv[0][j];
#pragma unroll
                            for (int cc = 1; cc < BM_REG_COLS; cc++)
                                if (in.col == cc) x = cv[cc][j];
                            v[j] = x;
                        }
                    } else {
                        const double *c = cols + (uint64_t)in.col * nrows;
#pragma unroll
                        for (int j = 0; j < 4; j++) v[j] = live[j] ? __ldg(c + row[j]) : 0.0;
                    }
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        bool b;
                        if (in.kind == FV_NODE_CMP) {
                            b = cmp_op(v[j], in.op, in.value);
                        } else {
                            b = false;
                            for (int k = 0; k < in.n; k++) {
                                const int ci = in.val0 + k;
                                b |= ci < nconsts && v[j] == s_const[ci];
                            }
                        }
                        st[j] = (st[j] << 1) | (b ? 1u : 0u);
                    }
                } else if (in.kind == FV_NODE_AND || in.kind == FV_NODE_OR) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        if (in.n == 0) {
                            st[j] = (st[j] << 1) | (in.kind == FV_NODE_AND ? 1u : 0u);
                        } else {
                            const uint64_t b = st[j] & 3u;
                            const bool r = in.kind == FV_NODE_AND ? b == 3u : b != 0u;
                            st[j] = ((st[j] >> 2) << 1) | (r ? 1u : 0u);
                        }
                    }
                } else {  // NOT
#pragma unroll
                    for (int j = 0; j < 4; j++) st[j] ^= 1u;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t word = __ballot_sync(0xffffffffu, live[j] && (st[j] & 1u));
                const uint64_t w = grp * 4 + j;
                if (lane == 0 && w < bm_words) {
                    bitmaps[(uint64_t)p * bm_words + w] = word;
                    if (word) atomicAdd(&s_cnt[p], (unsigned)__popc(word));
                }
            }
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += blockDim.x)
        if (s_cnt[p]) atomicAdd(popcnt + p, (unsigned long long)s_cnt[p]);
}

size_t bitmap_multi_smem(int P, int ninsns, int nconsts) {
    return (size_t)ninsns * sizeof(PredInsn) + (size_t)(P + (P & 1)) * sizeof(PredProg) +
           (size_t)nconsts * 8 + (size_t)P * 4;
}
constexpr size_t BM_SMEM_MAX = 200 * 1024;

static cudaError_t launch_multi(const double *cols, uint64_t nrows, const PredInsn *insns,
                                const PredProg *progs, const double *consts, int P,
                                int ninsns, int nconsts, const int *dcounts, int ncols,
                                uint32_t *bitmaps, uint64_t bm_words,
                                unsigned long long *popcnt, int sm_count, cudaStream_t st) {
    const size_t smem = bitmap_multi_smem(P, ninsns, nconsts);
    cudaError_t e = cudaFuncSetAttribute(bitmap_multi_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint64_t groups = (bm_words + 3) / 4;
    uint64_t blocks = (groups + 7) / 8;
    const uint64_t cap = (uint64_t)sm_count * (smem <= 48 * 1024 ? 4 : 1);
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    bitmap_multi_kernel<<<(unsigned)blocks, 256, smem, st>>>(cols, nrows, insns, ninsns, progs, P,
                                                             consts, nconsts, dcounts, ncols,
                                                             bitmaps, bm_words, popcnt);
    return cudaGetLastError();
}

cudaError_t launch_bitmaps(const double *cols, uint64_t nrows, const PredInsn *insns,
                           const PredProg *progs, const double *consts, int P,
                           uint32_t *bitmaps, uint64_t bm_words,
                           unsigned long long *popcnt, int sm_count, cudaStream_t st,
                           int ninsns, int nconsts, int ncols) {
    if (P <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(popcnt, 0, sizeof(unsigned long long) * P, st);
    if (e != cudaSuccess) return e;
    if (bitmap_multi_smem(P, ninsns, nconsts) <= BM_SMEM_MAX)
        return launch_multi(cols, nrows, insns, progs, consts, P, ninsns, nconsts, nullptr, ncols,
                            bitmaps, bm_words, popcnt, sm_count, st);
    uint64_t blocks = (bm_words + 7) / 8;
    uint64_t cap = (uint64_t)sm_count * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    dim3 grid((unsigned)blocks, (unsigned)P);
    bitmap_kernel<<<grid, 256, 0, st>>>(cols, nrows, insns, progs, consts, bitmaps,
                                        bm_words, popcnt);
    return cudaGetLastError();
}

cudaError_t launch_bitmaps_capped(const double *cols, uint64_t nrows, const PredInsn *insns,
                                  const PredProg *progs, const double *consts,
                                  const int *dcounts, int P_cap, int insn_cap, int const_cap,
                                  uint32_t *bitmaps, uint64_t bm_words,
                                  unsigned long long *popcnt, int sm_count, cudaStream_t st,
                                  int ncols) {
    if (P_cap <= 0) return cudaSuccess;
    if (bitmap_multi_smem(P_cap, insn_cap, const_cap) > BM_SMEM_MAX) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(popcnt, 0, sizeof(unsigned long long) * P_cap, st);
    if (e != cudaSuccess) return e;
    return launch_multi(cols, nrows, insns, progs, consts, P_cap, insn_cap, const_cap, dcounts, ncols,
                        bitmaps, bm_words, popcnt, sm_count, st);
}

}  // namespace pv
