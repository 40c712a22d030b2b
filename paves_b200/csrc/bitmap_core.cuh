// bitmap_core.cuh — predicate programs evaluated into packed row bitmaps
// (the work of bitmap_multi_kernel as a device function, so a persistent
// kernel can run it as one of its phases). See bitmap.cu for the design.
#pragma once
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

constexpr int BM_REG_COLS = 4;    // columns held in registers per row group
constexpr int BM_PCH = 8;         // programs per work item
constexpr int BM_INS_WIN = 256;   // a work item's instructions kept in shared memory
constexpr int BM_CONST_WIN = 256; // constants kept in shared memory
constexpr int BM_BLOCKS_PER_SM = 2;

// All programs of a batch, by blocks bid = 0 .. nblk-1 of the caller's grid. Work items are (program chunk of
// BM_PCH programs, row block); items of the same row block sit next to each
// other in launch order, so the chunks that run together read the same
// attribute values (from HBM once, then L2). A warp takes 4 consecutive
// 32-row words, holds their column values in registers (<= BM_REG_COLS
// columns) and evaluates its chunk's programs on them, 4 rows per lane in
// flight. Shared memory is fixed and small (the chunk's programs, their
// instruction window, the constants if they fit; otherwise read from
// global memory), so several blocks share an SM whatever the batch size.
// dcounts, if given, holds the batch's {P, ninsns, nconsts} in device
// memory (each <= the launch's values): the split into chunks follows the
// actual P, so one launch shape of a CUDA graph serves any batch.
static __device__ __forceinline__ void bitmap_work(
    int bid, int nblk, const double *__restrict__ cols, uint64_t nrows,
    const PredInsn *__restrict__ insns, int ninsns, const PredProg *__restrict__ progs, int P,
    const double *__restrict__ consts, int nconsts, const int *__restrict__ dcounts, int ncols,
    uint32_t *__restrict__ bitmaps, uint64_t bm_words, unsigned long long *__restrict__ popcnt) {
    __shared__ PredInsn s_ins[BM_INS_WIN];
    __shared__ double s_const[BM_CONST_WIN];
    __shared__ PredProg s_prog[BM_PCH];
    __shared__ unsigned int s_cnt[BM_PCH];
    // range programs of the chunk, decoded: s_nt terms (-1: stack program)
    __shared__ int s_nt[BM_PCH];
    __shared__ int s_tcol[BM_PCH][PV_RANGE_MAX_TERMS];  // col | PV_TERM_MASK
    __shared__ double s_tlo[BM_PCH][PV_RANGE_MAX_TERMS], s_thi[BM_PCH][PV_RANGE_MAX_TERMS];
    __shared__ unsigned long long s_tbits[BM_PCH][PV_RANGE_MAX_TERMS];
    __shared__ int s_mcols;  // register columns that IN-set terms test
    __shared__ int s_ucols;  // register columns that the chunk's programs read
    if (dcounts) {
        P = min(P, dcounts[0]);
        ninsns = min(ninsns, dcounts[1]);
        nconsts = min(nconsts, dcounts[2]);
    }
    const int nch = (P + BM_PCH - 1) / BM_PCH;
    if (nch == 0) return;
    const bool const_sm = nconsts <= BM_CONST_WIN;
    for (int i = threadIdx.x; i < nconsts && const_sm; i += blockDim.x) s_const[i] = consts[i];
    const double *cst = const_sm ? s_const : consts;
    const int lane = threadIdx.x & 31;
    const uint64_t groups = (bm_words + 3) / 4;
    const uint64_t nrb = (unsigned)nblk >= (unsigned)nch ? (unsigned)nblk / nch : 1;
    for (uint64_t item = bid; item < nrb * nch; item += (unsigned)nblk) {
        const int chunk = (int)(item % nch);
        const uint64_t rb = item / nch;
        const int p0 = chunk * BM_PCH, np = min(BM_PCH, P - p0);
        // the chunk's instruction window [lo, hi)
        // a program reaching past the batch's instructions evaluates to false
        auto prog_at = [&](int i) {
            PredProg pg = i < np ? progs[p0 + i] : PredProg{0, 0};
            if (pg.insn0 < 0 || pg.ninsn < 0 || pg.insn0 + pg.ninsn > ninsns) pg.ninsn = 0;
            return pg;
        };
        int lo = ninsns, hi = 0;
        for (int i = 0; i < np; i++) {
            const PredProg pg = prog_at(i);
            if (pg.ninsn > 0) {
                lo = min(lo, pg.insn0);
                hi = max(hi, pg.insn0 + pg.ninsn);
            }
        }
        const bool ins_sm = hi - lo <= BM_INS_WIN;
        __syncthreads();  // the previous item is done with s_ins / s_prog
        if (ins_sm)
            for (int i = threadIdx.x; i < hi - lo; i += blockDim.x) s_ins[i] = insns[lo + i];
        if (threadIdx.x < BM_PCH) {
            PredProg pg = prog_at(threadIdx.x);
            if (ins_sm && pg.ninsn > 0) pg.insn0 -= lo;
            s_prog[threadIdx.x] = pg;
            s_cnt[threadIdx.x] = 0;
        }
        if (threadIdx.x == 0) {
            s_mcols = 0;
            s_ucols = 0;
        }
        __syncthreads();
        const PredInsn *ins = ins_sm ? s_ins : insns;
        if (threadIdx.x < BM_PCH) {
            // decode a range program's terms; a term whose constants lie
            // outside the batch's pool admits nothing
            const int p = threadIdx.x;
            const PredProg pg = s_prog[p];
            int nt = -1;
            if (p < np && pg.ninsn == 1 && ins[pg.insn0].kind == PV_NODE_RANGE) {
                const PredInsn r = ins[pg.insn0];
                nt = min(max(r.n, 0), PV_RANGE_MAX_TERMS);
                int ci = r.val0;
                for (int k = 0; k < nt; k++) {
                    int tc = 0;
                    double tlo = NAN, thi = NAN;
                    unsigned long long bits = 0;
                    if (ci >= 0 && ci + 2 <= nconsts) {
                        const int meta = (int)cst[ci];
                        const int col = meta & 0xFFFF;
                        if (meta & PV_TERM_MASK) {
                            tc = col | PV_TERM_MASK;
                            bits = (unsigned long long)__double_as_longlong(cst[ci + 1]);
                            if (col < BM_REG_COLS) atomicOr(&s_mcols, 1 << col);
                            ci += 2;
                        } else {
                            tc = col;
                            if (ci + 3 <= nconsts) {
                                tlo = cst[ci + 1];
                                thi = cst[ci + 2];
                            }
                            ci += 3;
                        }
                    }
                    s_tcol[p][k] = tc;
                    s_tlo[p][k] = tlo;
                    s_thi[p][k] = thi;
                    s_tbits[p][k] = bits;
                }
            }
            s_nt[p] = nt;
            // the register columns these programs read (a column past the
            // register set reads the one that stands in for it below)
            int used = 0;
            if (p < np) {
                if (nt >= 0) {
                    for (int k = 0; k < nt; k++) used |= 1 << min(s_tcol[p][k] & 0xFFFF, 3);
                } else {
                    for (int i = 0; i < pg.ninsn; i++) {
                        const PredInsn in = ins[pg.insn0 + i];
                        if (in.kind == FV_NODE_CMP || in.kind == FV_NODE_IN)
                            used |= 1 << ((unsigned)in.col < (unsigned)BM_REG_COLS ? in.col : 0);
                    }
                }
            }
            if (used) atomicOr(&s_ucols, used);
        }
        __syncthreads();
        const int mcols = s_mcols;
        const uint64_t gw = rb * (blockDim.x / 32) + (threadIdx.x >> 5);
        const uint64_t nw = nrb * (blockDim.x / 32);
        for (uint64_t grp = gw; grp < groups; grp += nw) {
            uint64_t row[4];
            bool live[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                row[j] = (grp * 4 + j) * 32 + lane;
                live[j] = row[j] < nrows;
            }
            // with few columns, each row's values are read once into
            // registers for all programs of the chunk (only the columns they
            // test: a one-column filter reads one column of the table)
            double cv[BM_REG_COLS][4];
            if (ncols <= BM_REG_COLS) {
#pragma unroll
                for (int cc = 0; cc < BM_REG_COLS; cc++)
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        cv[cc][j] = (cc < ncols && ((s_ucols >> cc) & 1) && live[j])
                                        ? __ldg(cols + (uint64_t)cc * nrows + row[j])
                                        : 0.0;
            }
            // value of column col for the 4 rows (registers or global memory)
            auto colval = [&](int col, double (&v)[4]) {
                if (ncols <= BM_REG_COLS) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        double x = cv[0][j];
#pragma unroll
                        for (int cc = 1; cc < BM_REG_COLS; cc++)
                            if (col == cc) x = cv[cc][j];
                        v[j] = x;
                    }
                } else {
                    const double *c = cols + (uint64_t)col * nrows;
#pragma unroll
                    for (int j = 0; j < 4; j++) v[j] = live[j] ? __ldg(c + row[j]) : 0.0;
                }
            };
            // small-integer code of the values of columns that IN-set terms
            // test (64: not an integer in [0, 64))
            int code[BM_REG_COLS][4];
            if (ncols <= BM_REG_COLS && mcols) {
#pragma unroll
                for (int cc = 0; cc < BM_REG_COLS; cc++)
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const double x = cv[cc][j];
                        const bool in = (mcols >> cc) & 1 && x >= 0.0 && x < 64.0;
                        const int b = in ? (int)x : 64;
                        code[cc][j] = (in && (double)b == x) ? b : 64;
                    }
            }
            // the 4 words of program p: lanes 0-3 store one each, lane 0
            // adds their population to the program's count
            auto store_words = [&](int p, const bool (&b)[4]) {
                uint32_t wd[4];
#pragma unroll
                for (int j = 0; j < 4; j++) wd[j] = __ballot_sync(0xffffffffu, b[j]);
                const uint64_t w = grp * 4 + lane;
                if (lane < 4 && w < bm_words) {
                    const uint32_t mine = lane == 0 ? wd[0] : lane == 1 ? wd[1] : lane == 2 ? wd[2] : wd[3];
                    bitmaps[(uint64_t)(p0 + p) * bm_words + w] = mine;
                }
                if (lane == 0) {
                    const unsigned c = __popc(wd[0]) + __popc(wd[1]) + __popc(wd[2]) + __popc(wd[3]);
                    if (c) atomicAdd(&s_cnt[p], c);
                }
            };
            for (int p = 0; p < np; p++) {
                const PredProg pg = s_prog[p];
                const int nt = s_nt[p];
                if (nt >= 0) {
                    // range form: AND of closed intervals and small-integer sets
                    bool ok[4] = {live[0], live[1], live[2], live[3]};
                    auto iv = [&](const double (&x)[4], double tlo, double thi) {
#pragma unroll
                        for (int j = 0; j < 4; j++) ok[j] = ok[j] && x[j] >= tlo && x[j] <= thi;
                    };
                    auto mk = [&](const int (&c)[4], unsigned long long bits) {
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            ok[j] = ok[j] && c[j] < 64 && ((bits >> (c[j] & 63)) & 1ull);
                    };
                    for (int k = 0; k < nt; k++) {
                        const int tc = s_tcol[p][k];
                        const int col = tc & 0xFFFF;
                        const bool is_mask = tc & PV_TERM_MASK;
                        if (ncols <= BM_REG_COLS) {
                            if (is_mask) {
                                const unsigned long long bits = s_tbits[p][k];
                                switch (col) {
                                    case 0: mk(code[0], bits); break;
                                    case 1: mk(code[1], bits); break;
                                    case 2: mk(code[2], bits); break;
                                    default: mk(code[3], bits); break;
                                }
                            } else {
                                const double tlo = s_tlo[p][k], thi = s_thi[p][k];
                                switch (col) {
                                    case 0: iv(cv[0], tlo, thi); break;
                                    case 1: iv(cv[1], tlo, thi); break;
                                    case 2: iv(cv[2], tlo, thi); break;
                                    default: iv(cv[3], tlo, thi); break;
                                }
                            }
                        } else {
                            double v[4];
                            colval(col, v);
                            if (is_mask) {
                                int c[4];
#pragma unroll
                                for (int j = 0; j < 4; j++) {
                                    const bool in = v[j] >= 0.0 && v[j] < 64.0;
                                    const int b = in ? (int)v[j] : 64;
                                    c[j] = (in && (double)b == v[j]) ? b : 64;
                                }
                                mk(c, s_tbits[p][k]);
                            } else {
                                iv(v, s_tlo[p][k], s_thi[p][k]);
                            }
                        }
                    }
                    store_words(p, ok);
                    continue;
                }
                uint64_t st[4] = {0, 0, 0, 0};
                for (int i = 0; i < pg.ninsn; i++) {
                    const PredInsn in = ins[pg.insn0 + i];
                    if (in.kind == FV_NODE_CMP || in.kind == FV_NODE_IN) {
                        double v[4];
                        colval(in.col, v);
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            bool b;
                            if (in.kind == FV_NODE_CMP) {
                                b = cmp_op(v[j], in.op, in.value);
                            } else {
                                b = false;
                                for (int k = 0; k < in.n; k++) {
                                    const int ci = in.val0 + k;
                                    b |= (unsigned)ci < (unsigned)nconsts && v[j] == cst[ci];
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
                bool res[4];
#pragma unroll
                for (int j = 0; j < 4; j++) res[j] = live[j] && (st[j] & 1u);
                store_words(p, res);
            }
        }
        __syncthreads();
        if (threadIdx.x < np && s_cnt[threadIdx.x])
            atomicAdd(popcnt + p0 + threadIdx.x, (unsigned long long)s_cnt[threadIdx.x]);
    }
}

}  // namespace pv
