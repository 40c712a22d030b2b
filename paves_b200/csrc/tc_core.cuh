// tc_core.cuh — the tensor-core filtered scan's per-CTA pass, shared by the
// one-shot scan kernel (scan_tc.cu) and the persistent micro-batch kernel.
//
// A pass streams one query tile against a CTA's row tiles:
//     D[128 queries][128 rows] = Q[128 x K] * X_tile[128 x K]^T
// (A = query tile, resident in shared memory; B = row tile, streamed by
// TMA in 128-byte-swizzled K-major boxes), D in TMEM, double buffered, so
// the MMA of tile t+1 overlaps the epilogue of tile t. In TMEM, lane =
// query and column = row: each epilogue thread owns ONE query, walks the
// tile's rows and keeps that query's best K' keys in a private
// shared-memory list with its threshold in a register. Row norms (and FP8
// scales) arrive in a shared-memory ring beside the rows; the filter is a
// bitmap word per 32 rows, or, for lazy batches, the query's range program
// evaluated only on rows that beat the threshold.
//
// Warp roles (64 + 128 * EPI threads): warp 0 TMA producer, warp 1 MMA
// issuer, then EPI groups of 4 epilogue warps (warp w reads TMEM lanes
// 32*(w%4).. ; group h takes its share of each tile's rows). A batch of at
// most 64 (32) queries is replicated 2 (4) times down the 128 query slots.
// All waits are bounded by a deadline and unwind through an abort flag.
#pragma once
#include <cuda.h>

#include "pv_internal.h"
#include "sm100.cuh"

namespace pv {

using namespace sm100;

constexpr int TC_BM = 128;          // queries per tile (MMA M)
constexpr int TC_BN = 128;          // rows per tile (MMA N)
constexpr int TC_KB_BYTES = 128;    // bytes of K per swizzle row / TMA box
constexpr int TC_BOX = TC_BN * TC_KB_BYTES;  // 16 KB per K-block box
constexpr int TC_KBS = 2;           // K-blocks per pipeline stage
// Candidates per query kept for the exact re-rank at most (the superset),
// and the list length per (query, CTA half) that holds them: when the
// superset is longer than a list, the union of the lists is the superset
// only if no full list could have dropped a member of it, which the merge
// certifies per query (queries it cannot certify are re-run exactly).
constexpr int TC_MAX_SUPERSET = 1024;
constexpr int TC_MAX_LIST = 64;
constexpr int TC_MAX_STAGES = 8;   // TMA pipeline stages at most
constexpr int TC_NR = 8;            // tiles of row norms in flight (shared-memory ring)
constexpr int TC_NSLOT_F = 2 * TC_BN;  // floats per norm slot: norms, then fp8 scales

template <bool FP8>
__device__ __forceinline__ void mma_f16_or_f8(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                              uint32_t acc) {
    if (FP8) mma_f8(d, a, b, idesc, acc);
    else mma_f16(d, a, b, idesc, acc);
}

struct TcArgs {
    uint64_t nrows;
    int kblocks;        // K-blocks (128 bytes of K each) per row
    int nq;
    int qtiles;
    int grow;           // CTAs along rows per query tile
    uint64_t tiles_per_cta;
    uint64_t tile0_mul;  // first tile of CTA group g = g * tile0_mul
    uint64_t tile_step;  // stride between a CTA's tiles
    int KP;             // list length per (query, CTA part)
    int rep;            // query replicas down the tile's 128 slots (1, 2, 4)
    int bq;             // query slots per replica = TC_BM / rep
    int push_tau;       // a full list's last key bounds the superset (lists hold it all)
    int NS;             // pipeline stages
    const float *__restrict__ xnorm;   // [rows padded to 128]
    const float *__restrict__ xscale;  // fp8: per-row scale, else null
    const float *__restrict__ qnorm;   // [nqpad]
    const float *__restrict__ qscale;  // fp8: per-query scale, else null
    const int32_t *__restrict__ qprog;
    const uint32_t *__restrict__ bitmaps;
    uint64_t bm_words;
    // lazy filters: when *lazy != 0 the batch has no bitmaps; every program
    // is in range form and is evaluated from the attribute columns only for
    // rows whose key already beats the threshold (null: bitmaps)
    const int *lazy;
    const PredProg *__restrict__ progs;
    const PredInsn *__restrict__ insns;
    const double *__restrict__ consts;
    int nconsts;
    const double *__restrict__ cols;
    int ncols;
    unsigned long long *tau;  // [nq] grid-wide bound
    // kept keys: each list appends its best kwrite keys to its query's dense
    // run dense[q][0 .. dcnt[q]) (any order; dcap >= lists per query * kwrite)
    uint64_t *dense;
    uint32_t *dcnt;
    uint64_t dcap;
    int kwrite;
    // [nq] smallest last key of a full list (the merge's certificate), or null
    unsigned long long *fullmin;
    int *err;
    // waits give up after timeout_ns (the kernel then sets *err and
    // unwinds); once unwinding, it still waits up to drain_ns for the copies
    // and MMAs it issued, so none is in flight when the CTA leaves
    uint64_t timeout_ns;
    uint64_t drain_ns;
    // optional per-tile timestamps of CTA 0 (globaltimer ns):
    // [t][0] stage issued, [t][1] MMA issued, [t][2] epilogue start, [t][3] end
    uint64_t *trace;
    int trace_tiles;
};

// Shared-memory carve of a CTA running passes: lists sized for up to KPcap
// keys per (query, part); barriers after the buffers.
struct TcSmem {
    unsigned char *sQ, *sX;
    size_t SB;  // bytes per pipeline stage
    uint64_t *lists;
    float *stage, *snorm;
    uint64_t *full, *empty, *tfull, *tempty, *qbar, *done, *nfull, *nempty;
};

__device__ __forceinline__ TcSmem tc_carve(unsigned char *base, int KBt, int NS, int KPcap,
                                           int EPI) {
    TcSmem m;
    m.sQ = base;                                       // KBt boxes
    m.sX = m.sQ + (size_t)KBt * TC_BOX;                // NS stages
    // a stage holds one K-chunk of a row tile: min(TC_KBS, KBt) boxes
    m.SB = (size_t)(KBt < TC_KBS ? KBt : TC_KBS) * TC_BOX;
    // per (query, part) lists [KP][128*EPI] and candidate staging [32][128*EPI]
    m.lists = (uint64_t *)(m.sX + (size_t)NS * m.SB);
    m.stage = (float *)(m.lists + (size_t)TC_BM * EPI * KPcap);
    // row norms (and fp8 scales) of a tile, TC_NR tiles in flight (slot =
    // [norms 128][scales 128])
    m.snorm = m.stage + 32 * TC_BM * EPI;
    uint64_t *bars = (uint64_t *)(m.snorm + (size_t)TC_NR * TC_NSLOT_F);
    m.full = bars;              // [NS]
    m.empty = m.full + NS;      // [NS]
    m.tfull = m.empty + NS;     // [2]
    m.tempty = m.tfull + 2;     // [2]
    m.qbar = m.tempty + 2;      // [1]
    m.done = m.qbar + 1;        // [1]
    m.nfull = m.done + 1;       // [TC_NR]
    m.nempty = m.nfull + TC_NR; // [TC_NR]
    return m;
}

inline size_t tc_smem_bytes(int kblocks, int NS, int KPcap, int EPI) {
    return 1024 + (size_t)kblocks * TC_BOX +
           (size_t)NS * (kblocks < TC_KBS ? kblocks : TC_KBS) * TC_BOX +
           (size_t)TC_BM * EPI * KPcap * 8 + (size_t)32 * TC_BM * EPI * 4 +
           (size_t)TC_NR * TC_NSLOT_F * 4 + (size_t)(2 * NS + 6 + 2 * TC_NR) * 8;
}

// by one thread, before the CTA's first pass
__device__ __forceinline__ void tc_init_barriers(const TcSmem &m, int NS, int EPI) {
    for (int i = 0; i < NS; i++) {
        mbar_init(&m.full[i], 1);
        mbar_init(&m.empty[i], 1);
    }
    for (int i = 0; i < 2; i++) {
        mbar_init(&m.tfull[i], 1);
        mbar_init(&m.tempty[i], TC_BM * EPI);
    }
    for (int i = 0; i < TC_NR; i++) {
        mbar_init(&m.nfull[i], 1);
        mbar_init(&m.nempty[i], 4 * EPI);  // one arrival per epilogue warp
    }
    mbar_init(m.qbar, 1);
    mbar_init(m.done, 1);
    fence_mbar_init();
}

// Running counts of a CTA's passes (phase bookkeeping of its barriers).
struct TcRun {
    uint64_t it = 0;  // pipeline stages issued / consumed
    uint64_t t = 0;   // row tiles
    uint32_t qph = 0; // passes (query-tile loads, MMA drains)
};

// One pass of the tensor-core scan by one CTA: its query tile `qtile` and
// the tiles of row group `rgrp`; all threads of the CTA call it. Barrier
// phases come from `run`, the CTA's running counts of pipeline stages,
// tiles and passes, so a kernel can run several passes over the same
// barriers and tensor memory (every role advances the counts alike).
// Returns false when a wait of this CTA gave up (*abort_flag set).
template <bool FP8, int EPI>
__device__ __forceinline__ bool tc_pass(const CUtensorMap *tmXp, const CUtensorMap *tmQp,
                                        const TcArgs &a, const TcSmem &sm, uint32_t tmem,
                                        TcRun &run, volatile int *abort_flag, int qtile,
                                        int rgrp) {
    const CUtensorMap &tmX = *tmXp;
    const CUtensorMap &tmQ = *tmQp;
    const int KBt = a.kblocks;
    const int NS = a.NS;
    const int KP = a.KP;
    unsigned char *sQ = sm.sQ;
    unsigned char *sX = sm.sX;
    const size_t SB = sm.SB;
    uint64_t *lists = sm.lists;
    float *stage = sm.stage;
    float *snorm = sm.snorm;
    uint64_t *full = sm.full, *empty = sm.empty, *tfull = sm.tfull, *tempty = sm.tempty;
    uint64_t *qbar = sm.qbar, *done = sm.done, *nfull = sm.nfull, *nempty = sm.nempty;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // this CTA's tiles: tile0 + t * tile_step, t < ntiles
    const uint64_t tile0 = (uint64_t)rgrp * a.tile0_mul;
    const uint64_t ntiles_all = (a.nrows + TC_BN - 1) / TC_BN;
    uint64_t ntiles =
        tile0 < ntiles_all ? (ntiles_all - tile0 + a.tile_step - 1) / a.tile_step : 0;
    if (ntiles > a.tiles_per_cta) ntiles = a.tiles_per_cta;
    const int nkc = (KBt + TC_KBS - 1) / TC_KBS;
    const uint64_t deadline = globaltimer() + a.timeout_ns;
    const uint64_t it0 = run.it, T0 = run.t;
    const uint32_t qph = run.qph & 1;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            prefetch_tmap(&tmX);
            prefetch_tmap(&tmQ);
            mbar_arrive_expect_tx(qbar, (uint32_t)KBt * TC_BOX);
            for (int kb = 0; kb < KBt; kb++)
                tma_load_2d(sQ + (size_t)kb * TC_BOX, &tmQ, kb * (FP8 ? 128 : 64),
                            qtile * TC_BM, qbar);
            const uint32_t nbytes = (FP8 ? 2 : 1) * TC_BN * 4;
            uint64_t it = it0, nt = T0;  // stages and norm slots issued (running)
            bool ok = true;
            for (uint64_t t = 0; t < ntiles && ok; t++) {
                const uint64_t tile = tile0 + t * a.tile_step;
                const int y = (int)(tile * TC_BN);
                // the tile's norms (and scales): arrays are padded to whole
                // tiles, rows of a tile are 512 contiguous bytes
                {
                    const uint64_t T = T0 + t;
                    const int ns = (int)(T % TC_NR);
                    if (!mbar_wait(&nempty[ns], (uint32_t)(((T / TC_NR) & 1) ^ 1), deadline,
                                   abort_flag)) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&nfull[ns], nbytes);
                    float *dst = snorm + (size_t)ns * TC_NSLOT_F;
                    bulk_load(dst, a.xnorm + tile * TC_BN, TC_BN * 4, &nfull[ns]);
                    if (FP8) bulk_load(dst + TC_BN, a.xscale + tile * TC_BN, TC_BN * 4, &nfull[ns]);
                    nt = T + 1;
                }
                for (int kc = 0; kc < nkc; kc++, it++) {
                    const int s = (int)(it % NS);
                    const uint32_t ph = (uint32_t)((it / NS) & 1);
                    if (!mbar_wait(&empty[s], ph ^ 1, deadline, abort_flag)) { ok = false; break; }
                    const int nkb = min(TC_KBS, KBt - kc * TC_KBS);
                    mbar_arrive_expect_tx(&full[s], (uint32_t)nkb * TC_BOX);
                    for (int kb = 0; kb < nkb; kb++)
                        tma_load_2d(sX + (size_t)s * SB + (size_t)kb * TC_BOX, &tmX,
                                    (kc * TC_KBS + kb) * (FP8 ? 128 : 64), y, &full[s]);
                }
                if (a.trace && blockIdx.x == 0 && t < (uint64_t)a.trace_tiles)
                    a.trace[t * 4 + 0] = globaltimer();
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(a.err, 1);
            }
            // copies still in flight land before the CTA leaves
            const uint64_t d2 = globaltimer() + a.drain_ns;
            volatile int zero = 0;
            const uint64_t first = it > it0 + NS ? it - NS : it0;
            for (uint64_t j = first; j < it; j++)
                mbar_wait(&full[j % NS], (uint32_t)((j / NS) & 1), d2, &zero);
            const uint64_t nfirst = nt > T0 + TC_NR ? nt - TC_NR : T0;
            for (uint64_t j = nfirst; j < nt; j++)
                mbar_wait(&nfull[j % TC_NR], (uint32_t)((j / TC_NR) & 1), d2, &zero);
            mbar_wait(qbar, qph, d2, &zero);
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = FP8 ? idesc_make(FMT_E4M3, FMT_E4M3, TC_BM, TC_BN)
                                       : idesc_make(FMT_BF16, FMT_BF16, TC_BM, TC_BN);
            bool ok = mbar_wait(qbar, qph, deadline, abort_flag);
            uint64_t it = it0;
            for (uint64_t t = 0; t < ntiles && ok; t++) {
                const uint64_t T = T0 + t;
                const int acc = (int)(T & 1);
                const uint32_t aph = (uint32_t)((T >> 1) & 1);
                if (!mbar_wait(&tempty[acc], aph ^ 1, deadline, abort_flag)) { ok = false; break; }
                tc_fence_after();
                const uint32_t dcol = tmem + (uint32_t)acc * TC_BN;
                for (int kc = 0; kc < nkc && ok; kc++, it++) {
                    const int s = (int)(it % NS);
                    const uint32_t ph = (uint32_t)((it / NS) & 1);
                    if (!mbar_wait(&full[s], ph, deadline, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const int nkb = min(TC_KBS, KBt - kc * TC_KBS);
                    for (int kb = 0; kb < nkb; kb++) {
                        const uint64_t ad = desc_sw128(sQ + (size_t)(kc * TC_KBS + kb) * TC_BOX);
                        const uint64_t bd = desc_sw128(sX + (size_t)s * SB + (size_t)kb * TC_BOX);
#pragma unroll
                        for (int kk = 0; kk < 4; kk++)  // 4 x 32 bytes of K per block
                            mma_f16_or_f8<FP8>(dcol, ad + 2 * kk, bd + 2 * kk, idesc,
                                               (kc | kb | kk) != 0);
                    }
                    mma_commit(&empty[s]);
                }
                if (ok) mma_commit(&tfull[acc]);
                if (a.trace && blockIdx.x == 0 && t < (uint64_t)a.trace_tiles)
                    a.trace[t * 4 + 1] = globaltimer();
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(a.err, 2);
            }
            // all issued MMAs complete before TMEM is released
            mma_commit(done);
            volatile int zero = 0;
            mbar_wait(done, qph, globaltimer() + a.drain_ns, &zero);
        }
    } else {
        // ------------------------------------------------ epilogue
        // EPI warps per TMEM lane quadrant: warp w serves the query slots of
        // lanes 32*(w%4).. (replica m / bq of query m % bq) and, of every
        // tile, the CW rows of part (half, replica).
        constexpr int CPH = 4 / EPI;         // 32-row chunks per half at most
        constexpr int NSLOT = TC_BM * EPI;   // list / stage slots
        const int qd = warp & 3;
        const int half = (warp - 2) >> 2;
        const int m = qd * 32 + lane;        // TMEM lane = query slot of the tile
        const int rp = m / a.bq;             // replica (uniform within a warp)
        const int slot = half * TC_BM + m;
        const int qg = qtile * TC_BM + (m - rp * a.bq);
        const int CW = TC_BN / (EPI * a.rep);  // rows of a tile per part (>= 32)
        const int nch = CW / 32;
        const int col0 = (half * a.rep + rp) * CW;
        const bool qvalid = qg < a.nq;
        const float qn = qvalid ? a.qnorm[qg] : 0.f;
        const float qs = (FP8 && qvalid) ? a.qscale[qg] : 1.f;
        const int pg = qvalid ? a.qprog[qg] : -1;
        const bool lazy = a.lazy && *a.lazy;
        const uint32_t *bm = (pg >= 0 && !lazy) ? a.bitmaps + (uint64_t)pg * a.bm_words : nullptr;
        // lazy: the query's range program (AND of per-column intervals and
        // small-integer sets, the encoding of common.cuh) in registers
        int nterm = 0;
        int tcol[PV_RANGE_MAX_TERMS];
        double tlo[PV_RANGE_MAX_TERMS], thi[PV_RANGE_MAX_TERMS];
        if (lazy && pg >= 0) {
            const PredProg pp = a.progs[pg];
            const PredInsn r = a.insns[pp.insn0];
            int ci = r.val0;
            nterm = min(max(r.n, 0), PV_RANGE_MAX_TERMS);
#pragma unroll
            for (int k = 0; k < PV_RANGE_MAX_TERMS; k++) {
                tcol[k] = -1;  // a malformed term admits nothing
                tlo[k] = 1.0;
                thi[k] = 0.0;
                if (k >= nterm || ci < 0 || ci + 2 > a.nconsts) continue;
                const int meta = (int)a.consts[ci];
                const int col = meta & 0xFFFF;
                const bool mask = meta & PV_TERM_MASK;
                if (col < a.ncols && (mask || ci + 3 <= a.nconsts)) {
                    tcol[k] = col | (mask ? PV_TERM_MASK : 0);
                    tlo[k] = a.consts[ci + 1];  // a mask term: its bits
                    thi[k] = mask ? 0.0 : a.consts[ci + 2];
                }
                ci += mask ? 2 : 3;
            }
        }
        // the range program on row `row`: f64 compares, NaN fails (the
        // bitmap kernel's test of the same encoding)
        auto lazy_pass = [&](uint64_t row) -> bool {
            bool ok = true;
#pragma unroll
            for (int k = 0; k < PV_RANGE_MAX_TERMS; k++) {
                if (k >= nterm) break;
                if (tcol[k] < 0) return false;
                const int col = tcol[k] & 0xFFFF;
                const double v = __ldg(a.cols + (uint64_t)col * a.nrows + row);
                if (tcol[k] & PV_TERM_MASK) {
                    const bool in = v >= 0.0 && v < 64.0;
                    const int b = in ? (int)v : 64;
                    const int code = (in && (double)b == v) ? b : 64;
                    const unsigned long long bits =
                        (unsigned long long)__double_as_longlong(tlo[k]);
                    ok = ok && code < 64 && ((bits >> (code & 63)) & 1ull);
                } else {
                    ok = ok && v >= tlo[k] && v <= thi[k];
                }
            }
            return ok;
        };
        // thread-private list, interleaved [KP][NSLOT] so a warp's accesses to
        // the same slot index hit 32 different banks
        uint64_t *L = lists + slot;
#define PV_L(j) L[(size_t)(j) * NSLOT]
        int n = 0;
        uint64_t lmax = KEY_MAX;   // worst kept key once the list is full
        uint64_t thr = qvalid ? KEY_MAX : 0ull;  // admission threshold
        float thr_d = qvalid ? __int_as_float(0x7f800000) : -1.f;  // its distance
        bool ok = true;
        // per-tile words in registers, loaded one tile ahead into the set the
        // previous tile released (two sets, no register moves: a move would
        // wait for the load): predicate words of the 32-row chunks and the
        // grid-wide bound
        auto load_words = [&](uint64_t tt, uint32_t (&w)[CPH], unsigned long long &g) {
            const uint64_t rb = (tile0 + tt * a.tile_step) * TC_BN + col0;
#pragma unroll
            for (int j = 0; j < CPH; j++) {
                if (j >= nch) break;
                const uint64_t r0 = rb + j * 32;
                uint32_t v = 0;
                if (r0 < a.nrows) {
                    v = bm ? __ldg(bm + (r0 >> 5)) : 0xFFFFFFFFu;
                    if (a.nrows - r0 < 32) v &= (1u << (a.nrows - r0)) - 1u;
                }
                w[j] = v;
            }
            g = qvalid ? *((volatile unsigned long long *)(a.tau + qg)) : KEY_MAX;
        };
        // one tile: false when a wait gave up
        auto tile_body = [&](uint64_t t, const uint32_t (&bw)[CPH], unsigned long long gt,
                             uint32_t (&nbw)[CPH], unsigned long long &ngt) -> bool {
            if (t + 1 < ntiles) load_words(t + 1, nbw, ngt);
            const uint64_t T = T0 + t;  // running tile count: barrier phases
            const int acc = (int)(T & 1);
            const uint32_t aph = (uint32_t)((T >> 1) & 1);
            const int ns = (int)(T % TC_NR);
            if (!mbar_wait(&tfull[acc], aph, deadline, abort_flag)) return false;
            if (!mbar_wait(&nfull[ns], (uint32_t)((T / TC_NR) & 1), deadline, abort_flag))
                return false;
            tc_fence_after();
            const bool tr =
                a.trace && blockIdx.x == 0 && slot == 0 && t < (uint64_t)a.trace_tiles;
            if (tr) a.trace[t * 4 + 2] = globaltimer();
            const uint64_t rbase = (tile0 + t * a.tile_step) * TC_BN + col0;
            const float *xnv = snorm + (size_t)ns * TC_NSLOT_F + col0;
            const float *xsv = xnv + TC_BN;
            if (gt < thr) {
                thr = gt;
                thr_d = key_dist(gt);
            }
#pragma unroll
            for (int c = 0; c < CPH; c++) {
                if (c >= nch) break;
                uint32_t r[32];
                tmem_ld_32x32b_x32(tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)acc * TC_BN +
                                       col0 + c * 32,
                                   r);
                tmem_ld_wait();
                // hot loop: distances and a candidate mask only; the rare
                // admissions run below, outside the unrolled code (a negative
                // norm-form value is clamped there)
                uint32_t cmask = 0;
#pragma unroll
                for (int i4 = 0; i4 < 32; i4 += 4) {
                    const float4 xn4 = *(const float4 *)(xnv + c * 32 + i4);
                    float4 xs4 = make_float4(1.f, 1.f, 1.f, 1.f);
                    if (FP8) xs4 = *(const float4 *)(xsv + c * 32 + i4);
                    const float xna[4] = {xn4.x, xn4.y, xn4.z, xn4.w};
                    const float xsa[4] = {xs4.x, xs4.y, xs4.z, xs4.w};
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int i = i4 + u;
                        float dot = __uint_as_float(r[i]);
                        if (FP8) dot *= xsa[u] * qs;
                        const float d = fmaf(-2.f, dot, xna[u] + qn);
                        if (d <= thr_d) {
                            stage[i * NSLOT + slot] = d;
                            cmask |= 1u << i;
                        }
                    }
                }
                cmask &= bw[c];
#pragma unroll 1
                while (cmask) {
                    const int i = __ffs(cmask) - 1;
                    cmask &= cmask - 1;
                    const float d = fmaxf(stage[i * NSLOT + slot], 0.f);
                    const uint64_t row = rbase + c * 32 + i;
                    const uint64_t key = make_key(d, (uint32_t)row);
                    // <= : the seeded bound is itself a row key that this
                    // pass must admit again (keys are unique)
                    if (key > thr) continue;
                    if (lazy && !lazy_pass(row)) continue;
                    // the list is a max-heap (root = worst kept key): an
                    // admission costs O(log KP) shared-memory steps
                    if (n < KP) {
                        int j = n++;
                        while (j > 0) {
                            const int p = (j - 1) >> 1;
                            const uint64_t pv = PV_L(p);
                            if (pv >= key) break;
                            PV_L(j) = pv;
                            j = p;
                        }
                        PV_L(j) = key;
                        if (n < KP) continue;
                    } else {
                        int j = 0;
                        for (;;) {
                            int ch = 2 * j + 1;
                            if (ch >= KP) break;
                            uint64_t cv = PV_L(ch);
                            if (ch + 1 < KP) {
                                const uint64_t c2 = PV_L(ch + 1);
                                if (c2 > cv) {
                                    cv = c2;
                                    ch++;
                                }
                            }
                            if (cv <= key) break;
                            PV_L(j) = cv;
                            j = ch;
                        }
                        PV_L(j) = key;
                    }
                    lmax = PV_L(0);
                    if (lmax < thr) {
                        thr = lmax;
                        thr_d = key_dist(lmax);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
            __syncwarp();
            if (lane == 0) mbar_arrive(&nempty[ns]);
            if (tr) a.trace[t * 4 + 3] = globaltimer();
            if (a.push_tau && qvalid && n == KP && lmax < KEY_MAX) atomicMin(a.tau + qg, lmax);
            return true;
        };
        uint32_t wA[CPH], wB[CPH];
        unsigned long long gA = KEY_MAX, gB = KEY_MAX;
        if (ntiles) load_words(0, wA, gA);
        for (uint64_t t = 0; t < ntiles; t += 2) {
            if (!tile_body(t, wA, gA, wB, gB)) { ok = false; break; }
            if (t + 1 < ntiles && !tile_body(t + 1, wB, gB, wA, gA)) { ok = false; break; }
        }
        if (!ok) {
            *abort_flag = 1;
            atomicExch(a.err, 3);
        }
        if (qvalid) {
            // heap -> ascending list (heapsort in place)
            for (int end = n - 1; end > 0; end--) {
                const uint64_t top = PV_L(0), v = PV_L(end);
                PV_L(end) = top;
                int j = 0;
                for (;;) {
                    int ch = 2 * j + 1;
                    if (ch >= end) break;
                    uint64_t cv = PV_L(ch);
                    if (ch + 1 < end) {
                        const uint64_t c2 = PV_L(ch + 1);
                        if (c2 > cv) {
                            cv = c2;
                            ch++;
                        }
                    }
                    if (cv <= v) break;
                    PV_L(j) = cv;
                    j = ch;
                }
                PV_L(j) = v;
            }
            // the list's best kwrite keys at or below the grid-wide bound join
            // its query's dense run (one atomic per list: keys above the bound
            // cannot be in the answer); a full list reports its last key,
            // below which it cannot have dropped anything
            const unsigned long long bound = *((volatile unsigned long long *)(a.tau + qg));
            int nw = n < a.kwrite ? n : a.kwrite;
            while (nw > 0 && PV_L(nw - 1) > bound) nw--;
            if (nw > 0) {
                const uint64_t b0 = atomicAdd(a.dcnt + qg, (uint32_t)nw);
                uint64_t *dst = a.dense + (uint64_t)qg * a.dcap;
                for (int i = 0; i < nw && b0 + i < a.dcap; i++) dst[b0 + i] = PV_L(i);
            }
            if (a.fullmin && n == KP) atomicMin(a.fullmin + qg, (unsigned long long)PV_L(KP - 1));
        }
#undef PV_L
    }
    run.it = it0 + ntiles * (uint64_t)nkc;
    run.t = T0 + ntiles;
    run.qph++;
    __syncthreads();
    return *abort_flag == 0;
}

}  // namespace pv
