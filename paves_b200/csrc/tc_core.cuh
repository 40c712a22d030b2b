// tc_core.cuh — the tensor-core filtered scan's per-CTA pass, shared by the
// one-shot scan kernel (scan_tc.cu) and the persistent micro-batch kernel.
//
// A pass streams one query tile against a CTA's row tiles:
//     D[128 queries][128 rows] = Q[128 x K] * X_tile[128 x K]^T
// (A = query tile, resident in shared memory; B = row tile, streamed by
// TMA in 128-byte-swizzled K-major boxes), D in TMEM, four buffers, so
// the MMAs of tiles t+1..t+3 overlap the epilogue of tile t. In TMEM, lane =
// query and column = row: each epilogue thread owns ONE query, walks the
// tile's rows and keeps that query's best K' keys in a private
// shared-memory list with its threshold in a register. Row norms (and FP8
// scales) arrive in a shared-memory ring beside the rows; the filter is a
// bitmap word per 32 rows, or, for lazy batches, the query's range program
// evaluated only on rows that beat the threshold.
//
// Warp roles (64 + 128 * EPI threads): warp 0 TMA producer, warp 1 MMA
// issuer, then EPI groups of 4 epilogue warps (warp w reads TMEM lanes
// 32*(w%4).. ; group h owns the tiles h, h + EPI, ...). A batch of at
// most 64 (32) queries is replicated 2 (4) times down the 128 query slots.
// All waits are bounded by a deadline and unwind through an abort flag.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

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
// words per norm slot: norms, fp8 scales, then the index rows of a
// compacted row set (each part one tile's 128 entries)
constexpr int TC_NSLOT_F = 3 * TC_BN;
// TMEM accumulators (128 columns each, all 512 of the SM's): the MMA of a
// tile waits only for the epilogue of the tile NACC back, so the MMA's own
// latency (issue to completion ~1 us for a BF16 tile) overlaps up to three
// epilogues instead of one
constexpr int TC_NACC = 4;
constexpr uint32_t TC_TMEM_COLS = TC_NACC * TC_BN;

// Operand kinds of a pass: rows and queries as BF16, FP8-E4M3 (per-row and
// per-query scales) or the f32 rows themselves read as TF32.
constexpr int TCK_BF16 = 0;
constexpr int TCK_FP8 = 1;
constexpr int TCK_TF32 = 2;
__host__ __device__ constexpr int tck_esz(int kind) {
    return kind == TCK_FP8 ? 1 : kind == TCK_TF32 ? 4 : 2;
}

template <int KIND>
__device__ __forceinline__ void mma_kind(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t acc) {
    if (KIND == TCK_FP8) mma_f8(d, a, b, idesc, acc);
    else if (KIND == TCK_TF32) mma_tf32(d, a, b, idesc, acc);
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
    // rows scanned are a compacted set: scanned row i is index row rowids[i]
    // (padded to whole tiles; keys carry the index row), of which the first
    // *nrows_dev exist (tiles past them are skipped); null: the index's rows
    const uint32_t *__restrict__ rowids;
    const unsigned long long *nrows_dev;
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

// staged: the candidate staging slots exist (every kind but TF32, whose
// admissions re-read the accumulator registers; its 32-32 KB go to stages)
__device__ __forceinline__ TcSmem tc_carve(unsigned char *base, int KBt, int NS, int KPcap,
                                           int EPI, bool staged = true) {
    TcSmem m;
    m.sQ = base;                                       // KBt boxes
    m.sX = m.sQ + (size_t)KBt * TC_BOX;                // NS stages
    // a stage holds one K-chunk of a row tile: min(TC_KBS, KBt) boxes
    m.SB = (size_t)(KBt < TC_KBS ? KBt : TC_KBS) * TC_BOX;
    // per (query, part) lists [KP][128*EPI] and candidate staging [32][128*EPI]
    m.lists = (uint64_t *)(m.sX + (size_t)NS * m.SB);
    m.stage = (float *)(m.lists + (size_t)TC_BM * EPI * KPcap);
    // row norms (and fp8 scales, compacted-set row ids) of a tile, TC_NR
    // tiles in flight (slot = [norms 128][scales 128][row ids 128])
    m.snorm = m.stage + (staged ? 32 * TC_BM * EPI : 0);
    if (!staged) m.stage = nullptr;
    uint64_t *bars = (uint64_t *)(m.snorm + (size_t)TC_NR * TC_NSLOT_F);
    m.full = bars;              // [NS]
    m.empty = m.full + NS;      // [NS]
    m.tfull = m.empty + NS;           // [TC_NACC]
    m.tempty = m.tfull + TC_NACC;     // [TC_NACC]
    m.qbar = m.tempty + TC_NACC;      // [1]
    m.done = m.qbar + 1;        // [1]
    m.nfull = m.done + 1;       // [TC_NR]
    m.nempty = m.nfull + TC_NR; // [TC_NR]
    return m;
}

inline size_t tc_smem_bytes(int kblocks, int NS, int KPcap, int EPI, bool staged = true) {
    return 1024 + (size_t)kblocks * TC_BOX +
           (size_t)NS * (kblocks < TC_KBS ? kblocks : TC_KBS) * TC_BOX +
           (size_t)TC_BM * EPI * KPcap * 8 + (staged ? (size_t)32 * TC_BM * EPI * 4 : 0) +
           (size_t)TC_NR * TC_NSLOT_F * 4 + (size_t)(2 * NS + 2 * TC_NACC + 2 + 2 * TC_NR) * 8;
}

// by one thread, before the CTA's first pass
__device__ __forceinline__ void tc_init_barriers(const TcSmem &m, int NS, int EPI) {
    for (int i = 0; i < NS; i++) {
        mbar_init(&m.full[i], 1);
        mbar_init(&m.empty[i], 1);
    }
    for (int i = 0; i < TC_NACC; i++) {
        mbar_init(&m.tfull[i], 1);
        mbar_init(&m.tempty[i], TC_BM);  // the epilogue group that owns the tile
    }
    for (int i = 0; i < TC_NR; i++) {
        mbar_init(&m.nfull[i], 1);
        mbar_init(&m.nempty[i], 4);  // one arrival per warp of the owning group
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
// WARM: compile the warm-up admission bound (passes that start without a
// bound: seeding passes, compacted sets; it costs the main pass over the
// whole index ~7 % in registers and code for nothing, so that one omits it)
template <int KIND, int EPI, bool WARM = false>
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
    constexpr bool FP8 = KIND == TCK_FP8;
    constexpr int BOXE = TC_KB_BYTES / tck_esz(KIND);  // elements of K per box
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // this CTA's tiles: tile0 + t * tile_step, t < ntiles
    const uint64_t tile0 = (uint64_t)rgrp * a.tile0_mul;
    uint64_t nrows_eff = a.nrows;
    if (a.nrows_dev) {
        const unsigned long long nd = *a.nrows_dev;
        if (nd < nrows_eff) nrows_eff = nd;
    }
    const uint64_t ntiles_all = (nrows_eff + TC_BN - 1) / TC_BN;
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
                tma_load_2d(sQ + (size_t)kb * TC_BOX, &tmQ, kb * BOXE,
                            qtile * TC_BM, qbar);
            const uint32_t nbytes = ((FP8 ? 2 : 1) + (a.rowids ? 1 : 0)) * TC_BN * 4;
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
                    if (a.rowids)
                        bulk_load(dst + 2 * TC_BN, a.rowids + tile * TC_BN, TC_BN * 4, &nfull[ns]);
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
                                    (kc * TC_KBS + kb) * BOXE, y, &full[s]);
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
                                   : KIND == TCK_TF32 ? idesc_make(FMT_TF32, FMT_TF32, TC_BM, TC_BN)
                                                      : idesc_make(FMT_BF16, FMT_BF16, TC_BM, TC_BN);
            bool ok = mbar_wait(qbar, qph, deadline, abort_flag);
            uint64_t it = it0;
            for (uint64_t t = 0; t < ntiles && ok; t++) {
                const uint64_t T = T0 + t;
                const int acc = (int)(T % TC_NACC);
                const uint32_t aph = (uint32_t)((T / TC_NACC) & 1);
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
                            mma_kind<KIND>(dcol, ad + 2 * kk, bd + 2 * kk, idesc,
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
        // EPI groups of 4 warps; warp w serves the query slots of TMEM lanes
        // 32*(w%4).. (replica m / bq of query m % bq). Group h owns the tiles
        // whose running number T has T % EPI == h, so each group pays a
        // tile's fixed costs (barrier waits, word loads, arrivals) once per
        // EPI tiles, and takes the CW rows of its replica from each of them.
        constexpr int CPH = TC_BN / 32;      // 32-row chunks per part at most
        constexpr int NSLOT = TC_BM * EPI;   // list / stage slots
        const int qd = warp & 3;
        const int half = (warp - 2) >> 2;
        const int m = qd * 32 + lane;        // TMEM lane = query slot of the tile
        const int rp = m / a.bq;             // replica (uniform within a warp)
        const int slot = half * TC_BM + m;
        const int qg = qtile * TC_BM + (m - rp * a.bq);
        const int CW = TC_BN / a.rep;  // rows of a tile per replica (>= 32)
        const int nch = CW / 32;
        const int col0 = rp * CW;
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
        uint64_t pushed = KEY_MAX; // last key this list pushed to the grid-wide bound
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
            if (t + EPI < ntiles) load_words(t + EPI, nbw, ngt);
            const uint64_t T = T0 + t;  // running tile count: barrier phases
            const int acc = (int)(T % TC_NACC);
            const uint32_t aph = (uint32_t)((T / TC_NACC) & 1);
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
            const uint32_t *ridv = (const uint32_t *)(xnv + 2 * TC_BN);
            if (gt < thr) {
                thr = gt;
                thr_d = key_dist(gt);
            }
            // one 32-row chunk of the tile, its accumulator columns in r
            auto chunk = [&](const int c, const uint32_t(&r)[32]) {
                // hot loop: distances and a candidate mask only; the rare
                // admissions run below, outside the unrolled code (a negative
                // norm-form value is clamped there). They take a candidate's
                // distance from the staging slots, or, in a TF32 pass, again
                // from the accumulator registers (the same operations on the
                // same values: the same bits), whose freed shared memory
                // holds a third stage of its 512-byte rows: measured at batch
                // 64 the TF32 pass ran 0.098 vs 0.102 ms; the BF16 pass the
                // same way ran 0.069 vs 0.064 ms (its accumulators stay live
                // through the admissions: 144 registers instead of 128, and
                // more stages did not help it)
                constexpr bool RECOMP = KIND == TCK_TF32;
                auto dist_of = [&](const int i, const uint32_t acc_bits) -> float {
                    float dot = __uint_as_float(acc_bits);
                    if (FP8) dot *= xsv[c * 32 + i] * qs;
                    return fmaf(-2.f, dot, xnv[c * 32 + i] + qn);
                };
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
                            if (!RECOMP) stage[i * NSLOT + slot] = d;
                            cmask |= 1u << i;
                        }
                    }
                }
                cmask &= bw[c];
                // warm-up: an empty list facing more than KP candidates (a
                // pass without a bound: the first chunk of a compacted set,
                // of a seeding pass) admits only the chunk's KP best - the
                // KP-th smallest distance becomes the admission bound -
                // instead of inserting every candidate into its heap one by
                // one (the bound: ascending distinct values, counting ties)
                if (WARM && !lazy && n == 0 && __popc(cmask) > KP) {
                    float v[32];
#pragma unroll
                    for (int i = 0; i < 32; i++)
                        v[i] = ((cmask >> i) & 1u)
                                   ? fmaxf(RECOMP ? dist_of(i, r[i]) : stage[i * NSLOT + slot], 0.f)
                                   : __int_as_float(0x7f800000);
                    float kth = -1.f;
                    for (int cnt = 0; cnt < KP;) {
                        float m = __int_as_float(0x7f800000);
#pragma unroll
                        for (int i = 0; i < 32; i++)
                            if (v[i] > kth) m = fminf(m, v[i]);
                        int c2 = 0;
#pragma unroll
                        for (int i = 0; i < 32; i++) c2 += v[i] == m ? 1 : 0;
                        kth = m;
                        cnt += c2;
                    }
                    if (kth < thr_d) thr_d = kth;
#pragma unroll
                    for (int i = 0; i < 32; i++)
                        if (v[i] > thr_d) cmask &= ~(1u << i);
                }
#pragma unroll 1
                while (cmask) {
                    const int i = __ffs(cmask) - 1;
                    cmask &= cmask - 1;
                    float dv;
                    if (RECOMP) {
                        uint32_t bits = 0;
#pragma unroll
                        for (int j = 0; j < 32; j++)
                            if (j == i) bits = r[j];
                        dv = dist_of(i, bits);
                    } else {
                        dv = stage[i * NSLOT + slot];
                    }
                    const float d = fmaxf(dv, 0.f);
                    const uint64_t row = rbase + c * 32 + i;
                    const uint32_t rid = a.rowids ? ridv[c * 32 + i] : (uint32_t)row;
                    const uint64_t key = make_key(d, rid);
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
            };
            // (loading two chunks before one wait measured slower: 0.0644 vs
            // 0.0615 ms for the BF16 pass at batch 64)
            const uint32_t tbase =
                tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)acc * TC_BN + col0;
#pragma unroll
            for (int c = 0; c < CPH; c++) {
                if (c >= nch) break;
                uint32_t r0[32];
                tmem_ld_32x32b_x32(tbase + c * 32, r0);
                tmem_ld_wait();
                chunk(c, r0);
            }
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
            __syncwarp();
            if (lane == 0) mbar_arrive(&nempty[ns]);
            if (tr) a.trace[t * 4 + 3] = globaltimer();
            // a full list's last key bounds the grid-wide bound; pushed only
            // when it improved (all lists of a query push to one word)
            if (a.push_tau && qvalid && n == KP && lmax < pushed) {
                atomicMin(a.tau + qg, lmax);
                pushed = lmax;
            }
            return true;
        };
        uint32_t wA[CPH], wB[CPH];
        unsigned long long gA = KEY_MAX, gB = KEY_MAX;
        // this group's first tile of the pass
        const uint64_t tfirst = (uint64_t)((half - (int)(T0 % EPI) + EPI) % EPI);
        if (tfirst < ntiles) load_words(tfirst, wA, gA);
        for (uint64_t t = tfirst; t < ntiles; t += 2 * EPI) {
            if (!tile_body(t, wA, gA, wB, gB)) { ok = false; break; }
            if (t + EPI < ntiles && !tile_body(t + EPI, wB, gB, wA, gA)) { ok = false; break; }
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

// ---- per-query steps after a pass (kernels in scan_tc.cu wrap them)

// one warp: query row qi of the tile (qi < nqpad)
__device__ __forceinline__ void query_prep_row(int qi, int lane, const float *__restrict__ q,
                                               int nq, int dpad, int dim, int bq, int kelems,
                                               int kind, unsigned char *__restrict__ out,
                                               float *__restrict__ qnorm,
                                               float *__restrict__ qscale,
                                               unsigned long long *__restrict__ tau,
                                               uint32_t *__restrict__ dcnt,
                                               unsigned long long *__restrict__ fullmin,
                                               int *__restrict__ err) {
    if (lane == 0 && qi < nq) {
        tau[qi] = KEY_MAX;
        dcnt[qi] = 0;
        if (fullmin) fullmin[qi] = KEY_MAX;
        if (qi == 0) *err = 0;
    }
    const int src = qi % bq;
    const bool ok = src < nq;
    const bool fp8 = kind == TCK_FP8;
    float amax = 0.f;
    if (fp8 && ok)
        for (int j = lane; j < dim; j += 32) amax = fmaxf(amax, fabsf(q[(size_t)src * dpad + j]));
    for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const float s = amax > 0.f ? amax / 448.f : 1.f;
    float acc = 0.f;
    for (int j = lane; j < kelems; j += 32) {
        const float v = (ok && j < dim) ? q[(size_t)src * dpad + j] : 0.f;
        float r;
        if (fp8) {
            __nv_fp8_e4m3 b(v / s);
            out[(size_t)qi * kelems + j] = *(unsigned char *)&b;
            r = float(b) * s;
        } else if (kind == TCK_TF32) {
            // the f32 value itself (the MMA reads its tf32 part); the norm
            // is the exact row's
            ((float *)out)[(size_t)qi * kelems + j] = v;
            r = v;
        } else {
            __nv_bfloat16 b = __float2bfloat16_rn(v);
            ((__nv_bfloat16 *)out)[(size_t)qi * kelems + j] = b;
            r = __bfloat162float(b);
        }
        acc = fmaf(r, r, acc);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        qnorm[qi] = acc;
        if (qscale) qscale[qi] = s;
    }
}

// The numerical certificate of a re-ranked superset whose scan distances
// were inexact (f32 rows read as TF32): qnorm = null turns it off.
//
// A row outside the superset has scan key >= the superset's last key A
// (the merge kept the S smallest keys), so its scan distance is >= A, and
// its exact distance exceeds the answer's last exact distance Dk if
//     (A - E) * (1 - c2) > Dk,
// E bounding |scan distance - true distance| and c2 the relative error of
// the f32 difference-form sum (the exact distance) against the true one:
//   * the MMA reads each f32 operand with its low 13 mantissa bits
//     dropped, a relative change below 2^-10 per operand, so each product
//     moves by at most (2^-9 + 2^-20) |x_i| |q_i|; the f32 accumulation in
//     the tensor core adds at most about dim * 2^-22 of sum |x_i q_i|; and
//     sum |x_i| |q_i| <= ||x|| ||q|| (Cauchy-Schwarz), with ||x||^2 at most
//     xnmax over all rows;
//   * the f32 norms (dim terms) and the two roundings of ||x||^2 + ||q||^2
//     - 2 q.x stay within c2 = (dim + 8) * 2^-23 of the values they round.
// E = 1.25 * 2^-8 ||q|| sqrt(xnmax) (1 + c2) + c2 (xnmax + ||q||^2 + A)
// covers both terms with a margin (the first has 2^-8 * 1.25 against the
// 2^-8 + 2^-19 + dim * 2^-21 the analysis needs for dim <= 128). Queries
// that fail are flagged in unc[] for an exact re-run.
struct RerankCert {
    const float *qnorm = nullptr;  // [nq] ||q||^2 (f32)
    float xnmax = 0.f;             // max ||x||^2 over the rows (f32 norms)
    int dim = 0;
    uint8_t *unc = nullptr;        // [nq] set to 1 when not certified
};

// One query's re-rank by the block's NT threads (8 lanes per candidate,
// NT / 8 in flight); keys: TC_MAX_SUPERSET slots of shared memory. Ends
// with the block synchronized.
template <int NT>
__device__ __forceinline__ void rerank_query(int q, uint64_t *keys, const float *__restrict__ vecs,
                                             int dpad, const float *__restrict__ queries,
                                             const FvHit *__restrict__ cand,
                                             const uint32_t *__restrict__ cand_cnt, int S,
                                             uint32_t topb, const int32_t *__restrict__ qprog,
                                             const unsigned long long *__restrict__ popcnt,
                                             uint64_t nrows, FvHit *__restrict__ out,
                                             uint32_t *__restrict__ out_cnt,
                                             uint8_t *__restrict__ trunc,
                                             const RerankCert cert = RerankCert()) {
    const int tid = threadIdx.x;
    const int grp = tid >> 3, sub = tid & 7;
    const int ncand = (int)cand_cnt[q];
    int n = ncand;
    if (n > S) n = S;
    const float *qv = queries + (size_t)q * dpad;
    for (int base = 0; base < n; base += NT / 8) {
        const int j = base + grp;
        const bool ok = j < n;
        const uint32_t row = (uint32_t)cand[(size_t)q * S + (ok ? j : 0)].node;
        const float *x = vecs + (size_t)row * dpad;
        float acc = 0.f;
        for (int k = sub * 4; k < dpad; k += 32) {
            const float4 v = __ldg((const float4 *)(x + k));
            const float4 w = __ldg((const float4 *)(qv + k));
            const float d0 = v.x - w.x, d1 = v.y - w.y, d2 = v.z - w.z, d3 = v.w - w.w;
            acc = fmaf(d0, d0, acc);
            acc = fmaf(d1, d1, acc);
            acc = fmaf(d2, d2, acc);
            acc = fmaf(d3, d3, acc);
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        if (ok && sub == 0) keys[j] = make_key(acc, row);
    }
    int n2 = 1;
    while (n2 < n) n2 <<= 1;
    for (int i = n + tid; i < n2; i += blockDim.x) keys[i] = KEY_MAX;
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < (n2 >> 1); i += blockDim.x) {
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo | j;
                const uint64_t x = keys[lo], y = keys[hi];
                if ((x > y) == ((lo & k) == 0)) {
                    keys[lo] = y;
                    keys[hi] = x;
                }
            }
            __syncthreads();
        }
    }
    const int nout = n < (int)topb ? n : (int)topb;
    for (int i = tid; i < nout; i += blockDim.x) {
        FvHit h;
        h.node = key_row(keys[i]);
        h.dist = key_dist(keys[i]);
        out[(size_t)q * topb + i] = h;
    }
    if (tid == 0) {
        out_cnt[q] = (uint32_t)nout;
        const int pg = qprog[q];
        const unsigned long long passing = pg >= 0 ? popcnt[pg] : nrows;
        trunc[q] = passing > (unsigned long long)topb ? 1 : 0;
        // a superset short of S holds every row that can pass: nothing to certify
        if (cert.qnorm && ncand >= S && nout == (int)topb) {
            const double A = (double)cand[(size_t)q * S + (S - 1)].dist;
            const double Dk = (double)key_dist(keys[nout - 1]);
            const double qn = (double)cert.qnorm[q], xm = (double)cert.xnmax;
            const double c2 = (double)(cert.dim + 8) * 0x1p-23;
            const double E = 1.25 * 0x1p-8 * sqrt(qn * xm) * (1.0 + c2) + c2 * (xm + qn + A);
            if (!((A - E) * (1.0 - c2) > Dk)) cert.unc[q] = 1;
        }
    }
    __syncthreads();
}

constexpr int DM_THREADS = 512;
constexpr int DM_CAP_MAX = 24576;   // largest shared-memory stage
constexpr int DM_OUT = TC_MAX_SUPERSET;

__device__ __forceinline__ void dm_hist_add(unsigned *hist, bool act, unsigned d, int lane) {
    const int tag = act ? (int)d : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, tag);
    if (act && lane == __ffs(peers) - 1) atomicAdd(&hist[d], (unsigned)__popc(peers));
}

// One query's merge (radix select, any KO <= DM_OUT) by all threads of the
// block; smem_keys: stage_cap + DM_OUT keys of shared memory. Ends with the
// block synchronized.
static __device__ __noinline__ void dense_merge_query(
    int q, uint64_t *smem_keys, const uint64_t *__restrict__ dense, uint64_t dcap, int stage_cap,
    uint32_t *__restrict__ dcnt, int reset_cnt, const unsigned long long *__restrict__ fullmin,
    const unsigned long long *tau, int KO, const int32_t *__restrict__ qprog,
    const unsigned long long *__restrict__ popcnt, uint64_t nrows, FvHit *__restrict__ out,
    uint32_t *__restrict__ out_cnt, uint8_t *__restrict__ trunc, unsigned long long *tau_out,
    uint8_t *__restrict__ unc) {
    uint64_t *buf = smem_keys;        // [stage_cap] staged keys
    uint64_t *res = buf + stage_cap;  // [DM_OUT] the answer, sorted
    __shared__ unsigned hist[256];
    __shared__ int s_m, s_c, s_digit, s_rank, s_tot;
    const int NW = blockDim.x >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned long long bound = tau ? tau[q] : KEY_MAX;
    uint64_t n = dcnt[q];
    if (n > dcap) n = dcap;
    const uint64_t *src = dense + (uint64_t)q * dcap;
    if (tid == 0) {
        s_m = 0;
        s_c = 0;
    }
    __syncthreads();
    if (reset_cnt && tid == 0) dcnt[q] = 0;  // every thread has read it
    const bool staged = n <= (uint64_t)stage_cap;
    if (staged) {
        for (uint64_t b = (uint64_t)warp * 32; b < n; b += NW * 32) {
            const uint64_t i = b + lane;
            const uint64_t key = i < n ? src[i] : KEY_MAX;
            const bool keep = i < n && key <= bound;
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            int base = 0;
            if (lane == 0 && bal) base = atomicAdd(&s_m, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (keep) buf[base + __popc(bal & ((1u << lane) - 1u))] = key;
        }
    }
    __syncthreads();
    // candidates: buf[0, s_m) if staged, else the keys <= bound of src[0, n)
    const uint64_t N = staged ? (uint64_t)s_m : n;
    uint64_t kth = KEY_MAX;  // keep every candidate unless there are more than KO
    if (!staged || s_m > KO) {
        uint64_t prefix = 0;
        int rank = KO;
        bool selected = true;
        for (int pass = 0; pass < 8; pass++) {
            const int shift = 56 - 8 * pass;
            for (int i = tid; i < 256; i += (int)blockDim.x) hist[i] = 0;
            __syncthreads();
            for (uint64_t b = (uint64_t)warp * 128; b < N; b += NW * 128) {
                uint64_t key[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const uint64_t i = b + u * 32 + lane;
                    key[u] = i < N ? (staged ? buf[i] : src[i]) : KEY_MAX;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    bool act = b + u * 32 + lane < N && (staged || key[u] <= bound);
                    if (pass > 0) act = act && (key[u] >> (shift + 8)) == (prefix >> (shift + 8));
                    dm_hist_add(hist, act, (unsigned)(key[u] >> shift) & 255u, lane);
                }
            }
            __syncthreads();
            if (warp == 0) {
                unsigned c[8], sum = 0;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    c[j] = hist[lane * 8 + j];
                    sum += c[j];
                }
                unsigned incl = sum;
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const unsigned excl = incl - sum;
                if (pass == 0 && lane == 31) s_tot = (int)incl;
                if (excl < (unsigned)rank && (unsigned)rank <= incl) {
                    unsigned cum = excl;
                    int j = 0;
                    for (; j < 7; j++) {
                        if (cum + c[j] >= (unsigned)rank) break;
                        cum += c[j];
                    }
                    s_digit = lane * 8 + j;
                    s_rank = rank - (int)cum;
                }
            }
            __syncthreads();
            if (pass == 0 && s_tot <= KO) {  // no more than KO candidates
                selected = false;
                break;
            }
            prefix |= (uint64_t)s_digit << shift;
            rank = s_rank;
        }
        if (selected) kth = prefix;
    }
    // the answer: candidates <= kth (exactly min(count, KO) keys)
    for (uint64_t b = (uint64_t)warp * 128; b < N; b += NW * 128) {
        uint64_t key[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t i = b + u * 32 + lane;
            key[u] = i < N ? (staged ? buf[i] : src[i]) : KEY_MAX;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const bool keep = b + u * 32 + lane < N && key[u] <= bound && key[u] <= kth;
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            int base = 0;
            if (lane == 0 && bal) base = atomicAdd(&s_c, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            const int pos = base + __popc(bal & ((1u << lane) - 1u));
            if (keep && pos < DM_OUT) res[pos] = key[u];
        }
    }
    __syncthreads();
    const int c = min(min(s_c, KO), DM_OUT);
    int n2 = 1;
    while (n2 < c) n2 <<= 1;
    for (int i = c + tid; i < n2; i += (int)blockDim.x) res[i] = KEY_MAX;
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < (n2 >> 1); i += (int)blockDim.x) {
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo | j;
                const uint64_t x = res[lo], y = res[hi];
                if ((x > y) == ((lo & k) == 0)) {
                    res[lo] = y;
                    res[hi] = x;
                }
            }
            __syncthreads();
        }
    }
    for (int i = tid; i < c; i += (int)blockDim.x) {
        FvHit h;
        h.node = (uint64_t)key_row(res[i]);
        h.dist = key_dist(res[i]);
        out[(uint64_t)q * KO + i] = h;
    }
    if (tid == 0) {
        out_cnt[q] = (uint32_t)c;
        const int pg = qprog[q];
        const unsigned long long passing = pg >= 0 ? popcnt[pg] : nrows;
        trunc[q] = passing > (unsigned long long)KO ? 1 : 0;
        // the KO-th merged key bounds the KO-th key of any superset of rows
        if (tau_out && c == KO && res[KO - 1] < tau_out[q]) tau_out[q] = res[KO - 1];
        if (unc) {
            // a full list whose last key is at or below the answer's last key
            // (or the bound while the answer is short) may have dropped a
            // member of it
            const unsigned long long lim = c == KO ? res[KO - 1] : bound;
            const unsigned long long fm = fullmin ? fullmin[q] : KEY_MAX;
            unc[q] = (fm != KEY_MAX && fm <= lim) ? 1 : 0;
        }
    }
    __syncthreads();
}

// The same for KO <= 32, without block barriers in the hot loop: each warp
// keeps its 32 best keys sorted across its lanes (one key per lane) and
// folds in 32 new keys at a time (a shuffle bitonic sort of the new keys in
// descending order, an elementwise min with the list, which leaves the 32
// smallest as a bitonic sequence, and a bitonic clean back to ascending);
// a batch none of whose keys beats the list's last key is skipped. The
// warps' lists then fold pairwise into warp 0's.
__device__ __forceinline__ uint64_t warp_sort32(uint64_t x, int lane, bool descending) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint64_t o = __shfl_xor_sync(0xffffffffu, x, j);
            const bool up = ((lane & k) == 0) != descending;
            const bool lower = (lane & j) == 0;
            x = (lower == up) ? (x < o ? x : o) : (x > o ? x : o);
        }
    return x;
}

__device__ __forceinline__ uint64_t warp_clean32(uint64_t x, int lane) {
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, x, j);
        x = (lane & j) == 0 ? (x < o ? x : o) : (x > o ? x : o);
    }
    return x;
}

// One query's merge for KO <= 32 by all threads of the block (any whole
// number of warps); lists: one 32-key slot per warp in shared memory.
// Ends with the block synchronized.
__device__ __forceinline__ void dense_top32_query(
    int q, uint64_t (*lists)[32], const uint64_t *__restrict__ dense, uint64_t dcap,
    uint32_t *__restrict__ dcnt, int reset_cnt, const unsigned long long *__restrict__ fullmin,
    const unsigned long long *tau, int KO, const int32_t *__restrict__ qprog,
    const unsigned long long *__restrict__ popcnt, uint64_t nrows, FvHit *__restrict__ out,
    uint32_t *__restrict__ out_cnt, uint8_t *__restrict__ trunc, unsigned long long *tau_out,
    uint8_t *__restrict__ unc, long long passing_pre = -1) {
    const int NW = blockDim.x >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned long long bound = tau ? tau[q] : KEY_MAX;
    uint64_t n = dcnt[q];
    if (n > dcap) n = dcap;
    const uint64_t *src = dense + (uint64_t)q * dcap;
    __syncthreads();
    if (reset_cnt && tid == 0) dcnt[q] = 0;  // every thread has read it
    uint64_t best = KEY_MAX;  // ascending across the lanes
    for (uint64_t b = (uint64_t)warp * 64; b < n; b += NW * 64) {
        uint64_t k2[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint64_t i = b + u * 32 + lane;
            k2[u] = i < n ? src[i] : KEY_MAX;
            if (k2[u] > bound) k2[u] = KEY_MAX;
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint64_t worst = __shfl_sync(0xffffffffu, best, 31);
            if (!__any_sync(0xffffffffu, k2[u] < worst)) continue;
            const uint64_t d = warp_sort32(k2[u], lane, true);
            best = warp_clean32(best < d ? best : d, lane);
        }
    }
    // the warps' lists fold pairwise, log2(NW) rounds (warp w takes in
    // warp w + step's list, read descending, while w is a multiple of 2 step)
    lists[warp][lane] = best;
    for (int step = 1; step < NW; step <<= 1) {
        __syncthreads();
        if ((warp & (2 * step - 1)) == 0 && warp + step < NW) {
            const uint64_t d = lists[warp + step][31 - lane];
            const uint64_t m = best < d ? best : d;
            if (__any_sync(0xffffffffu, m != best)) {
                best = warp_clean32(m, lane);
                lists[warp][lane] = best;
            }
        }
    }
    if (warp == 0) {
        const bool have = lane < KO && best != KEY_MAX;
        const int c = __popc(__ballot_sync(0xffffffffu, have));
        if (have) {
            FvHit h;
            h.node = (uint64_t)key_row(best);
            h.dist = key_dist(best);
            out[(uint64_t)q * KO + lane] = h;
        }
        const uint64_t last = __shfl_sync(0xffffffffu, best, KO - 1);
        if (lane == 0) {
            out_cnt[q] = (uint32_t)c;
            unsigned long long passing = (unsigned long long)passing_pre;
            if (passing_pre < 0) {
                const int pg = qprog[q];
                passing = pg >= 0 ? popcnt[pg] : nrows;
            }
            trunc[q] = passing > (unsigned long long)KO ? 1 : 0;
            if (tau_out && c == KO && last < tau_out[q]) tau_out[q] = last;
            if (unc) {
                const unsigned long long lim = c == KO ? last : bound;
                const unsigned long long fm = fullmin ? fullmin[q] : KEY_MAX;
                unc[q] = (fm != KEY_MAX && fm <= lim) ? 1 : 0;
            }
        }
    }
    __syncthreads();
}

// host: a 2-D tensor map over [rows][inner] elements of operand kind `kind`
// with 128-byte swizzled boxes of [128 rows][128 bytes] (false if encoding
// failed)
bool tc_make_tmap(CUtensorMap *m, const void *ptr, int kind, uint64_t inner, uint64_t rows);

}  // namespace pv
