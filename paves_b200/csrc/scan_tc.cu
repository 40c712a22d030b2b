// scan_tc.cu — reduced-precision filtered L2 scan on the 5th-gen tensor
// cores (tcgen05, TMEM accumulators, TMA-fed shared memory).
//
// New path beside the exact scan (the reference has no tensor-core path;
// its approximate SQ8 scan is gpu_engine.cu:759-893 + rerank :934-992).
// Distances use the norm form ||x||^2 + ||q||^2 - 2 q.x with the dot
// products from one GEMM per 128-row tile:
//     D[128 queries][128 rows] = Q[128 x K] * X_tile[128 x K]^T
// (A = query tile, resident in shared memory; B = row tile, streamed by
// TMA in 128-byte-swizzled K-major boxes). D lives in TMEM in four
// buffers, so the MMAs of the next tiles overlap the epilogue of tile t.
// In TMEM, lane = query and column = row: each epilogue thread owns ONE
// query, walks the tile's 128 rows and keeps that query's best K' keys
// in a private shared-memory list with its threshold in a register; the
// bitmap predicate is read only for rows that beat the threshold. The
// grid-wide per-query bound in global memory lets CTAs prune with each
// other's K'-th key. Per-CTA lists are merged per query and the K'
// survivors re-ranked with exact FP32 distances (rerank_kernel).
//
// BF16 operands are exact for integers up to 256, so on integer-valued
// rows (the benchmark data) every distance is exact; FP8-E4M3 rows carry a
// per-row scale (absmax / 448) and the query a per-query scale.
//
// Warp roles (64 + 128 * EPI threads): warp 0 TMA producer, warp 1 TMEM
// allocator + MMA issuer, then EPI groups of 4 epilogue warps (warp w reads
// TMEM lanes 32*(w%4)..+31; group h owns the tiles h, h + EPI, ...).
// A batch of at most 64 (32) queries is replicated 2 (4) times down the
// 128 query slots of the A tile: the MMA costs the same, and each replica
// takes a disjoint share of every tile's rows, so the epilogue work per
// warp shrinks by the replication factor and all four SM sub-partitions
// work (without it the warps of the padding lanes idle).
// All waits are bounded by a deadline and unwind through an abort flag.
#include <algorithm>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "pv_internal.h"
#include "sm100.cuh"
#include "launch.cuh"
#include "tc_core.cuh"

namespace pv {

using namespace sm100;

template <int KIND, int EPI, bool WARM>
__global__ void __launch_bounds__(64 + 128 * EPI, 1)
scan_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmQ,
               TcArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled operand tiles
    unsigned char *base = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const TcSmem sm = tc_carve(base, a.kblocks, a.NS, a.KP, EPI, KIND != TCK_TF32);
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_abort = 0;
        tc_init_barriers(sm, a.NS, EPI);
    }
    if (warp == 1) {
        tmem_alloc(&s_tmem, TC_TMEM_COLS);
        tmem_relinquish();
    }
    __syncthreads();
    tc_fence_after();
    pdl_wait();  // the previous kernel's outputs (query tile, bounds, bitmaps)
    pdl_trigger();
    TcRun run;
    tc_pass<KIND, EPI, WARM>(&tmX, &tmQ, a, sm, s_tmem, run, &s_abort, blockIdx.x % a.qtiles,
                      blockIdx.x / a.qtiles);
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(s_tmem, TC_TMEM_COLS);
    }
}

}  // namespace pv

namespace pv {

// ---------------------------------------------------------------- queries
// f32 queries [nq][dpad] -> low-precision tile rows [nqpad][row_bytes] with
// zero padding, plus ||q||^2 of the rounded query (and the fp8 scale).
// Row qi holds query qi % bq (bq = nqpad without replication). Also resets
// the scan's per-query state for query qi < nq: bound tau (none), dense run
// count, full-list minimum (if tracked), and the watchdog word.
__global__ void query_prep_kernel(const float *__restrict__ q, int nq, int dpad, int dim,
                                  int nqpad, int bq, int kelems, int kind,
                                  unsigned char *__restrict__ out, float *__restrict__ qnorm,
                                  float *__restrict__ qscale, unsigned long long *__restrict__ tau,
                                  uint32_t *__restrict__ dcnt,
                                  unsigned long long *__restrict__ fullmin, int *__restrict__ err,
                                  int behind_bitmaps) {
    // behind_bitmaps: the kernel ahead is this batch's bitmap kernel, which
    // touches nothing this one reads or writes (the queries were copied
    // before it), so the work runs beside it and only the completion waits
    if (!behind_bitmaps) {
        pdl_wait();
        pdl_trigger();
    }
    const int qi = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (qi < nqpad)
        query_prep_row(qi, threadIdx.x & 31, q, nq, dpad, dim, bq, kelems, kind, out, qnorm,
                       qscale, tau, dcnt, fullmin, err);
    if (behind_bitmaps) {
        pdl_wait();
        pdl_trigger();
    }
}

// ---------------------------------------------------------------- re-rank
// Exact FP32 distances (difference form) for each query's merged candidates
// (up to TC_MAX_SUPERSET, row stride S); keeps the best topb by (dist, id).
// One CTA (8 warps) per query: 8 lanes per candidate, 32 candidates in
// flight, then a bitonic sort of the keys in shared memory.
__global__ void __launch_bounds__(256)
rerank_kernel(const float *__restrict__ vecs, int dpad, const float *__restrict__ queries,
              const FvHit *__restrict__ cand, const uint32_t *__restrict__ cand_cnt, int S,
              uint32_t topb, const int32_t *__restrict__ qprog,
              const unsigned long long *__restrict__ popcnt, uint64_t nrows,
              FvHit *__restrict__ out, uint32_t *__restrict__ out_cnt,
              uint8_t *__restrict__ trunc, const RerankCert cert) {
    __shared__ uint64_t keys[TC_MAX_SUPERSET];
    pdl_wait();
    pdl_trigger();
    rerank_query<256>(blockIdx.x, keys, vecs, dpad, queries, cand, cand_cnt, S, topb, qprog, popcnt,
                      nrows, out, out_cnt, trunc, cert);
}

// ---------------------------------------------------------------- merge
// Per-query merge of the tensor-core scan's kept keys (one CTA per query).
// Query q's keys are dense[q][0 .. dcnt[q]) in any order; only keys at or
// below the grid-wide bound can be in the answer. Keys are unique 64-bit
// (distance bits, row) values, so the KO-th smallest is found exactly by a
// radix select, 8 bits per pass (a histogram of the digit among the keys
// that share the digits chosen so far), and only the at most KO keys at or
// below it are sorted. Runs up to stage_cap keys are staged in shared
// memory; longer ones are read from global memory on every pass (4 loads
// in flight per lane).
__global__ void __launch_bounds__(DM_THREADS)
dense_merge_kernel(const uint64_t *__restrict__ dense, uint64_t dcap, int stage_cap,
                   uint32_t *__restrict__ dcnt, int reset_cnt,
                   const unsigned long long *__restrict__ fullmin,
                   const unsigned long long *tau, int KO, const int32_t *__restrict__ qprog,
                   const unsigned long long *__restrict__ popcnt, uint64_t nrows,
                   FvHit *__restrict__ out, uint32_t *__restrict__ out_cnt,
                   uint8_t *__restrict__ trunc, unsigned long long *tau_out,
                   uint8_t *__restrict__ unc) {
    extern __shared__ __align__(16) unsigned char dm_smem[];
    pdl_wait();
    pdl_trigger();
    dense_merge_query(blockIdx.x, (uint64_t *)dm_smem, dense, dcap, stage_cap, dcnt, reset_cnt,
                      fullmin, tau, KO, qprog, popcnt, nrows, out, out_cnt, trunc, tau_out, unc);
}

__global__ void __launch_bounds__(DM_THREADS)
dense_top32_kernel(const uint64_t *__restrict__ dense, uint64_t dcap, uint32_t *__restrict__ dcnt,
                   int reset_cnt, const unsigned long long *__restrict__ fullmin,
                   const unsigned long long *tau, int KO, const int32_t *__restrict__ qprog,
                   const unsigned long long *__restrict__ popcnt, uint64_t nrows,
                   FvHit *__restrict__ out, uint32_t *__restrict__ out_cnt,
                   uint8_t *__restrict__ trunc, unsigned long long *tau_out,
                   uint8_t *__restrict__ unc) {
    __shared__ uint64_t lists[DM_THREADS / 32][32];
    // the batch's programs and the bitmap kernel's counts were written two
    // or more kernels back (each kernel of the chain triggers the next only
    // after its own wait): read them while the kernel ahead finishes
    long long passing = -1;
    if (threadIdx.x == 0) {
        const int pg = qprog[blockIdx.x];
        passing = (long long)(pg >= 0 ? popcnt[pg] : nrows);
    }
    pdl_wait();
    pdl_trigger();
    dense_top32_query(blockIdx.x, lists, dense, dcap, dcnt, reset_cnt, fullmin, tau, KO, qprog,
                      popcnt, nrows, out, out_cnt, trunc, tau_out, unc, passing);
}

cudaError_t launch_dense_merge(const uint64_t *dense, uint64_t dcap, uint32_t *dcnt,
                               bool reset_cnt, const unsigned long long *fullmin,
                               const unsigned long long *tau, int KO, const int32_t *qprog,
                               const unsigned long long *popcnt, uint64_t nrows, int nq,
                               FvHit *out, uint32_t *out_cnt, uint8_t *trunc,
                               unsigned long long *tau_out, uint8_t *unc, cudaStream_t st) {
    if (KO < 1 || KO > DM_OUT) return cudaErrorInvalidValue;
    if (KO <= 32) {
        return launch_pdl(dense_top32_kernel, dim3(nq), dim3(DM_THREADS), 0, st, dense, dcap,
                          dcnt, reset_cnt ? 1 : 0, fullmin, tau, KO, qprog, popcnt, nrows, out,
                          out_cnt, trunc, tau_out, unc);
    }
    // the stage holds a whole run when it can (runs never exceed dcap)
    const int stage_cap = (int)std::min<uint64_t>(std::max<uint64_t>(dcap, 1), DM_CAP_MAX);
    const size_t smem = (size_t)(stage_cap + DM_OUT) * 8;
    cudaError_t e = raise_smem_limit((const void *)dense_merge_kernel, smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(dense_merge_kernel, dim3(nq), dim3(DM_THREADS), smem, st, dense, dcap,
                      stage_cap, dcnt, reset_cnt ? 1 : 0, fullmin, tau, KO, qprog, popcnt, nrows,
                      out, out_cnt, trunc, tau_out, unc);
}

// ---------------------------------------------------------------- host side
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) ==
                cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// 2-D row-major [rows][inner] tensor map with 128-byte swizzled boxes of
// [128 rows][128 bytes] (elements of the operand kind: fp8, bf16 or f32).
// Columns past `inner` read as zeros.
bool tc_make_tmap(CUtensorMap *m, const void *ptr, int kind, uint64_t inner, uint64_t rows) {
    auto enc = get_encode();
    if (!enc) return false;
    const uint32_t esz = (uint32_t)tck_esz(kind);
    cuuint64_t dims[2] = {inner, rows};
    cuuint64_t strides[1] = {inner * esz};
    cuuint32_t box[2] = {TC_KB_BYTES / esz, TC_BN};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapDataType dt = kind == TCK_FP8    ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                   : kind == TCK_TF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                      : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUresult r = enc(m, dt, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Candidates kept per query before the exact re-rank (the superset): 4k
// while the scan's distances may be inexact; k itself when the upload
// certified that BF16 distances are exact (integer rows, |x| <= 256, all
// sums below 2^24), since then the scan's top-k already is the exact top-k.
// 0 = topb too large.
int tc_superset(const FvGpuIndex *g, uint32_t topb, float q_amax) {
    const bool exact = g->precision != FV_GPU_PREC_FP8 && !g->force_wide_superset &&
                       pv_bf16_exact(g->dim, g->row_amax, q_amax);
    const int s = exact ? (int)topb : 4 * (int)topb;
    return s <= TC_MAX_SUPERSET ? s : 0;  // 0: topb beyond the superset capacity
}

// The exact scan on the tensor cores reads the f32 rows as TF32 and
// re-ranks a superset exactly: S = k when the upload certified integer rows
// (TF32 keeps integers up to 2048 exactly, so the norm-form distances are
// exact as in the BF16 case), else 4k (at least 16), each query's answer
// then certified by the re-rank's error bound (RerankCert) and re-run on the
// CUDA cores when the bound does not separate it. 0 = topb too large.
int tf32_superset(const FvGpuIndex *g, uint32_t topb, float q_amax) {
    const bool exact = !g->force_wide_superset && pv_bf16_exact(g->dim, g->row_amax, q_amax);
    const int s = exact ? (int)topb : std::max(4 * (int)topb, 16);
    return s <= TC_MAX_SUPERSET ? s : 0;
}

// Rows of at most 128 f32 (the query tile stays 64 KB of shared memory),
// at least 8 row tiles, and not switched off for the index.
bool tf32_supported(const FvGpuIndex *g) {
    return g->exact_tc && g->d_norm32 && g->dpad <= 128 && g->count >= 8 * (uint64_t)TC_BN;
}

bool tc_supported(const FvGpuIndex *g) {
    if (g->precision == FV_GPU_PREC_FP32 || !g->d_vlow) return false;
    const int row_bytes = g->kpad * (g->precision == FV_GPU_PREC_FP8 ? 1 : 2);
    return row_bytes <= 512;  // query tile <= 64 KB of shared memory
}

static size_t tc_smem(int kblocks, int NS, int KP, int EPI, bool staged = true) {
    return tc_smem_bytes(kblocks, NS, KP, EPI, staged);
}

bool tc_shape_fits(const FvGpuIndex *g, uint32_t topb, int epi, int ns) {
    if (!tc_supported(g) || epi < 1 || epi > 3 || ns < 2 || ns > TC_MAX_STAGES) return false;
    const int S = tc_superset(g, topb, -1.f);
    if (!S) return false;
    const int KP = S < TC_MAX_LIST ? S : TC_MAX_LIST;
    const int esz = g->precision == FV_GPU_PREC_FP8 ? 1 : 2;
    return tc_smem(g->kpad * esz / TC_KB_BYTES, ns, KP, epi) <= 227 * 1024;
}

template <int KIND, int EPI, bool WARM>
static cudaError_t tc_launch_kind(int grid, size_t smem, cudaStream_t st, const CUtensorMap &tmX,
                                  const CUtensorMap &tmQ, const TcArgs &a) {
    cudaError_t e = raise_smem_limit((const void *)scan_tc_kernel<KIND, EPI, WARM>, smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(scan_tc_kernel<KIND, EPI, WARM>, dim3(grid), dim3(64 + 128 * EPI), smem,
                      st, tmX, tmQ, a);
}

template <int EPI, bool WARM>
static cudaError_t tc_launch(int kind, int grid, size_t smem, cudaStream_t st,
                            const CUtensorMap &tmX, const CUtensorMap &tmQ, const TcArgs &a) {
    if (kind == TCK_FP8) return tc_launch_kind<TCK_FP8, EPI, WARM>(grid, smem, st, tmX, tmQ, a);
    if (kind == TCK_TF32) return tc_launch_kind<TCK_TF32, EPI, WARM>(grid, smem, st, tmX, tmQ, a);
    return tc_launch_kind<TCK_BF16, EPI, WARM>(grid, smem, st, tmX, tmQ, a);
}

// Launches query prep, the tensor-core scan, the per-query merge and the
// exact re-rank. Inputs: f32 queries [nq][dpad] on the device, predicate
// programs/bitmaps already built. tf32: scan the f32 rows themselves (the
// exact mode), else the upload's BF16 / FP8 rows.
int launch_scan_tc(FvGpuIndex *g, int nq, float q_amax, const float *d_q,
                   const int32_t *d_qprog,
                   const uint32_t *bitmaps, uint64_t bm_words,
                   const unsigned long long *popcnt, uint32_t topb, FvHit *d_out,
                   uint32_t *d_cnt, uint8_t *d_trunc, cudaEvent_t *ev, char *errbuf,
                   size_t errlen, const TcLazy *lz, bool tf32, const TcRowSet *rs,
                   bool behind_bitmaps, cudaEvent_t prep_done) {
    const bool fp8 = !tf32 && g->precision == FV_GPU_PREC_FP8;
    const int kind = tf32 ? TCK_TF32 : fp8 ? TCK_FP8 : TCK_BF16;
    const int esz = tck_esz(kind);
    // elements of K per row: the low-precision row pitch, or dpad rounded up
    // to whole 32-element boxes (the f32 rows' tail boxes read zeros)
    const int kelems = tf32 ? ((g->dpad + 31) & ~31) : g->kpad;
    const int kblocks = kelems * esz / TC_KB_BYTES;
    const int S = tf32 ? tf32_superset(g, topb, q_amax) : tc_superset(g, topb, q_amax);
    const int KP = S < TC_MAX_LIST ? S : TC_MAX_LIST;
    g->last_superset = S;
    g->tc_unc = nullptr;
    if (!S || !(tf32 ? tf32_supported(g) : tc_supported(g)) || (rs && lz)) {
        snprintf(errbuf, errlen, "gpu: tensor-core scan not available for this batch");
        return -1;
    }
    // epilogue warp groups (each owning every EPI-th tile): two when the
    // lists fit with at least two pipeline stages, else one (three groups
    // measured no faster at batch 64: 0.0654 vs 0.0643 ms; pv_tc_shape can
    // ask for them). The automatic shape stays within smem_pref, which
    // leaves each SM a few KB for a small kernel beside the scan (the
    // router's, a merge launched early).
    const size_t smem_cap = 227 * 1024;
    const size_t smem_pref = 222 * 1024;
    // stages: up to 128 KB of rows in flight
    const int ns0 = std::min(TC_MAX_STAGES, std::max(
        2, (int)(128 * 1024 / ((size_t)std::min(kblocks, TC_KBS) * TC_BOX))));
    int EPI = 0, NS = 0;
    for (int e = 2; e >= 1 && !EPI; e--) {
        const int nmin = e == 3 ? 3 : 2;
        int n = ns0;
        while (n > nmin && tc_smem(kblocks, n, KP, e, !tf32) > smem_pref) n--;
        if (n >= nmin && tc_smem(kblocks, n, KP, e, !tf32) <= smem_pref) {
            EPI = e;
            NS = n;
        }
    }
    if (!EPI) {  // the smallest shape, within the hard limit
        EPI = 1;
        NS = 2;
    }
    if (g->tune_epi || g->tune_ns) {  // a tuned shape, if it fits
        const int e = g->tune_epi ? g->tune_epi : EPI, n = g->tune_ns ? g->tune_ns : NS;
        if (e >= 1 && e <= 3 && n >= 2 && n <= TC_MAX_STAGES &&
            tc_smem(kblocks, n, KP, e, !tf32) <= smem_cap) {
            EPI = e;
            NS = n;
        }
    }
    const size_t smem = tc_smem(kblocks, NS, KP, EPI, !tf32);
    const int qtiles = (nq + TC_BM - 1) / TC_BM;
    const int nqpad = qtiles * TC_BM;
    // query replicas: as many as the batch leaves room for, while each
    // part of a tile keeps at least 32 rows (one TMEM load)
    int R = 1;
    if (g->tune_rep > 0) R = g->tune_rep;
    else if (qtiles == 1) R = nq <= 32 ? 4 : nq <= 64 ? 2 : 1;
    while (R > 1 && (TC_BM / R < nq || TC_BN / R < 32)) R >>= 1;
    const int bq = TC_BM / R;
    // rows scanned: the index's, or a compacted set
    const uint64_t nrows_scan = rs ? rs->nrows : g->count;
    const uint64_t ntiles_all = (nrows_scan + TC_BN - 1) / TC_BN;
    int grow = g->tune_grow > 0 ? g->tune_grow : g->sm_count / qtiles;
    if (grow < 1) grow = 1;
    uint64_t maxg = (ntiles_all + 3) / 4;
    if ((uint64_t)grow > maxg) grow = (int)maxg;
    const uint64_t tpc = (ntiles_all + grow - 1) / grow;
    grow = (int)((ntiles_all + tpc - 1) / tpc);

    ScanScratch &s = g->scan;
    const size_t qbytes = (size_t)nqpad * kelems * esz;
    const size_t off_qn = (qbytes + 255) & ~(size_t)255;
    const size_t off_qs = off_qn + (((size_t)nqpad * 4 + 255) & ~(size_t)255);
    const size_t off_err = off_qs + (((size_t)nqpad * 4 + 255) & ~(size_t)255);
    const size_t off_cand = off_err + 256;
    const size_t off_ccnt = off_cand + (((size_t)nq * S * sizeof(FvHit) + 255) & ~(size_t)255);
    const size_t off_ctr = off_ccnt + (((size_t)nq * 4 + 255) & ~(size_t)255);
    const size_t off_unc = off_ctr + (((size_t)nq + 255) & ~(size_t)255);
    const size_t cbytes = off_unc + (size_t)nq + 256;
    PV_CUDA_OK(s.cand.ensure(cbytes), errbuf, errlen);
    PV_CUDA_OK(s.tau.ensure((size_t)nq * 8), errbuf, errlen);
    const int nlists = grow * EPI * R;  // lists per query
    const uint64_t dcap = (uint64_t)nlists * KP;  // a query's dense run at most
    PV_CUDA_OK(s.part.ensure((size_t)nq * dcap * 8), errbuf, errlen);
    // [dcnt u32 x nq][fullmin u64 x nq]
    const size_t off_fm = ((size_t)nq * 4 + 255) & ~(size_t)255;
    PV_CUDA_OK(s.part_cnt.ensure(off_fm + (size_t)nq * 8), errbuf, errlen);
    uint32_t *d_dcnt = s.part_cnt.as<uint32_t>();
    unsigned long long *d_fullmin = (unsigned long long *)(s.part_cnt.as<char>() + off_fm);
    unsigned char *c = s.cand.as<unsigned char>();
    int *d_err = (int *)(c + off_err);
    const bool certify = KP < S;  // lists shorter than the superset
    // inexact scan distances of exact-mode batches: the re-rank certifies
    const bool num_cert = tf32 && S > (int)topb;

    g->launches += 4;  // query prep, main pass, merge, re-rank
    PV_CUDA_OK(launch_pdl(query_prep_kernel, dim3((nqpad + 7) / 8), dim3(256), 0, g->stream, d_q,
                          nq, g->dpad, g->dim, nqpad, R > 1 ? bq : nqpad, kelems, kind, c,
                          (float *)(c + off_qn), fp8 ? (float *)(c + off_qs) : nullptr,
                          s.tau.as<unsigned long long>(), d_dcnt,
                          certify ? d_fullmin : nullptr, d_err, behind_bitmaps ? 1 : 0),
               errbuf, errlen);
    if (prep_done) PV_CUDA_OK(cudaEventRecord(prep_done, g->stream), errbuf, errlen);

    static_assert(sizeof(CUtensorMap) == sizeof(g->tmap_x), "CUtensorMap size");
    CUtensorMap tmX, tmQ;
    bool &x_ok = rs ? g->tmap_c_ok : tf32 ? g->tmap_x32_ok : g->tmap_x_ok;
    unsigned char *x_map = rs ? g->tmap_c : tf32 ? g->tmap_x32 : g->tmap_x;
    if (tf32 && !rs && g->tmap_x32_rows != g->count) x_ok = false;  // encoded for the current rows
    if (rs && (g->tmap_c_ptr != rs->rows || g->tmap_c_rows != rs->nrows || g->tmap_c_kind != kind))
        x_ok = false;
    if (rs && !x_ok) {
        if (!tc_make_tmap(&tmX, rs->rows, kind, (uint64_t)(tf32 ? g->dpad : g->kpad), rs->nrows)) {
            snprintf(errbuf, errlen, "gpu: tensor map encoding failed");
            return -1;
        }
        memcpy(x_map, &tmX, sizeof(tmX));
        x_ok = true;
        g->tmap_c_ptr = rs->rows;
        g->tmap_c_rows = rs->nrows;
        g->tmap_c_kind = kind;
    }
    if (!x_ok) {
        const bool okm = tf32 ? tc_make_tmap(&tmX, g->d_vecs, kind, (uint64_t)g->dpad, g->count)
                              : tc_make_tmap(&tmX, g->d_vlow, kind, (uint64_t)g->kpad, g->count);
        if (!okm) {
            snprintf(errbuf, errlen, "gpu: tensor map encoding failed");
            return -1;
        }
        memcpy(x_map, &tmX, sizeof(tmX));
        x_ok = true;
        if (tf32) g->tmap_x32_rows = g->count;
    }
    memcpy(&tmX, x_map, sizeof(tmX));
    if (g->tmap_q_ptr != c || g->tmap_q_rows != (uint64_t)nqpad || g->tmap_q_kind != kind) {
        if (!tc_make_tmap(&tmQ, c, kind, (uint64_t)kelems, (uint64_t)nqpad)) {
            g->tmap_q_ptr = nullptr;
            snprintf(errbuf, errlen, "gpu: tensor map encoding failed");
            return -1;
        }
        memcpy(g->tmap_q, &tmQ, sizeof(tmQ));
        g->tmap_q_ptr = c;
        g->tmap_q_rows = (uint64_t)nqpad;
        g->tmap_q_kind = kind;
    }
    memcpy(&tmQ, g->tmap_q, sizeof(tmQ));
    TcArgs a;
    a.nrows = nrows_scan;
    a.kblocks = kblocks;
    a.nq = nq;
    a.qtiles = qtiles;
    a.grow = grow;
    a.tiles_per_cta = tpc;
    a.KP = KP;
    a.rep = R;
    a.bq = bq;
    a.push_tau = KP == S ? 1 : 0;
    a.NS = NS;
    a.xnorm = rs ? rs->norms : tf32 ? g->d_norm32 : g->d_norm;
    a.xscale = fp8 ? (rs ? rs->scales : g->d_vscale) : nullptr;
    a.rowids = rs ? rs->rowids : nullptr;
    a.nrows_dev = rs ? rs->nrows_dev : nullptr;
    a.qnorm = (const float *)(c + off_qn);
    a.qscale = fp8 ? (const float *)(c + off_qs) : nullptr;
    a.qprog = d_qprog;
    a.bitmaps = bitmaps;
    a.bm_words = bm_words;
    a.lazy = lz ? lz->flag : nullptr;
    a.progs = lz ? lz->progs : nullptr;
    a.insns = lz ? lz->insns : nullptr;
    a.consts = lz ? lz->consts : nullptr;
    a.nconsts = lz ? lz->nconsts : 0;
    a.cols = g->d_cols;
    a.ncols = g->ncols;
    a.tau = s.tau.as<unsigned long long>();
    a.dense = s.part.as<uint64_t>();
    a.dcnt = d_dcnt;
    a.dcap = dcap;
    a.kwrite = KP;
    a.fullmin = certify ? d_fullmin : nullptr;
    a.err = d_err;
    a.timeout_ns = g->tc_timeout_ns ? g->tc_timeout_ns : 2000000000ull;
    a.drain_ns = 2000000000ull;
    a.trace = nullptr;
    a.trace_tiles = 0;
    static const bool tracing = getenv("PV_TC_TRACE") != nullptr;
    static uint64_t *d_trace = nullptr;
    if (tracing) {
        if (!d_trace) cudaMalloc(&d_trace, 64 * 4 * 8);
        if (d_trace) {
            cudaMemsetAsync(d_trace, 0, 64 * 4 * 8, g->stream);
            a.trace = d_trace;
            a.trace_tiles = 64;
        }
    }
    // warm: a pass that starts without a bound (see tc_pass)
    // (a warm pass with three groups would not fit its registers: it runs
    // with two, inside the same shared-memory carve and dense runs)
    auto run = [&](const TcArgs &args, bool warm) {
        const int gr = args.grow * qtiles;
        if (warm)
            return EPI >= 2 ? tc_launch<2, true>(kind, gr, smem, g->stream, tmX, tmQ, args)
                            : tc_launch<1, true>(kind, gr, smem, g->stream, tmX, tmQ, args);
        if (EPI == 3) return tc_launch<3, false>(kind, gr, smem, g->stream, tmX, tmQ, args);
        if (EPI == 2) return tc_launch<2, false>(kind, gr, smem, g->stream, tmX, tmQ, args);
        return tc_launch<1, false>(kind, gr, smem, g->stream, tmX, tmQ, args);
    };
    FvHit *cand = (FvHit *)(c + off_cand);
    uint32_t *ccnt = (uint32_t *)(c + off_ccnt);
    // Seeding pass: a few tiles per CTA from an evenly strided sample; the
    // merged K'-th key of the sample bounds the K'-th key of the whole
    // scan, so the main pass admits only rows that can still matter.
    const bool seed = g->tune_seed == 2 ? false : ntiles_all >= 8 * (uint64_t)grow;
    if (seed) {
        TcArgs sa = a;
        // larger supersets take a larger sample (up to 8 tiles per CTA,
        // spread over the CTA's own range), so the bound stays near the
        // S-th key and the final merge's survivors fit one pass
        const uint64_t region = ntiles_all / grow;
        const uint64_t m = std::min<uint64_t>(std::min<uint64_t>(8, region),
                                              std::max<uint64_t>(1, ((uint64_t)S + 15) / 16));
        sa.tile0_mul = region;
        sa.tile_step = std::max<uint64_t>(1, region / m);
        sa.tiles_per_cta = m;
        // only each list's best keys: the S-th key of a subset of the
        // sample still bounds the S-th key of the scan, and a short run
        // keeps the merge cheap (the radix select of S > 32 reads its run
        // 8 times). The sample's S best keys are spread over many lists
        // (S / nlists per list on average): 4S keys in all, at least one
        // per list, never more than the main pass's list length (its
        // shared memory). One key per list when that suffices measured
        // 3.5 µs less before the main pass than two (batch 64, S = 10,
        // 592 lists: heaps of one, half the seeding merge's keys), for a
        // bound barely looser (the main pass ran the same).
        sa.kwrite = std::min(KP, std::max(1, (4 * S + nlists - 1) / std::max(1, nlists)));
        // lists need hold no more than that (short heaps admit fewer rows);
        // a full list's last key bounds the S-th key only if it holds S
        sa.KP = sa.kwrite;
        sa.push_tau = sa.KP == S ? 1 : 0;
        sa.fullmin = nullptr;
        g->launches += 2;  // seeding pass + its merge
        PV_CUDA_OK(run(sa, true), errbuf, errlen);
        // the merge leaves the counts at zero for the main pass
        PV_CUDA_OK(launch_dense_merge(a.dense, dcap, d_dcnt, true, nullptr, a.tau, S, d_qprog,
                                      popcnt, g->count, nq, cand, ccnt,
                                      (uint8_t *)(c + off_ctr), a.tau, nullptr, g->stream),
                   errbuf, errlen);
    }
    // stage boundary: everything before the main pass (bitmaps, query prep,
    // seeding) is stage 0, the main pass alone is stage 1
    if (ev) cudaEventRecord(ev[1], g->stream);
    // contiguous tile ranges per CTA; a compacted set's tiles are dealt
    // round robin instead, so the rows that exist (a prefix of its tiles)
    // spread over the CTAs
    a.tile0_mul = rs ? 1 : tpc;
    a.tile_step = rs ? (uint64_t)grow : 1;
    PV_CUDA_OK(run(a, rs != nullptr), errbuf, errlen);
    if (ev) cudaEventRecord(ev[2], g->stream);
    uint8_t *d_unc = (certify || num_cert) ? (uint8_t *)(c + off_unc) : nullptr;
    if (S == (int)topb) {
        // certified exact (integer rows and queries, all sums below 2^24):
        // every norm-form distance already is the exact squared L2 distance,
        // so the merged top-k is the answer and needs no re-rank
        g->launches--;
        PV_CUDA_OK(launch_dense_merge(a.dense, dcap, d_dcnt, false, a.fullmin, a.tau, S,
                                      d_qprog, popcnt, g->count, nq, d_out, d_cnt, d_trunc,
                                      nullptr, d_unc, g->stream),
                   errbuf, errlen);
    } else {
        PV_CUDA_OK(launch_dense_merge(a.dense, dcap, d_dcnt, false, a.fullmin, a.tau, S,
                                      d_qprog, popcnt, g->count, nq, cand, ccnt,
                                      (uint8_t *)(c + off_ctr), nullptr, d_unc, g->stream),
                   errbuf, errlen);
        RerankCert cert;
        if (num_cert) {
            cert.qnorm = (const float *)(c + off_qn);
            cert.xnmax = g->norm32_max;
            cert.dim = g->dpad;
            cert.unc = d_unc;
        }
        PV_CUDA_OK(launch_pdl(rerank_kernel, dim3(nq), dim3(256), 0, g->stream, g->d_vecs,
                              g->dpad, d_q, cand, ccnt, S, topb, d_qprog, popcnt, g->count, d_out,
                              d_cnt, d_trunc, cert),
                   errbuf, errlen);
    }
    g->tc_unc = d_unc;
    g->tc_unc_n = nq;
    if (ev) cudaEventRecord(ev[3], g->stream);
    g->tc_err = d_err;
    g->tc_err_h = nullptr;  // its host copy, if any, is queued by the caller
    if (tracing && d_trace) {
        uint64_t h[64 * 4];
        cudaStreamSynchronize(g->stream);
        cudaMemcpy(h, d_trace, sizeof(h), cudaMemcpyDeviceToHost);
        const uint64_t t0 = h[0];
        for (int t = 0; t < 64 && h[t * 4]; t++)
            fprintf(stderr, "PVTRACE tile %d issue %.2f mma %.2f epi %.2f done %.2f us\n", t,
                    (h[t * 4] - t0) / 1e3, (h[t * 4 + 1] - t0) / 1e3,
                    (h[t * 4 + 2] - t0) / 1e3, (h[t * 4 + 3] - t0) / 1e3);
    }
    return 0;
}

}  // namespace pv

namespace pv {
// Queues the copy of the watchdog word into pinned host memory behind the
// batch's own result copy, so reading it costs no extra round trip.
void tc_watchdog_enqueue(FvGpuIndex *g, int *h_word) {
    g->tc_err_h = nullptr;
    if (!g->tc_err) return;
    if (cudaMemcpyAsync(h_word, g->tc_err, 4, cudaMemcpyDeviceToHost, g->stream) == cudaSuccess)
        g->tc_err_h = h_word;
    else
        (void)cudaGetLastError();
}

int check_tc_watchdog(FvGpuIndex *g, char *errbuf, size_t errlen) {
    if (!g->tc_err) return 0;
    int e = 0;
    if (g->tc_err_h) {  // queued with the results
        PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
        e = *(volatile int *)g->tc_err_h;
        g->tc_err_h = nullptr;
    } else {
        PV_CUDA_OK(cudaMemcpyAsync(&e, g->tc_err, 4, cudaMemcpyDeviceToHost, g->stream), errbuf,
                   errlen);
        PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
    }
    if (e) {
        cudaMemsetAsync(g->tc_err, 0, 4, g->stream);
        snprintf(errbuf, errlen, "gpu: tensor-core scan wait expired (role %d)", e);
        return -1;
    }
    return 0;
}
}  // namespace pv
