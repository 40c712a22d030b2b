// index.h — device-resident index layout and per-call staging (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace pv {

// Grow-only device or pinned-host buffer. A buffer keeps its kind for life
// (device memory is never released with the pinned-host call or the reverse).
struct Buf {
    void *p = nullptr;
    size_t cap = 0;
    bool host = false;
    explicit Buf(bool pinned_host = false) : host(pinned_host) {}
    cudaError_t ensure(size_t need) {
        if (need <= cap) return cudaSuccess;
        release();
        size_t n = need + need / 4 + 256;
        cudaError_t e = host ? cudaMallocHost(&p, n) : cudaMalloc(&p, n);
        if (e == cudaSuccess) cap = n;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p) {
            if (host) cudaFreeHost(p); else cudaFree(p);
        }
        p = nullptr;
        cap = 0;
    }
    template <typename T> T *as() const { return (T *)p; }
};

// Host-compiled predicates of one batch (see pred.cpp).
struct PredBatch {
    std::vector<PredInsn> insns;
    std::vector<PredProg> progs;
    std::vector<double> consts;
    std::vector<int32_t> qprog;  // per query: program id or -1
    std::vector<int32_t> cols_used;  // per program: bit mask of columns (<=32)
};

// Per-call scratch for the scan path (device unless noted).
struct ScanScratch {
    Buf stage_h{true};   // pinned: packed inputs
    Buf stage_d;         // device copy of the packed inputs
    Buf bitmaps;         // [P][bm_words] u32
    Buf popcnt;          // [P] u64
    Buf tau;             // [nq] u64
    Buf part;            // [nq][grow][K] u64 keys
    Buf part_cnt;        // [nq][grow] u32
    Buf cand;            // reduced-precision candidate superset keys
    Buf out_d;           // FvHit [nq][topb] + cnt [nq] + trunc [nq]
    Buf out_h{true};
    Buf sparse;          // selective filters: row count, row ids, no-filter programs
};

struct GraphScratch {
    Buf visited;  // per query overflow bitmap (words), zeroed by the kernel
    Buf res;      // per query results
    Buf stats;    // per query counters
    Buf route;    // routed batches: features, logits, beam widths
    Buf route_h{true};  // routed batches: beam widths and graph results on the host
    Buf gout;     // routed batches: graph results on the device
};

}  // namespace pv

// The opaque handle of the C ABI.
struct FvGpuIndex {
    int device = -1;
    int precision = FV_GPU_PREC_FP32;
    uint64_t count = 0;
    int dim = 0;
    int ncols = 0;
    uint32_t l0_stride = 0;

    int dpad = 0;            // f32 row stride in floats (dim rounded up to 4)
    float *d_vecs = nullptr; // [count][dpad] exact rows (always resident)
    double *d_cols = nullptr;     // [ncols][count]
    uint32_t *d_prows = nullptr;  // [ncols][count]

    // level-0 graph as fixed-degree device adjacency ("device CSR"):
    // d_adj[node*deg_cap + i], padded with UINT32_MAX; d_deg[node]
    uint32_t *d_adj = nullptr;
    uint16_t *d_deg = nullptr;
    int deg_cap = 0;

    // reduced-precision copies (precision != FP32)
    int kpad = 0;               // bf16/fp8 row stride in elements
    void *d_vlow = nullptr;     // bf16 [count][kpad] or fp8 [count][kpad]
    float *d_vscale = nullptr;  // fp8 per-row scale
    float *d_norm = nullptr;    // ||x||^2 of the stored low-precision row
    float row_amax = -1.f;      // max |x| if all rows are integers <= 256, else -1
    // the exact mode's tensor-core scan (f32 rows read as TF32)
    float *d_norm32 = nullptr;  // [rows padded to 128] ||x||^2 of the f32 rows
    float norm32_max = 0.f;     // largest of them
    int exact_tc = 1;           // exact-mode batches may take it (0: CUDA cores only)
    int last_exact_tc = 0;      // the last brute batch took it

    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;  // side stream (routing beside a speculative scan)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t rev[6] = {};  // routed batches (created on first use)
    std::mutex mu;  // ABI calls are serialized per handle

    pv::ScanScratch scan;
    pv::GraphScratch graph;
    int *tc_err = nullptr;  // watchdog word of the last tensor-core scan (device)
    int *tc_err_h = nullptr;  // its copy in pinned memory, queued with the results
    uint8_t *tc_unc = nullptr;  // per query: superset not certified (last TC scan)
    int tc_unc_n = 0;
    int last_uncertain = 0;  // queries of the last call re-run exactly (or flagged)
    // tensor-core scan shape overrides (0 = built-in choice): epilogue warp
    // groups, pipeline stages, CTAs along the rows per query tile
    int tune_epi = 0, tune_ns = 0, tune_grow = 0, tune_rep = 0, tune_seed = 0;
    int force_wide_superset = 0;  // re-rank 4 x topb even when BF16 is certified exact
    uint64_t tc_timeout_ns = 0;   // tensor-core scan wait limit (0: 2 s)
    // encoded TMA descriptors of the tensor-core scan (CUtensorMap, 128 B):
    // the rows' (fixed after upload) and the staged queries' (re-encoded
    // when their buffer or row count changes)
    alignas(64) unsigned char tmap_x[128] = {};
    alignas(64) unsigned char tmap_q[128] = {};
    alignas(64) unsigned char tmap_x32[128] = {};  // the f32 rows (exact mode)
    alignas(64) unsigned char tmap_c[128] = {};    // a compacted row set (sparse route)
    bool tmap_c_ok = false;
    const void *tmap_c_ptr = nullptr;
    uint64_t tmap_c_rows = 0;
    int tmap_c_kind = -1;
    bool tmap_x_ok = false;
    bool tmap_x32_ok = false;
    uint64_t tmap_x32_rows = 0;
    const void *tmap_q_ptr = nullptr;
    uint64_t tmap_q_rows = 0;
    int tmap_q_kind = -1;
    bool view = false;  // shares another handle's device data, owns only scratch
    int last_superset = 0;  // candidates re-ranked per query by the last TC scan
    float last_kernel_ms = 0.f;  // device time of the last batch's kernels
    int launches = 0;  // kernels launched by the last call (all iterations)
    std::vector<uint32_t> graph_stats;  // last graph batch: [nq][4] counters
    // host copy of each attribute column's non-NaN values, ascending: bounds
    // a filter's matches by binary search (sparse routing)
    std::vector<std::vector<double>> sorted_cols;
    int last_sparse = 0;  // the last brute batch took the sparse route
};
