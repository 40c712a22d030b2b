// pserve.cu — one persistent kernel serving a queue of uneven micro-batches.
//
// No reference counterpart: the reference worker answers each micro-batch
// with separate synchronous launches (worker.c:268-276 through
// fv_gpu_brute_batch, loop worker.c:453-598). Here a cooperative kernel of
// one CTA per SM stays resident and consumes batches the host stages into
// a ring of device slots (queries, per-query k, compiled range filters and
// a plan); each batch runs as grid-synchronous phases over the same
// barriers and tensor memory:
//     query prep (low-precision query tile, norms, per-query state)
//  -> predicate bitmaps, unless every filter is broad (then each query's
//     range program is tested lazily, on rows that beat its threshold)
//  -> seeding pass (a strided sample of every CTA's rows)
//  -> seed merge (each query's bound from the sample)
//  -> main pass (tc_pass over all rows)
//  -> per-query merge (+ exact FP32 re-rank), written straight into
//     host-mapped result buffers, then the batch's completion word.
// CTA 0 waits for the next batch (a tail counter the host advances with an
// ordered copy after the batch's data), bounded by an idle limit after
// which the kernel leaves; every grid barrier is bounded too (a CTA that
// does not arrive makes the others leave with a failure status), and the
// scan's own waits are bounded as in the one-shot kernel. The launch is
// captured in a CUDA graph once and replayed whenever the kernel must be
// (re)started. Batches beyond the slots' capacities and queries whose
// candidate superset the merge could not certify run on the index's
// ordinary path with the kernel stopped.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include "index.h"
#include "paves_ext.h"
#include "bitmap_core.cuh"
#include "pv_internal.h"
#include "tc_core.cuh"

namespace pv {

constexpr int SV_SLOTS = 2;

// control words in device memory (the tail lives apart: the host's copy
// stream writes it while the kernel runs)
struct SvCtl {
    unsigned long long processed;  // batches completed; set by the host before a launch
    int stop;                      // host: leave before the next batch
    int skip_cta;                  // test: this CTA skips the first barrier of the next batch
    unsigned bar_count, bar_gen;   // grid barrier
    int cmd;                       // CTA 0 -> all: 1 run a batch, 0 stop, 2 idle
    int failed;                    // a wait expired (set by any CTA)
};

// one batch's plan (host computed, copied at the head of its slot)
struct SvPlan {
    unsigned long long seq;  // batch number, 1-based
    int nq, nqpad, qtiles, rep, bq, grow;
    int S, KP, push_tau, certify, topb, lazy;
    unsigned long long tpc, dcap;
    int seed, seed_kwrite;
    unsigned long long seed_mul, seed_step, seed_tiles;
    int nconsts, P, ninsns, pad;
};

struct SvArgs {
    // index
    uint64_t nrows;
    int dim, dpad, kpad, kblocks, NS, KPcap, ncols;
    const float *vecs, *xnorm, *xscale;
    const double *cols;
    // queue
    SvCtl *ctl;
    const unsigned long long *tail;
    unsigned char *slots;  // SV_SLOTS x slot_bytes
    size_t slot_bytes, off_q, off_qprog, off_progs, off_insns, off_consts;
    unsigned char *qbuf;   // SV_SLOTS x qbuf_bytes: low-precision query tiles
    size_t qbuf_bytes;
    const CUtensorMap *tmQ;  // [SV_SLOTS], over each slot's query tile
    // scratch
    float *qnorm, *qscale;
    unsigned long long *tau, *fullmin;
    uint64_t *dense;
    uint32_t *dcnt;
    FvHit *cand;
    uint32_t *ccnt;
    uint8_t *ctr;
    unsigned long long *popcnt;  // [max_batch] passing rows per program
    uint32_t *bitmaps;           // [max_batch][bm_words]
    int *err;
    // host-mapped results per slot
    FvHit *out;          // [SV_SLOTS][max_batch][max_k]
    uint32_t *out_cnt;   // [SV_SLOTS][max_batch]
    uint8_t *out_unc;    // [SV_SLOTS][max_batch]
    unsigned long long *done;    // [SV_SLOTS] completed batch number
    unsigned long long *tstamp;  // [SV_SLOTS][2] globaltimer at start / end
    int max_batch, max_k;
    // limits
    uint64_t idle_ns, bar_ns, timeout_ns, drain_ns;
    size_t merge_smem;  // shared bytes the per-query phases may use
};

__device__ __forceinline__ unsigned long long sv_ld(const unsigned long long *p) {
    return *(const volatile unsigned long long *)p;
}
__device__ __forceinline__ int sv_ldi(const int *p) { return *(const volatile int *)p; }

// Grid barrier of all CTAs (co-resident: cooperative launch), bounded:
// false when the other CTAs did not all arrive within limit_ns.
__device__ bool sv_grid_sync(SvCtl *c, uint64_t limit_ns, bool skip) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (!skip) {
            const unsigned gen = *(volatile unsigned *)&c->bar_gen;
            __threadfence();
            const unsigned arrived = atomicAdd(&c->bar_count, 1u);
            if (arrived == gridDim.x - 1) {
                *(volatile unsigned *)&c->bar_count = 0;
                __threadfence();
                atomicAdd(&c->bar_gen, 1u);
            } else {
                const uint64_t dl = sm100::globaltimer() + limit_ns;
                while (*(volatile unsigned *)&c->bar_gen == gen) {
                    if (sm100::globaltimer() > dl) {
                        ok = 0;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __threadfence();
        } else {
            ok = 0;  // a CTA told to skip its arrival leaves like one that timed out
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <bool FP8, int EPI>
__global__ void __launch_bounds__(64 + 128 * EPI, 1)
pserve_kernel(const __grid_constant__ CUtensorMap tmX, SvArgs p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = smem_raw + ((1024 - (sm100::smem_u32(smem_raw) & 1023)) & 1023);
    const TcSmem sm = tc_carve(base, p.kblocks, p.NS, p.KPcap, EPI);
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int NT = 64 + 128 * EPI;
    constexpr int NW = NT / 32;
    const int G = gridDim.x;
    if (tid == 0) {
        s_abort = 0;
        tc_init_barriers(sm, p.NS, EPI);
    }
    if (warp == 1) {
        tmem_alloc(&s_tmem, TC_TMEM_COLS);
        tmem_relinquish();
    }
    __syncthreads();
    tc_fence_after();
    TcRun run;
    unsigned long long done = sv_ld(&p.ctl->processed);
    bool failed = false;
    const int skip_cta = sv_ldi(&p.ctl->skip_cta);
    bool skip_next = skip_cta == (int)blockIdx.x;
    // shared memory the per-query phases use: the pass buffers before the
    // barriers (idle between passes)
    uint64_t *mkeys = (uint64_t *)sm.sQ;
    const int stage_cap =
        (int)std::min<size_t>(DM_CAP_MAX, p.merge_smem / 8 > (size_t)DM_OUT ? p.merge_smem / 8 - DM_OUT : 0);

    for (;;) {
        // ---- the next batch (CTA 0 waits; the others wait at the barrier)
        if (blockIdx.x == 0 && tid == 0) {
            const uint64_t dl = sm100::globaltimer() + p.idle_ns;
            int cmd;
            for (;;) {
                if (sv_ld(p.tail) > done) { cmd = 1; break; }
                if (sv_ldi(&p.ctl->stop)) { cmd = 0; break; }
                if (sm100::globaltimer() > dl) { cmd = 2; break; }
                __nanosleep(500);
            }
            p.ctl->cmd = cmd;
            if (cmd == 1) p.tstamp[(done % SV_SLOTS) * 2] = sm100::globaltimer();
            __threadfence();
        }
        // (barriers the other CTAs wait at outlast CTA 0's idle wait)
        if (!sv_grid_sync(p.ctl, p.idle_ns + p.bar_ns, skip_next)) {
            failed = true;
            break;
        }
        skip_next = false;
        const int cmd = sv_ldi(&p.ctl->cmd);
        if (cmd != 1) break;
        const int slot = (int)(done % SV_SLOTS);
        unsigned char *sb = p.slots + (size_t)slot * p.slot_bytes;
        const SvPlan pl = *(const SvPlan *)sb;
        const float *qf = (const float *)(sb + p.off_q);
        const int32_t *qprog = (const int32_t *)(sb + p.off_qprog);
        unsigned char *qb = p.qbuf + (size_t)slot * p.qbuf_bytes;

        // ---- query prep: low-precision tile rows, norms, per-query state
        {
            const int rows = pl.nqpad;
            for (int qi = blockIdx.x * NW + warp; qi < rows; qi += G * NW)
                query_prep_row(qi, lane, qf, pl.nq, p.dpad, p.dim, pl.bq, p.kpad, FP8 ? TCK_FP8 : TCK_BF16, qb,
                               p.qnorm, FP8 ? p.qscale : nullptr, p.tau, p.dcnt,
                               pl.certify ? p.fullmin : nullptr, p.err);
            for (int i = blockIdx.x * NT + tid; i < pl.P; i += G * NT) p.popcnt[i] = 0;
            // the tile is read by TMA (async proxy) after the barrier
            asm volatile("fence.proxy.async.global;" ::: "memory");
        }
        if (!sv_grid_sync(p.ctl, p.bar_ns, false)) { failed = true; break; }
        // ---- predicate bitmaps (filters that are not all broad)
        if (!pl.lazy && pl.P > 0) {
            bitmap_work(blockIdx.x, G, p.cols, p.nrows, (const PredInsn *)(sb + p.off_insns),
                        pl.ninsns, (const PredProg *)(sb + p.off_progs), pl.P,
                        (const double *)(sb + p.off_consts), pl.nconsts, nullptr, p.ncols,
                        p.bitmaps, (p.nrows + 31) / 32, p.popcnt);
            if (!sv_grid_sync(p.ctl, p.bar_ns, false)) { failed = true; break; }
        }

        TcArgs a;
        a.nrows = p.nrows;
        a.kblocks = p.kblocks;
        a.nq = pl.nq;
        a.qtiles = pl.qtiles;
        a.grow = pl.grow;
        a.rep = pl.rep;
        a.bq = pl.bq;
        a.NS = p.NS;
        a.xnorm = p.xnorm;
        a.xscale = FP8 ? p.xscale : nullptr;
        a.qnorm = p.qnorm;
        a.qscale = FP8 ? p.qscale : nullptr;
        a.qprog = qprog;
        a.bitmaps = p.bitmaps;
        a.bm_words = (p.nrows + 31) / 32;
        a.lazy = &((const SvPlan *)sb)->lazy;
        a.progs = (const PredProg *)(sb + p.off_progs);
        a.insns = (const PredInsn *)(sb + p.off_insns);
        a.consts = (const double *)(sb + p.off_consts);
        a.nconsts = pl.nconsts;
        a.cols = p.cols;
        a.ncols = p.ncols;
        a.rowids = nullptr;
        a.nrows_dev = nullptr;
        a.tau = p.tau;
        a.dense = p.dense;
        a.dcnt = p.dcnt;
        a.dcap = pl.dcap;
        a.err = p.err;
        a.timeout_ns = p.timeout_ns;
        a.drain_ns = p.drain_ns;
        a.trace = nullptr;
        a.trace_tiles = 0;
        const int qtile = blockIdx.x % pl.qtiles;
        const int rgrp = blockIdx.x / pl.qtiles;
        const bool scans = rgrp < pl.grow;

        // ---- seeding pass and its merge: each query's bound from a sample
        if (pl.seed) {
            TcArgs sa = a;
            sa.tile0_mul = pl.seed_mul;
            sa.tile_step = pl.seed_step;
            sa.tiles_per_cta = pl.seed_tiles;
            sa.KP = pl.seed_kwrite;
            sa.kwrite = pl.seed_kwrite;
            sa.push_tau = pl.seed_kwrite == pl.S ? 1 : 0;
            sa.fullmin = nullptr;
            // shared memory the merges wrote is refilled by TMA (async proxy)
            fence_proxy_async();
            __syncthreads();
            if (scans && !tc_pass<FP8 ? TCK_FP8 : TCK_BF16, EPI>(&tmX, &p.tmQ[slot], sa, sm, s_tmem, run, &s_abort,
                                            qtile, rgrp)) {
                failed = true;
                break;
            }
            if (!sv_grid_sync(p.ctl, p.bar_ns, false)) { failed = true; break; }
            for (int q = blockIdx.x; q < pl.nq; q += G) {
                if (pl.S <= 32)
                    dense_top32_query(q, (uint64_t(*)[32])mkeys, p.dense, pl.dcap, p.dcnt, 1,
                                      nullptr, p.tau, pl.S, qprog, p.popcnt, p.nrows, p.cand,
                                      p.ccnt, p.ctr, p.tau, nullptr);
                else
                    dense_merge_query(q, mkeys, p.dense, pl.dcap, stage_cap, p.dcnt, 1, nullptr,
                                      p.tau, pl.S, qprog, p.popcnt, p.nrows, p.cand, p.ccnt,
                                      p.ctr, p.tau, nullptr);
            }
            if (!sv_grid_sync(p.ctl, p.bar_ns, false)) { failed = true; break; }
        }

        // ---- main pass
        a.tile0_mul = pl.tpc;
        a.tile_step = 1;
        a.tiles_per_cta = pl.tpc;
        a.KP = pl.KP;
        a.kwrite = pl.KP;
        a.push_tau = pl.push_tau;
        a.fullmin = pl.certify ? p.fullmin : nullptr;
        fence_proxy_async();
        __syncthreads();
        if (scans && !tc_pass<FP8 ? TCK_FP8 : TCK_BF16, EPI>(&tmX, &p.tmQ[slot], a, sm, s_tmem, run, &s_abort, qtile,
                                        rgrp)) {
            failed = true;
            break;
        }
        if (!sv_grid_sync(p.ctl, p.bar_ns, false)) { failed = true; break; }

        // ---- per-query merge and re-rank, into the host-mapped results
        {
            FvHit *out = p.out + (size_t)slot * p.max_batch * p.max_k;
            uint32_t *ocnt = p.out_cnt + (size_t)slot * p.max_batch;
            uint8_t *ounc = pl.certify ? p.out_unc + (size_t)slot * p.max_batch : nullptr;
            const bool exact = pl.S == pl.topb;  // certified: the keys are exact distances
            for (int q = blockIdx.x; q < pl.nq; q += G) {
                FvHit *mo = exact ? out : p.cand;
                uint32_t *mc = exact ? ocnt : p.ccnt;
                if (pl.S <= 32)
                    dense_top32_query(q, (uint64_t(*)[32])mkeys, p.dense, pl.dcap, p.dcnt, 0,
                                      a.fullmin, p.tau, pl.S, qprog, p.popcnt, p.nrows, mo, mc,
                                      p.ctr, nullptr, ounc);
                else
                    dense_merge_query(q, mkeys, p.dense, pl.dcap, stage_cap, p.dcnt, 0,
                                      a.fullmin, p.tau, pl.S, qprog, p.popcnt, p.nrows, mo, mc,
                                      p.ctr, nullptr, ounc);
                if (!exact)
                    rerank_query<NT>(q, mkeys, p.vecs, p.dpad, qf, p.cand, p.ccnt, pl.S,
                                     (uint32_t)pl.topb, qprog, p.popcnt, p.nrows, out, ocnt,
                                     p.ctr);
            }
            __threadfence_system();
        }
        if (!sv_grid_sync(p.ctl, p.bar_ns, false)) { failed = true; break; }
        done++;
        if (blockIdx.x == 0 && tid == 0) {
            p.tstamp[slot * 2 + 1] = sm100::globaltimer();
            __threadfence_system();
            *(volatile unsigned long long *)&p.done[slot] = done;
            __threadfence_system();
            p.ctl->processed = done;
        }
    }
    if (failed && tid == 0) atomicExch(&p.ctl->failed, 1);
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(s_tmem, TC_TMEM_COLS);
    }
}

}  // namespace pv

using namespace pv;

struct PvServe {
    FvGpuIndex *g = nullptr;
    int max_batch = 0;
    uint32_t max_k = 0;
    int EPI = 2, NS = 2, KPcap = TC_MAX_LIST, grid = 0;
    size_t smem = 0;
    uint64_t idle_ns = 0, bar_ns = 0;
    cudaStream_t kstream = nullptr, cstream = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_launch = false;
    bool running = false;
    int last_exit = 0;   // 0 stopped / never ran, 1 idle, -1 a wait expired
    unsigned long long published = 0, completed = 0;
    int inject_skip = -1;
    // device
    SvCtl *ctl = nullptr;
    unsigned long long *tail = nullptr;
    Buf slots, qbuf, tmq, scratch;
    // host
    Buf slots_h{true};
    unsigned long long *tail_h = nullptr;  // pinned, one per publish slot
    void *mapped = nullptr;                // host-mapped results
    SvArgs args{};
    int insn_cap = 0, const_cap = 0;
    int last_fallback = 0, last_uncertain = 0;
    float last_ms = 0.f;
    std::mutex mu;
};

namespace {

size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

template <int EPI>
cudaError_t sv_launch_direct(PvServe *s) {
    const bool fp8 = s->g->precision == FV_GPU_PREC_FP8;
    CUtensorMap tmX;
    memcpy(&tmX, s->g->tmap_x, sizeof(tmX));
    void *params[2] = {&tmX, &s->args};
    const void *fn = fp8 ? (const void *)pserve_kernel<true, EPI> : (const void *)pserve_kernel<false, EPI>;
    return cudaLaunchCooperativeKernel(fn, dim3(s->grid), dim3(64 + 128 * EPI), params, s->smem,
                                       s->kstream);
}

cudaError_t sv_launch(PvServe *s) { return sv_launch_direct<1>(s); }

template <int EPI>
const void *sv_fn(bool fp8) {
    return fp8 ? (const void *)pserve_kernel<true, EPI> : (const void *)pserve_kernel<false, EPI>;
}

// (Re)starts the kernel: resets the control words, then launches (the
// captured graph when capture worked, else the cooperative launch itself).
int sv_start(PvServe *s, char *errbuf, size_t errlen) {
    SvCtl c{};
    c.processed = s->completed;
    c.stop = 0;
    c.skip_cta = s->inject_skip;
    s->inject_skip = -1;
    PV_CUDA_OK(cudaMemcpyAsync(s->ctl, &c, sizeof(c), cudaMemcpyHostToDevice, s->kstream), errbuf,
               errlen);
    PV_CUDA_OK(cudaStreamSynchronize(s->kstream), errbuf, errlen);
    if (s->exec) {
        PV_CUDA_OK(cudaGraphLaunch(s->exec, s->kstream), errbuf, errlen);
    } else {
        PV_CUDA_OK(sv_launch(s), errbuf, errlen);
    }
    s->running = true;
    return 0;
}

// After the kernel left: its exit (0 stopped, 1 idle, -1 a wait expired).
int sv_reap(PvServe *s, char *errbuf, size_t errlen) {
    PV_CUDA_OK(cudaStreamSynchronize(s->kstream), errbuf, errlen);
    SvCtl c;
    PV_CUDA_OK(cudaMemcpy(&c, s->ctl, sizeof(c), cudaMemcpyDeviceToHost), errbuf, errlen);
    s->running = false;
    s->last_exit = c.failed ? -1 : c.cmd == 2 ? 1 : 0;
    return 0;
}

int sv_stop(PvServe *s, char *errbuf, size_t errlen) {
    if (!s->running) return 0;
    static const int one = 1;
    PV_CUDA_OK(cudaMemcpyAsync(&s->ctl->stop, &one, 4, cudaMemcpyHostToDevice, s->cstream),
               errbuf, errlen);
    return sv_reap(s, errbuf, errlen);
}

bool sv_alive(PvServe *s) { return s->running && cudaStreamQuery(s->kstream) == cudaErrorNotReady; }

}  // namespace

extern "C" void pv_serve_free(PvServe *s) {
    if (!s) return;
    if (s->g) cudaSetDevice(s->g->device);
    char err[256];
    sv_stop(s, err, sizeof(err));
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->ctl) cudaFree(s->ctl);
    if (s->tail) cudaFree(s->tail);
    if (s->tail_h) cudaFreeHost(s->tail_h);
    if (s->mapped) cudaFreeHost(s->mapped);
    s->slots.release();
    s->qbuf.release();
    s->tmq.release();
    s->scratch.release();
    s->slots_h.release();
    if (s->kstream) cudaStreamDestroy(s->kstream);
    if (s->cstream) cudaStreamDestroy(s->cstream);
    delete s;
}

extern "C" PvServe *pv_serve_create(FvGpuIndex *g, int max_batch, uint32_t max_k,
                                    uint32_t idle_ms, char *errbuf, size_t errlen) {
    if (!g || max_batch < 1 || max_batch > FV_GPU_MAX_BATCH || max_k < 1 ||
        max_k > PV_SERVE_MAX_K || idle_ms < 1) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "serve: bad arguments");
        return nullptr;
    }
    if (!tc_supported(g)) {
        if (errbuf && errlen)
            snprintf(errbuf, errlen, "serve: the index needs a BF16 or FP8 upload");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    PvServe *s = new PvServe();
    s->g = g;
    s->max_batch = max_batch;
    s->max_k = max_k;
    s->idle_ns = (uint64_t)idle_ms * 1000000ull;
    s->bar_ns = 2000000000ull;
    auto fail = [&](const char *what, cudaError_t e) -> PvServe * {
        if (errbuf && errlen)
            snprintf(errbuf, errlen, "serve: %s%s%s", what, e != cudaSuccess ? ": " : "",
                     e != cudaSuccess ? cudaGetErrorString(e) : "");
        s->g = g;
        pv_serve_free(s);
        return nullptr;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(g->device)) != cudaSuccess) return fail("device", e);
    const bool fp8 = g->precision == FV_GPU_PREC_FP8;
    const int esz = fp8 ? 1 : 2;
    const int kblocks = g->kpad * esz / TC_KB_BYTES;
    // shape: one epilogue group (lists of 64 keys per query and part; two
    // groups would cap the 320 threads' registers below the kernel's
    // needs), as many stages as fit
    s->KPcap = TC_MAX_LIST;
    const size_t cap = 227 * 1024 - 16 * 1024;  // static shared memory of the bitmap phase
    s->EPI = 1;
    s->NS = 4;
    while (s->NS > 2 && tc_smem_bytes(kblocks, s->NS, s->KPcap, s->EPI) > cap) s->NS--;
    if (tc_smem_bytes(kblocks, s->NS, s->KPcap, s->EPI) > cap)
        return fail("rows too wide for the kernel's shared memory", cudaSuccess);
    s->smem = tc_smem_bytes(kblocks, s->NS, s->KPcap, s->EPI);
    const void *fn = sv_fn<1>(fp8);
    if ((e = raise_smem_limit(fn, s->smem)) != cudaSuccess) return fail("shared memory", e);
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 64 + 128 * s->EPI,
                                                           s->smem)) != cudaSuccess ||
        per_sm < 1)
        return fail("occupancy", e);
    s->grid = g->sm_count;  // one CTA per SM, all resident (cooperative launch)
    if ((e = cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail("streams", e);

    // row tensor map (the index's own)
    if (!g->tmap_x_ok) {
        CUtensorMap m;
        if (!tc_make_tmap(&m, g->d_vlow, fp8 ? TCK_FP8 : TCK_BF16, (uint64_t)g->kpad, g->count))
            return fail("tensor map", cudaSuccess);
        memcpy(g->tmap_x, &m, sizeof(m));
        g->tmap_x_ok = true;
    }
    // slots: [plan][queries f32][qprog][progs][insns][consts]
    const int B = max_batch;
    s->insn_cap = std::max(64, 16 * B);
    s->const_cap = std::max(64, 32 * B);
    SvArgs &a = s->args;
    a.off_q = al(sizeof(SvPlan));
    a.off_qprog = a.off_q + al((size_t)B * g->dpad * 4);
    a.off_progs = a.off_qprog + al((size_t)B * 4);
    a.off_insns = a.off_progs + al((size_t)B * sizeof(PredProg));
    a.off_consts = a.off_insns + al((size_t)s->insn_cap * sizeof(PredInsn));
    a.slot_bytes = a.off_consts + al((size_t)s->const_cap * 8);
    if ((e = s->slots.ensure(SV_SLOTS * a.slot_bytes)) != cudaSuccess ||
        (e = s->slots_h.ensure(SV_SLOTS * a.slot_bytes)) != cudaSuccess)
        return fail("slots", e);
    const int nqpad = (B + TC_BM - 1) / TC_BM * TC_BM;
    a.qbuf_bytes = al((size_t)nqpad * g->kpad * esz);
    if ((e = s->qbuf.ensure(SV_SLOTS * a.qbuf_bytes)) != cudaSuccess) return fail("query tiles", e);
    {
        std::vector<CUtensorMap> maps(SV_SLOTS);
        for (int i = 0; i < SV_SLOTS; i++)
            if (!tc_make_tmap(&maps[i], s->qbuf.as<unsigned char>() + i * a.qbuf_bytes,
                              fp8 ? TCK_FP8 : TCK_BF16,
                              (uint64_t)g->kpad, (uint64_t)nqpad))
                return fail("tensor map", cudaSuccess);
        if ((e = s->tmq.ensure(sizeof(CUtensorMap) * SV_SLOTS)) != cudaSuccess ||
            (e = cudaMemcpy(s->tmq.p, maps.data(), sizeof(CUtensorMap) * SV_SLOTS,
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail("tensor maps", e);
    }
    // scratch: dense runs sized for the largest plan (lists per query x 64)
    const uint64_t max_lists = (uint64_t)s->grid * s->EPI * 4;
    const uint64_t dense_keys =
        std::max<uint64_t>((uint64_t)std::min(B, 32) * max_lists, (uint64_t)B * s->grid * s->EPI) *
        s->KPcap;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += al(bytes);
        return o;
    };
    const size_t o_qn = take((size_t)nqpad * 4), o_qs = take((size_t)nqpad * 4);
    const size_t o_tau = take((size_t)B * 8), o_fm = take((size_t)B * 8);
    const size_t o_dense = take((size_t)dense_keys * 8), o_dcnt = take((size_t)B * 4);
    const size_t o_cand = take((size_t)B * TC_MAX_SUPERSET * sizeof(FvHit));
    const size_t o_ccnt = take((size_t)B * 4), o_ctr = take((size_t)B);
    const size_t o_pop = take((size_t)B * 8), o_err = take(16);
    const size_t o_bm = take((size_t)B * ((g->count + 31) / 32) * 4);
    if ((e = s->scratch.ensure(off)) != cudaSuccess) return fail("scratch", e);
    if ((e = cudaMemset(s->scratch.p, 0, off)) != cudaSuccess) return fail("scratch", e);
    unsigned char *sc = s->scratch.as<unsigned char>();
    // control words, tail, host-mapped results
    if ((e = cudaMalloc(&s->ctl, sizeof(SvCtl))) != cudaSuccess ||
        (e = cudaMalloc(&s->tail, 8)) != cudaSuccess || (e = cudaMemset(s->tail, 0, 8)) != cudaSuccess ||
        (e = cudaMallocHost(&s->tail_h, 8 * SV_SLOTS)) != cudaSuccess)
        return fail("control", e);
    const size_t m_out = al((size_t)SV_SLOTS * B * max_k * sizeof(FvHit));
    const size_t m_cnt = al((size_t)SV_SLOTS * B * 4), m_unc = al((size_t)SV_SLOTS * B);
    const size_t m_done = al(SV_SLOTS * 8), m_ts = al(SV_SLOTS * 16);
    const size_t mbytes = m_out + m_cnt + m_unc + m_done + m_ts;
    if ((e = cudaHostAlloc(&s->mapped, mbytes, cudaHostAllocMapped)) != cudaSuccess)
        return fail("mapped results", e);
    memset(s->mapped, 0, mbytes);
    unsigned char *md = nullptr;
    if ((e = cudaHostGetDevicePointer((void **)&md, s->mapped, 0)) != cudaSuccess)
        return fail("mapped results", e);

    a.nrows = g->count;
    a.dim = g->dim;
    a.dpad = g->dpad;
    a.kpad = g->kpad;
    a.kblocks = kblocks;
    a.NS = s->NS;
    a.KPcap = s->KPcap;
    a.ncols = g->ncols;
    a.vecs = g->d_vecs;
    a.xnorm = g->d_norm;
    a.xscale = g->d_vscale;
    a.cols = g->d_cols;
    a.ctl = s->ctl;
    a.tail = s->tail;
    a.slots = s->slots.as<unsigned char>();
    a.qbuf = s->qbuf.as<unsigned char>();
    a.tmQ = s->tmq.as<const CUtensorMap>();
    a.qnorm = (float *)(sc + o_qn);
    a.qscale = (float *)(sc + o_qs);
    a.tau = (unsigned long long *)(sc + o_tau);
    a.fullmin = (unsigned long long *)(sc + o_fm);
    a.dense = (uint64_t *)(sc + o_dense);
    a.dcnt = (uint32_t *)(sc + o_dcnt);
    a.cand = (FvHit *)(sc + o_cand);
    a.ccnt = (uint32_t *)(sc + o_ccnt);
    a.ctr = (uint8_t *)(sc + o_ctr);
    a.popcnt = (unsigned long long *)(sc + o_pop);
    a.bitmaps = (uint32_t *)(sc + o_bm);
    a.err = (int *)(sc + o_err);
    a.out = (FvHit *)md;
    a.out_cnt = (uint32_t *)(md + m_out);
    a.out_unc = (uint8_t *)(md + m_out + m_cnt);
    a.done = (unsigned long long *)(md + m_out + m_cnt + m_unc);
    a.tstamp = (unsigned long long *)(md + m_out + m_cnt + m_unc + m_done);
    a.max_batch = B;
    a.max_k = (int)max_k;
    a.idle_ns = s->idle_ns;
    a.bar_ns = s->bar_ns;
    a.timeout_ns = 2000000000ull;
    a.drain_ns = 2000000000ull;
    // (everything below the barriers: 2 per stage, per accumulator and per
    // norm slot, plus the query-tile and drain barriers)
    a.merge_smem = s->smem - 1024 - (size_t)(2 * s->NS + 2 * TC_NACC + 2 + 2 * TC_NR) * 8;

    // capture the launch once; replays restart the kernel
    {
        cudaGraph_t graph = nullptr;
        cudaError_t c1 = cudaStreamBeginCapture(s->kstream, cudaStreamCaptureModeThreadLocal);
        cudaError_t c2 = c1 == cudaSuccess ? sv_launch(s) : c1;
        cudaError_t c3 = cudaStreamEndCapture(s->kstream, &graph);
        if (c1 == cudaSuccess && c2 == cudaSuccess && c3 == cudaSuccess && graph &&
            cudaGraphInstantiate(&s->exec, graph, 0) == cudaSuccess) {
            s->graph_launch = true;
        } else {
            s->exec = nullptr;
            s->graph_launch = false;
        }
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();  // a refused capture leaves no sticky error
    }
    return s;
}

namespace {

// Plan of one batch, as the one-shot launch shapes it (launch_scan_tc).
bool sv_plan(PvServe *s, int nq, uint32_t topb, float q_amax, SvPlan &pl) {
    FvGpuIndex *g = s->g;
    const int S = tc_superset(g, topb, q_amax);
    if (!S) return false;
    const int KP = S < TC_MAX_LIST ? S : TC_MAX_LIST;
    memset(&pl, 0, sizeof(pl));
    pl.nq = nq;
    pl.qtiles = (nq + TC_BM - 1) / TC_BM;
    pl.nqpad = pl.qtiles * TC_BM;
    int R = 1;
    if (pl.qtiles == 1) R = nq <= 32 ? 4 : nq <= 64 ? 2 : 1;
    while (R > 1 && (TC_BM / R < nq || TC_BN / R < 32)) R >>= 1;
    pl.rep = R;
    pl.bq = pl.qtiles == 1 && R > 1 ? TC_BM / R : pl.nqpad;
    const uint64_t ntiles_all = (g->count + TC_BN - 1) / TC_BN;
    int grow = s->grid / pl.qtiles;
    if (grow < 1) grow = 1;
    const uint64_t maxg = (ntiles_all + 3) / 4;
    if ((uint64_t)grow > maxg) grow = (int)maxg;
    const uint64_t tpc = (ntiles_all + grow - 1) / grow;
    grow = (int)((ntiles_all + tpc - 1) / tpc);
    pl.grow = grow;
    pl.tpc = tpc;
    pl.S = S;
    pl.KP = KP;
    pl.push_tau = KP == S;
    pl.certify = KP < S;
    pl.topb = (int)topb;
    const int nlists = grow * s->EPI * R;
    pl.dcap = (uint64_t)nlists * KP;
    pl.seed = ntiles_all >= 8 * (uint64_t)grow;
    if (pl.seed) {
        const uint64_t region = ntiles_all / grow;
        const uint64_t m = std::min<uint64_t>(std::min<uint64_t>(8, region),
                                              std::max<uint64_t>(1, ((uint64_t)S + 15) / 16));
        pl.seed_mul = region;
        pl.seed_step = std::max<uint64_t>(1, region / m);
        pl.seed_tiles = m;
        pl.seed_kwrite = std::min(KP, std::max(2, (4 * S + nlists - 1) / std::max(1, nlists)));
    }
    return true;
}

}  // namespace

extern "C" int pv_serve_run(PvServe *s, int nq, const float *queries, const FvGpuQueryDesc *qd,
                            const FvGpuPredNode *nodes, int nnodes, const int32_t *children,
                            int nchildren, const double *invals, int ninvals, const uint32_t *k,
                            FvHit *out, uint32_t *out_cnt, float *device_ms, char *errbuf,
                            size_t errlen) {
    if (!s || nq < 1 || nq > s->max_batch || !queries || !qd || !k || !out || !out_cnt) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "serve: bad batch");
        return -1;
    }
    uint32_t kmax = 0;
    for (int i = 0; i < nq; i++) {
        if (k[i] < 1 || k[i] > s->max_k) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "serve: k[%d]=%u outside 1..%u", i, k[i], s->max_k);
            return -1;
        }
        kmax = std::max(kmax, k[i]);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    FvGpuIndex *g = s->g;
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return -1;
    const float q_amax = pv_integral_amax(queries, (uint64_t)nq * g->dim);
    SvPlan pl;
    bool ok = sv_plan(s, nq, kmax, q_amax, pl);
    ok = ok && (int)pb.insns.size() <= s->insn_cap && (int)pb.consts.size() <= s->const_cap &&
         (int)pb.progs.size() <= s->max_batch;
    // lazy filters only when every filter is broad (see PV_LAZY_MIN_PASS)
    pl.lazy = 1;
    for (size_t p = 0; p < pb.progs.size() && pl.lazy; p++)
        pl.lazy = prog_pass_estimate(g, pb.insns.data() + pb.progs[p].insn0, pb.progs[p].ninsn,
                                     pb.consts.data()) >= PV_LAZY_MIN_PASS;
    pl.P = (int)pb.progs.size();
    pl.ninsns = (int)pb.insns.size();
    s->last_fallback = 0;
    s->last_uncertain = 0;
    if (!ok) {
        // not for the kernel (capacities):
        // the index's ordinary path, with the GPU released
        s->last_fallback = 1;
        if (sv_stop(s, errbuf, errlen)) return -1;
        std::lock_guard<std::mutex> lg(g->mu);
        std::vector<FvHit> o((size_t)nq * kmax);
        std::vector<uint8_t> tr(nq);
        if (brute_run_host(g, nq, queries, pb, kmax,
                           g->precision != FV_GPU_PREC_FP32 ? PV_MODE_LOW : PV_MODE_EXACT,
                           o.data(), out_cnt, tr.data(), errbuf, errlen))
            return -1;
        for (int q = 0; q < nq; q++) {
            out_cnt[q] = std::min(out_cnt[q], k[q]);
            memcpy(out + (size_t)q * s->max_k, &o[(size_t)q * kmax], sizeof(FvHit) * out_cnt[q]);
        }
        if (device_ms) *device_ms = g->last_kernel_ms;
        return 0;
    }
    // stage into the next slot (the kernel finished with it: batches run in order)
    const unsigned long long seq = ++s->published;
    const int slot = (int)((seq - 1) % SV_SLOTS);
    SvArgs &a = s->args;
    pl.seq = seq;
    pl.nconsts = (int)pb.consts.size();
    unsigned char *h = s->slots_h.as<unsigned char>() + (size_t)slot * a.slot_bytes;
    memcpy(h, &pl, sizeof(pl));
    float *hq = (float *)(h + a.off_q);
    for (int q = 0; q < nq; q++) {
        memcpy(hq + (size_t)q * g->dpad, queries + (size_t)q * g->dim, (size_t)g->dim * 4);
        if (g->dpad > g->dim) memset(hq + (size_t)q * g->dpad + g->dim, 0, (size_t)(g->dpad - g->dim) * 4);
    }
    memcpy(h + a.off_qprog, pb.qprog.data(), (size_t)nq * 4);
    if (!pb.progs.empty()) memcpy(h + a.off_progs, pb.progs.data(), pb.progs.size() * sizeof(PredProg));
    if (!pb.insns.empty()) memcpy(h + a.off_insns, pb.insns.data(), pb.insns.size() * sizeof(PredInsn));
    if (!pb.consts.empty()) memcpy(h + a.off_consts, pb.consts.data(), pb.consts.size() * 8);
    const size_t bytes = a.off_consts + pb.consts.size() * 8;
    PV_CUDA_OK(cudaMemcpyAsync(s->slots.as<unsigned char>() + (size_t)slot * a.slot_bytes, h, bytes,
                               cudaMemcpyHostToDevice, s->cstream),
               errbuf, errlen);
    s->tail_h[slot] = seq;  // published after the data, on the same stream
    PV_CUDA_OK(cudaMemcpyAsync(s->tail, &s->tail_h[slot], 8, cudaMemcpyHostToDevice, s->cstream),
               errbuf, errlen);
    volatile unsigned long long *done =
        (volatile unsigned long long *)((unsigned char *)s->mapped +
                                        ((unsigned char *)a.done - (unsigned char *)a.out));
    // wait for the batch; restart the kernel when it is not running
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        if (done[slot] >= seq) break;
        if (!sv_alive(s)) {
            // a kernel that left with a failure while this batch waited (an
            // earlier failure is history: the kernel is simply started again)
            const bool reaped = s->running;
            if (reaped && sv_reap(s, errbuf, errlen)) return -1;
            if (reaped && s->last_exit < 0) {
                snprintf(errbuf, errlen, "serve: a wait of the persistent kernel expired");
                // the batch was not taken: rewind the queue, so a restarted
                // kernel never takes this slot before its next batch lands
                s->published = s->completed;
                s->tail_h[slot] = s->completed;
                cudaMemcpyAsync(s->tail, &s->tail_h[slot], 8, cudaMemcpyHostToDevice,
                                s->cstream);  // after the batch's own copies
                cudaStreamSynchronize(s->cstream);
                return -1;
            }
            if (done[slot] >= seq) break;
            if (sv_start(s, errbuf, errlen)) return -1;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(30)) {
            snprintf(errbuf, errlen, "serve: batch not answered in 30 s");
            return -1;
        }
        std::this_thread::yield();
    }
    s->completed = seq;
    // results (host-mapped): stride max_k, each query keeps min(k, found)
    const FvHit *ho = (const FvHit *)s->mapped + (size_t)slot * s->max_batch * s->max_k;
    const uint8_t *mb = (const uint8_t *)s->mapped;
    const uint32_t *hc = (const uint32_t *)(mb + ((unsigned char *)a.out_cnt - (unsigned char *)a.out)) +
                         (size_t)slot * s->max_batch;
    const uint8_t *hu = mb + ((unsigned char *)a.out_unc - (unsigned char *)a.out) + (size_t)slot * s->max_batch;
    const unsigned long long *ts =
        (const unsigned long long *)(mb + ((unsigned char *)a.tstamp - (unsigned char *)a.out));
    for (int q = 0; q < nq; q++) {
        const uint32_t c = std::min(std::min(hc[q], kmax), k[q]);
        memcpy(out + (size_t)q * s->max_k, ho + (size_t)q * kmax, sizeof(FvHit) * c);
        out_cnt[q] = c;
    }
    s->last_ms = (float)((double)(ts[slot * 2 + 1] - ts[slot * 2]) / 1e6);
    if (device_ms) *device_ms = s->last_ms;
    if (pl.certify) {
        std::vector<uint8_t> unc(hu, hu + nq);
        int n = 0;
        for (int q = 0; q < nq; q++) n += unc[q] ? 1 : 0;
        if (n) {
            // superset not certified: exact re-runs on the ordinary path
            if (sv_stop(s, errbuf, errlen)) return -1;
            std::lock_guard<std::mutex> lg(g->mu);
            std::vector<FvHit> o((size_t)nq * kmax);
            std::vector<uint32_t> oc(nq);
            std::vector<uint8_t> tr(nq);
            if (redo_flagged(g, nq, queries, pb, kmax, unc.data(), o.data(), oc.data(), tr.data(),
                             errbuf, errlen))
                return -1;
            for (int q = 0; q < nq; q++)
                if (unc[q]) {
                    out_cnt[q] = std::min(oc[q], k[q]);
                    memcpy(out + (size_t)q * s->max_k, &o[(size_t)q * kmax],
                           sizeof(FvHit) * out_cnt[q]);
                }
            s->last_uncertain = n;
        }
    }
    return 0;
}

extern "C" int pv_serve_status(PvServe *s, int *running, int *last_exit, uint64_t *batches,
                               int *graph_launch, int *fallback, int *uncertain) {
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->running && !sv_alive(s)) {
        char err[256];
        if (sv_reap(s, err, sizeof(err))) return -1;
    }
    if (running) *running = s->running ? 1 : 0;
    if (last_exit) *last_exit = s->last_exit;
    if (batches) *batches = s->completed;
    if (graph_launch) *graph_launch = s->graph_launch ? 1 : 0;
    if (fallback) *fallback = s->last_fallback;
    if (uncertain) *uncertain = s->last_uncertain;
    return 0;
}

extern "C" int pv_serve_stop(PvServe *s, char *errbuf, size_t errlen) {
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    PV_CUDA_OK(cudaSetDevice(s->g->device), errbuf, errlen);
    return sv_stop(s, errbuf, errlen);
}

extern "C" int pv_serve_limits(PvServe *s, uint32_t idle_ms, uint32_t barrier_ms, int skip_cta) {
    if (!s || idle_ms < 1 || barrier_ms < 1 || skip_cta < -1 || skip_cta >= s->grid) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    char err[256];
    if (sv_stop(s, err, sizeof(err))) return -1;  // limits take effect at the next start
    s->idle_ns = (uint64_t)idle_ms * 1000000ull;
    s->bar_ns = (uint64_t)barrier_ms * 1000000ull;
    s->args.idle_ns = s->idle_ns;
    s->args.bar_ns = s->bar_ns;
    s->inject_skip = skip_cta;
    // the captured launch holds the old arguments: re-capture
    if (s->exec) {
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(s->kstream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            cudaError_t c2 = sv_launch(s);
            cudaError_t c3 = cudaStreamEndCapture(s->kstream, &graph);
            if (c2 != cudaSuccess || c3 != cudaSuccess || !graph ||
                cudaGraphInstantiate(&s->exec, graph, 0) != cudaSuccess)
                s->exec = nullptr;
        }
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        s->graph_launch = s->exec != nullptr;
    }
    return 0;
}
