// ext.cu — the additions declared in include/paves_ext.h.
#include <string.h>

#include "paves_ext.h"
#include "pv_internal.h"

using namespace pv;

struct PvBatch {
    FvGpuIndex *g = nullptr;
    Buf stage_h{true}, stage_d, out_d, out_h{true};
    DevBatch db;
    uint32_t topb = 0;
    int mode = 0;
    size_t off_cnt = 0, off_tr = 0, obytes = 0;
    cudaEvent_t ev[5] = {};
};

extern "C" int pv_pred_check(int nq, const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes,
                             int nnodes, const int32_t *children, int nchildren,
                             const double *invals, int ninvals, int ncols, int *nprog,
                             char *errbuf, size_t errlen) {
    if (nq < 1 || !qd) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: empty batch");
        return -1;
    }
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, ncols, pb, errbuf, errlen) != 0)
        return -1;
    if (nprog) *nprog = (int)pb.progs.size();
    return 0;
}

extern "C" PvBatch *pv_batch_create(FvGpuIndex *g, int nq, const float *queries,
                                    const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes,
                                    int nnodes, const int32_t *children, int nchildren,
                                    const double *invals, int ninvals, uint32_t topb, int mode,
                                    char *errbuf, size_t errlen) {
    if (!g || nq < 1 || nq > 65536 || topb == 0 || topb > FV_GPU_MAX_TOPB || !queries || !qd ||
        (mode != PV_MODE_EXACT && mode != PV_MODE_LOW) ||
        (mode == PV_MODE_LOW && g->precision == FV_GPU_PREC_FP32)) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: bad batch (nq=%d topb=%u mode=%d)", nq, topb, mode);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    if (cudaSetDevice(g->device) != cudaSuccess) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: cudaSetDevice failed");
        return nullptr;
    }
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return nullptr;
    PvBatch *b = new PvBatch();
    b->g = g;
    b->topb = topb;
    b->mode = mode;
    b->db.stage_h = &b->stage_h;
    b->db.stage_d = &b->stage_d;
    auto fail = [&](const char *what, cudaError_t e) -> PvBatch * {
        if (errbuf && errlen && what)
            snprintf(errbuf, errlen, "gpu: %s: %s", what, cudaGetErrorString(e));
        pv_batch_free(b);
        return nullptr;
    };
    if (brute_prepare(g, nq, queries, pb, b->db, 0, errbuf, errlen)) {
        pv_batch_free(b);
        return nullptr;
    }
    cudaError_t e = cudaMemcpyAsync(b->stage_d.p, b->stage_h.p, b->db.bytes,
                                    cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return fail("upload", e);
    const size_t hit = (size_t)nq * topb * sizeof(FvHit);
    b->off_cnt = (hit + 255) & ~(size_t)255;
    b->off_tr = b->off_cnt + (((size_t)nq * 4 + 255) & ~(size_t)255);
    b->obytes = b->off_tr + (size_t)nq;
    if ((e = b->out_d.ensure(b->obytes)) != cudaSuccess) return fail("alloc", e);
    if ((e = b->out_h.ensure(b->obytes)) != cudaSuccess) return fail("alloc", e);
    for (auto &v : b->ev)
        if ((e = cudaEventCreate(&v)) != cudaSuccess) return fail("event", e);
    return b;
}

extern "C" int pv_batch_run(PvBatch *b, int iters, float *stage_ms, float *total_ms,
                            char *errbuf, size_t errlen) {
    if (!b || iters < 1) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: bad run");
        return -1;
    }
    FvGpuIndex *g = b->g;
    std::lock_guard<std::mutex> lk(g->mu);
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    g->launches = 0;
    char *od = b->out_d.as<char>();
    float st[4] = {0, 0, 0, 0}, tot = 0.f;
    if (stage_ms) {
        for (int i = 0; i < iters; i++) {
            if (brute_launch(g, b->db, b->topb, b->mode, (FvHit *)od,
                             (uint32_t *)(od + b->off_cnt), (uint8_t *)(od + b->off_tr), errbuf,
                             errlen, b->ev))
                return -1;
            PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
            if (check_tc_watchdog(g, errbuf, errlen)) return -1;
            for (int s = 0; s < 4; s++) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, b->ev[s], b->ev[s + 1]);
                st[s] += ms;
                tot += ms;
            }
        }
        memcpy(stage_ms, st, sizeof(st));
    } else {
        cudaEventRecord(b->ev[0], g->stream);
        for (int i = 0; i < iters; i++)
            if (brute_launch(g, b->db, b->topb, b->mode, (FvHit *)od,
                             (uint32_t *)(od + b->off_cnt), (uint8_t *)(od + b->off_tr), errbuf,
                             errlen, nullptr))
                return -1;
        cudaEventRecord(b->ev[4], g->stream);
        PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
        if (check_tc_watchdog(g, errbuf, errlen)) return -1;
        cudaEventElapsedTime(&tot, b->ev[0], b->ev[4]);
    }
    if (total_ms) *total_ms = tot;
    return 0;
}

extern "C" int pv_batch_fetch(PvBatch *b, FvHit *out, uint32_t *out_cnt, uint8_t *truncated,
                              char *errbuf, size_t errlen) {
    if (!b || !out || !out_cnt || !truncated) return -1;
    FvGpuIndex *g = b->g;
    std::lock_guard<std::mutex> lk(g->mu);
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    // in the order of the batch's own stream
    PV_CUDA_OK(cudaMemcpyAsync(b->out_h.p, b->out_d.p, b->obytes, cudaMemcpyDeviceToHost,
                               g->stream),
               errbuf, errlen);
    PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
    const int nq = b->db.nq;
    const char *oh = b->out_h.as<char>();
    const uint32_t *cnt = (const uint32_t *)(oh + b->off_cnt);
    for (int q = 0; q < nq; q++) {
        uint32_t c = cnt[q] > b->topb ? b->topb : cnt[q];
        memcpy(out + (size_t)q * b->topb, oh + (size_t)q * b->topb * sizeof(FvHit),
               c * sizeof(FvHit));
        out_cnt[q] = c;
    }
    memcpy(truncated, oh + b->off_tr, (size_t)nq);
    // prepared batches report, and do not re-run, uncertified supersets
    g->last_uncertain = 0;
    if (g->tc_unc && g->tc_unc_n == nq) {
        std::vector<uint8_t> unc((size_t)nq);
        PV_CUDA_OK(cudaMemcpyAsync(unc.data(), g->tc_unc, (size_t)nq, cudaMemcpyDeviceToHost,
                                   g->stream),
                   errbuf, errlen);
        PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
        for (int q = 0; q < nq; q++) g->last_uncertain += unc[q] ? 1 : 0;
    }
    return 0;
}

extern "C" int pv_last_uncertain(const FvGpuIndex *g) { return g ? g->last_uncertain : 0; }

extern "C" void pv_batch_free(PvBatch *b) {
    if (!b) return;
    if (b->g) cudaSetDevice(b->g->device);
    for (auto &v : b->ev)
        if (v) cudaEventDestroy(v);
    b->stage_h.release();
    b->stage_d.release();
    b->out_d.release();
    b->out_h.release();
    delete b;
}

extern "C" float pv_last_kernel_ms(const FvGpuIndex *g) { return g ? g->last_kernel_ms : 0.f; }

extern "C" int pv_last_superset(const FvGpuIndex *g) { return g ? g->last_superset : 0; }

extern "C" int pv_last_launches(const FvGpuIndex *g) { return g ? g->launches : 0; }

extern "C" int pv_graph_stats(const FvGpuIndex *g, uint32_t *out, int nq) {
    if (!g || !out) return 0;
    int n = (int)(g->graph_stats.size() / 4);
    if (nq < n) n = nq;
    memcpy(out, g->graph_stats.data(), (size_t)n * 16);
    return n;
}

extern "C" int pv_last_sparse(const FvGpuIndex *g) { return g ? g->last_sparse : 0; }

extern "C" int pv_tc_shape(FvGpuIndex *g, int epi, int ns, int grow, int rep, int seed) {
    if (!g || epi < 0 || epi > 3 || ns < 0 || ns > 8 || grow < 0 ||
        !(rep == 0 || rep == 1 || rep == 2 || rep == 4) || seed < 0 || seed > 2)
        return -1;
    std::lock_guard<std::mutex> lk(g->mu);
    g->tune_epi = epi;
    g->tune_ns = ns;
    g->tune_grow = grow;
    g->tune_rep = rep;
    g->tune_seed = seed;
    return 0;
}

extern "C" int pv_tc_timeout(FvGpuIndex *g, uint64_t ns) {
    if (!g || ns > 10000000000ull) return -1;
    std::lock_guard<std::mutex> lk(g->mu);
    g->tc_timeout_ns = ns;
    return 0;
}

extern "C" int pv_tc_wide_superset(FvGpuIndex *g, int on) {
    if (!g || on < 0 || on > 1) return -1;
    std::lock_guard<std::mutex> lk(g->mu);
    g->force_wide_superset = on;
    return 0;
}

extern "C" int pv_exact_tc(FvGpuIndex *g, int on) {
    if (!g || on < 0 || on > 1) return -1;
    std::lock_guard<std::mutex> lk(g->mu);
    g->exact_tc = on;
    return 0;
}

extern "C" int pv_last_exact_tc(const FvGpuIndex *g) { return g ? g->last_exact_tc : 0; }

extern "C" int pv_filter_bound(const FvGpuIndex *g, const FvGpuPredNode *nodes, int nnodes,
                               const int32_t *children, int nchildren, const double *invals,
                               int ninvals, uint64_t *bound, char *errbuf, size_t errlen) {
    if (!g || !bound) return -1;
    FvGpuQueryDesc qd;
    memset(&qd, 0, sizeof(qd));
    qd.proot = nnodes > 0 ? 0 : -1;
    PredBatch pb;
    if (compile_predicates(1, &qd.proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return -1;
    if (pb.progs.empty()) {
        *bound = g->count;
        return 0;
    }
    *bound = prog_upper_bound(g, pb.insns.data() + pb.progs[0].insn0, pb.progs[0].ninsn,
                              pb.consts.data());
    return 0;
}
