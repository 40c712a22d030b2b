// stream.cu — executor for an arrival stream of uneven micro-batches.
//
// No reference counterpart: the reference worker issues each micro-batch
// as separate synchronous launches (worker.c:268-276 through
// fv_gpu_brute_batch). Here a PvStream prepares, per batch-size bucket
// (1, 2, 4, ... max_batch queries) and result-width bucket, ONE CUDA graph
// holding the whole device side of a micro-batch:
//     H2D of the staged batch -> predicate bitmaps -> scan (tensor-core
//     reduced precision + exact FP32 re-rank, or the exact FP32 scan) ->
//     merge -> D2H of the results,
// and replays it for every micro-batch that falls in the bucket. A batch is
// padded up to its bucket (extra queries repeat the last one and their
// results are discarded); its predicates ride in a fixed-capacity section
// whose actual sizes the bitmap kernel reads on the device, so one graph
// serves batches with any mix of filters and k (k <= the bucket's width;
// each query keeps its own k results). The scan of one bucket is one
// launch of one CTA per SM (or per tuned count), each walking its rows for
// the batch's query tile.
//
// Shapes are picked by measurement: at creation the autotuner times every
// candidate scan shape of each bucket on the caller's sample queries (CUDA
// events, median of runs) and keeps the fastest; the choices are saved to
// a text file and reused when it matches the index.
//
// Graphs run on a view of the index (pv::index_view): its own stream and
// scratch, so captured addresses never move. Queries whose reduced-
// precision superset cannot be certified are re-run exactly on the index.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "paves_ext.h"
#include "pv_internal.h"

using namespace pv;

namespace {

struct Bucket {
    int B = 0;
    uint32_t topb = 0;
    int insn_cap = 0, const_cap = 0;
    Buf stage_h{true}, stage_d, out_h{true}, out_d;
    DevBatch db;
    size_t o_cnt = 0, o_tr = 0, obytes = 0;
    // tuned plan
    int mode = PV_MODE_EXACT, epi = 0, ns = 0, grow = 0;
    float ms = 0.f;
    const uint8_t *d_unc = nullptr;  // certificate flags of the TC merge (if any)
    int *d_err = nullptr;            // watchdog word of the TC scan (if any)
    cudaGraphExec_t exec = nullptr;
};

size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct PvStream {
    FvGpuIndex *g = nullptr;  // owner of the device data; exact re-runs
    FvGpuIndex *v = nullptr;  // view that runs the graphs
    int max_batch = 0;
    uint32_t max_k = 0;
    std::vector<Bucket *> buckets;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::mutex mu;
    int last_uncertain = 0;
    int last_fallback = 0;
};

namespace {

void layout(Bucket &b, const FvGpuIndex *g) {
    const int B = b.B;
    b.insn_cap = std::max(64, B * 8);
    b.const_cap = std::max(64, B * 8);
    DevBatch &db = b.db;
    db.nq = B;
    db.P = g->ncols > 0 ? B : 0;
    db.ninsns = b.insn_cap;
    db.nconsts = b.const_cap;
    db.counts_on_device = true;
    db.q_amax = -1.f;  // no exactness certificate from the queries: superset 4k
    db.off_q = 0;
    db.off_qprog = al((size_t)B * g->dpad * 4);
    db.off_progs = db.off_qprog + al((size_t)B * 4);
    db.off_insns = db.off_progs + al((size_t)B * sizeof(PredProg) + 8);
    db.off_consts = db.off_insns + al((size_t)b.insn_cap * sizeof(PredInsn));
    db.off_counts = db.off_consts + al((size_t)b.const_cap * 8);
    db.off_extra = db.off_counts + al(16);
    db.bytes = db.off_extra;
    db.stage_h = &b.stage_h;
    db.stage_d = &b.stage_d;
    b.o_cnt = al((size_t)B * b.topb * sizeof(FvHit));
    b.o_tr = b.o_cnt + al((size_t)B * 4);
    b.obytes = b.o_tr + al((size_t)B);
}

int alloc(Bucket &b, char *errbuf, size_t errlen) {
    PV_CUDA_OK(b.stage_h.ensure(b.db.bytes), errbuf, errlen);
    PV_CUDA_OK(b.stage_d.ensure(b.db.bytes), errbuf, errlen);
    PV_CUDA_OK(b.out_h.ensure(b.obytes), errbuf, errlen);
    PV_CUDA_OK(b.out_d.ensure(b.obytes), errbuf, errlen);
    memset(b.stage_h.p, 0, b.db.bytes);
    return 0;
}

// Writes nq queries (padded to B by repeating the last) and the compiled
// predicates into the bucket's staging buffer. Returns 1 if the predicates
// exceed the bucket's capacities.
int stage(Bucket &b, const FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
          const FvGpuIndex *owner = nullptr) {
    const int P = (int)pb.progs.size();
    if (P > b.db.P || (int)pb.insns.size() > b.insn_cap || (int)pb.consts.size() > b.const_cap)
        return 1;
    char *h = b.stage_h.as<char>();
    float *hq = (float *)(h + b.db.off_q);
    int32_t *qp = (int32_t *)(h + b.db.off_qprog);
    for (int q = 0; q < b.B; q++) {
        const int src = q < nq ? q : nq - 1;
        memcpy(hq + (size_t)q * g->dpad, queries + (size_t)src * g->dim, (size_t)g->dim * 4);
        if (g->dpad > g->dim) memset(hq + (size_t)q * g->dpad + g->dim, 0, (size_t)(g->dpad - g->dim) * 4);
        qp[q] = pb.qprog[src];
    }
    if (P) memcpy(h + b.db.off_progs, pb.progs.data(), (size_t)P * sizeof(PredProg));
    if (!pb.insns.empty())
        memcpy(h + b.db.off_insns, pb.insns.data(), pb.insns.size() * sizeof(PredInsn));
    if (!pb.consts.empty())
        memcpy(h + b.db.off_consts, pb.consts.data(), pb.consts.size() * 8);
    // lazy filters (tensor-core buckets whose programs are all broad range
    // forms): no bitmaps, the scan tests a query's filter only on rows that
    // beat its threshold, instead of one full bitmap per query
    bool lazy = b.mode == PV_MODE_LOW && owner != nullptr;
    for (int p = 0; p < P && lazy; p++) {
        const PredProg &pp = pb.progs[p];
        lazy = prog_pass_estimate(owner, pb.insns.data() + pp.insn0, pp.ninsn,
                                  pb.consts.data()) >= PV_LAZY_MIN_PASS;
    }
    int32_t *cnt = (int32_t *)(h + b.db.off_counts);
    cnt[0] = lazy ? 0 : P;
    cnt[1] = (int)pb.insns.size();
    cnt[2] = (int)pb.consts.size();
    cnt[3] = lazy ? 1 : 0;
    return 0;
}

// The device side of one micro-batch on the view, in stream order.
int enqueue(PvStream *s, Bucket &b, char *errbuf, size_t errlen) {
    FvGpuIndex *v = s->v;
    v->tune_epi = b.epi;
    v->tune_ns = b.ns;
    v->tune_grow = b.grow;
    PV_CUDA_OK(cudaMemcpyAsync(b.stage_d.p, b.stage_h.p, b.db.bytes, cudaMemcpyHostToDevice,
                               v->stream),
               errbuf, errlen);
    char *od = b.out_d.as<char>();
    if (brute_launch(v, b.db, b.topb, b.mode, (FvHit *)od, (uint32_t *)(od + b.o_cnt),
                     (uint8_t *)(od + b.o_tr), errbuf, errlen))
        return -1;
    b.d_unc = v->tc_unc;
    b.d_err = v->tc_err;
    PV_CUDA_OK(cudaMemcpyAsync(b.out_h.p, od, b.obytes, cudaMemcpyDeviceToHost, v->stream),
               errbuf, errlen);
    return 0;
}

std::string tune_key(const FvGpuIndex *g, const Bucket &b) {
    char k[128];
    snprintf(k, sizeof(k), "%llu %d %d %d %u", (unsigned long long)g->count, g->dim, g->precision,
             b.B, b.topb);
    return k;
}

bool load_tune(const char *path, const FvGpuIndex *g, std::vector<Bucket *> &bs) {
    if (!path || !*path) return false;
    FILE *f = fopen(path, "r");
    if (!f) return false;
    char line[256];
    int found = 0;
    while (fgets(line, sizeof(line), f)) {
        unsigned long long cnt;
        int dim, prec, B, mode, epi, ns, grow;
        unsigned topb;
        float ms;
        if (sscanf(line, "pvtune1 %llu %d %d %d %u %d %d %d %d %f", &cnt, &dim, &prec, &B, &topb,
                   &mode, &epi, &ns, &grow, &ms) != 10)
            continue;
        if (cnt != g->count || dim != g->dim || prec != g->precision) continue;
        for (Bucket *b : bs)
            if (b->B == B && b->topb == topb && b->ms == 0.f) {
                b->mode = mode;
                b->epi = epi;
                b->ns = ns;
                b->grow = grow;
                b->ms = ms > 0.f ? ms : 1e-6f;
                found++;
            }
    }
    fclose(f);
    return found == (int)bs.size();
}

void save_tune(const char *path, const FvGpuIndex *g, const std::vector<Bucket *> &bs) {
    if (!path || !*path) return;
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "w");
    if (!f) return;
    for (const Bucket *b : bs)
        fprintf(f, "pvtune1 %s %d %d %d %d %.6f\n", tune_key(g, *b).c_str(), b->mode, b->epi,
                b->ns, b->grow, b->ms);
    fclose(f);
    rename(tmp.c_str(), path);
}

// Times one plan of a bucket: staged sample batch, 2 warm-up and 5 timed
// eager runs on the view, median device time.
int time_plan(PvStream *s, Bucket &b, float *ms, char *errbuf, size_t errlen) {
    FvGpuIndex *v = s->v;
    std::vector<float> t;
    for (int r = 0; r < 7; r++) {
        PV_CUDA_OK(cudaEventRecord(s->e0, v->stream), errbuf, errlen);
        if (enqueue(s, b, errbuf, errlen)) return -1;
        PV_CUDA_OK(cudaEventRecord(s->e1, v->stream), errbuf, errlen);
        PV_CUDA_OK(cudaStreamSynchronize(v->stream), errbuf, errlen);
        if (check_tc_watchdog(v, errbuf, errlen)) return -1;
        float x = 0.f;
        cudaEventElapsedTime(&x, s->e0, s->e1);
        if (r >= 2) t.push_back(x);
    }
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return 0;
}

int autotune(PvStream *s, const float *tq, int ntq, char *errbuf, size_t errlen) {
    FvGpuIndex *v = s->v;
    std::vector<float> q((size_t)s->max_batch * v->dim);
    for (int i = 0; i < s->max_batch; i++)
        memcpy(&q[(size_t)i * v->dim], tq + (size_t)(i % ntq) * v->dim, sizeof(float) * v->dim);
    PredBatch none;
    none.qprog.assign(s->max_batch, -1);
    for (Bucket *b : s->buckets) {
        if (b->ms > 0.f) continue;
        stage(*b, v, b->B, q.data(), none);
        struct Cand { int mode, epi, ns, grow; };
        std::vector<Cand> cands = {{PV_MODE_EXACT, 0, 0, 0}};
        if (v->precision != FV_GPU_PREC_FP32 && tc_supported(v)) {
            const int qtiles = (b->B + 127) / 128;
            const int g1 = std::max(1, v->sm_count / qtiles);
            for (int epi : {1, 2})
                for (int ns : {2, 3, 4, 6, 8})
                    if (tc_shape_fits(v, b->topb, epi, ns))
                        for (int grow : {g1, std::max(1, g1 / 2)})
                            cands.push_back({PV_MODE_LOW, epi, ns, grow});
        }
        float best = INFINITY;
        Cand bc = cands[0];
        for (const Cand &c : cands) {
            b->mode = c.mode;
            b->epi = c.epi;
            b->ns = c.ns;
            b->grow = c.grow;
            float ms;
            if (time_plan(s, *b, &ms, errbuf, errlen)) return -1;
            if (ms < best) {
                best = ms;
                bc = c;
            }
        }
        b->mode = bc.mode;
        b->epi = bc.epi;
        b->ns = bc.ns;
        b->grow = bc.grow;
        b->ms = best;
    }
    return 0;
}

}  // namespace

extern "C" void pv_stream_free(PvStream *s) {
    if (!s) return;
    if (s->v) cudaSetDevice(s->v->device);
    for (Bucket *b : s->buckets) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        b->stage_h.release();
        b->stage_d.release();
        b->out_h.release();
        b->out_d.release();
        delete b;
    }
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    if (s->v) fv_gpu_index_free(s->v);
    delete s;
}

extern "C" PvStream *pv_stream_create(FvGpuIndex *g, int max_batch, uint32_t max_k,
                                      const float *tune_queries, int ntune,
                                      const char *tune_path, char *errbuf, size_t errlen) {
    if (!g || max_batch < 1 || max_batch > FV_GPU_MAX_BATCH || max_k < 1 ||
        max_k > PV_STREAM_MAX_K || !tune_queries || ntune < 1) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "stream: bad arguments");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    PvStream *s = new PvStream();
    s->g = g;
    s->max_batch = max_batch;
    s->max_k = max_k;
    auto fail = [&]() -> PvStream * {
        pv_stream_free(s);
        return nullptr;
    };
    if (cudaSetDevice(g->device) != cudaSuccess || !(s->v = index_view(g))) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "stream: cannot create the index view");
        return fail();
    }
    cudaEventCreate(&s->e0);
    cudaEventCreate(&s->e1);
    std::vector<uint32_t> widths;
    if (max_k > 16) widths = {16, max_k};
    else widths = {max_k};
    for (int B = 1;; B <<= 1) {
        const int bb = std::min(B, max_batch);
        for (uint32_t w : widths) {
            Bucket *b = new Bucket();
            b->B = bb;
            b->topb = w;
            layout(*b, g);
            s->buckets.push_back(b);
            if (alloc(*b, errbuf, errlen)) return fail();
        }
        if (bb == max_batch) break;
    }
    // tuning: saved choices for this index, else measured now
    if (!load_tune(tune_path, g, s->buckets)) {
        if (autotune(s, tune_queries, ntune, errbuf, errlen)) return fail();
        save_tune(tune_path, g, s->buckets);
    }
    // size every scratch buffer of the view at its largest, then capture:
    // captured addresses stay valid because nothing grows afterwards
    {
        std::vector<float> q((size_t)max_batch * g->dim);
        for (int i = 0; i < max_batch; i++)
            memcpy(&q[(size_t)i * g->dim], tune_queries + (size_t)(i % ntune) * g->dim,
                   sizeof(float) * g->dim);
        PredBatch none;
        none.qprog.assign(max_batch, -1);
        for (Bucket *b : s->buckets) {
            stage(*b, g, b->B, q.data(), none);
            if (enqueue(s, *b, errbuf, errlen)) return fail();
            if (cudaStreamSynchronize(s->v->stream) != cudaSuccess ||
                check_tc_watchdog(s->v, errbuf, errlen))
                return fail();
        }
    }
    for (Bucket *b : s->buckets) {
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s->v->stream, cudaStreamCaptureModeThreadLocal);
        int rc = e == cudaSuccess ? enqueue(s, *b, errbuf, errlen) : -1;
        cudaError_t e2 = cudaStreamEndCapture(s->v->stream, &graph);
        if (e == cudaSuccess && rc == 0 && e2 == cudaSuccess)
            e = cudaGraphInstantiate(&b->exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess || rc != 0 || e2 != cudaSuccess || !b->exec) {
            if (errbuf && errlen && rc == 0)
                snprintf(errbuf, errlen, "stream: graph capture failed (%s)",
                         cudaGetErrorString(e != cudaSuccess ? e : e2));
            return fail();
        }
    }
    return s;
}

extern "C" int pv_stream_run(PvStream *s, int nq, const float *queries, const FvGpuQueryDesc *qd,
                             const FvGpuPredNode *nodes, int nnodes, const int32_t *children,
                             int nchildren, const double *invals, int ninvals,
                             const uint32_t *k, FvHit *out, uint32_t *out_cnt, float *device_ms,
                             char *errbuf, size_t errlen) {
    if (!s || nq < 1 || nq > s->max_batch || !queries || !qd || !k || !out || !out_cnt) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "stream: bad batch");
        return -1;
    }
    uint32_t kmax = 0;
    for (int i = 0; i < nq; i++) {
        if (k[i] < 1 || k[i] > s->max_k) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "stream: k[%d]=%u outside 1..%u", i, k[i], s->max_k);
            return -1;
        }
        kmax = std::max(kmax, k[i]);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    FvGpuIndex *v = s->v;
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, v->ncols, pb, errbuf, errlen) != 0)
        return -1;
    Bucket *b = nullptr;
    for (Bucket *c : s->buckets)
        if (c->B >= nq && c->topb >= kmax && (!b || c->B < b->B || (c->B == b->B && c->topb < b->topb)))
            b = c;
    s->last_fallback = 0;
    s->last_uncertain = 0;
    if (!b || stage(*b, v, nq, queries, pb, s->g)) {
        // predicates beyond the bucket's capacities: the index's own path
        s->last_fallback = 1;
        std::lock_guard<std::mutex> lg(s->g->mu);
        std::vector<FvHit> o((size_t)nq * kmax);
        std::vector<uint8_t> tr(nq);
        if (cudaSetDevice(s->g->device) != cudaSuccess) return -1;
        if (brute_run_host(s->g, nq, queries, pb, kmax,
                           s->g->precision != FV_GPU_PREC_FP32 ? PV_MODE_LOW : PV_MODE_EXACT,
                           o.data(), out_cnt, tr.data(), errbuf, errlen))
            return -1;
        for (int q = 0; q < nq; q++) {
            out_cnt[q] = std::min(out_cnt[q], k[q]);
            memcpy(out + (size_t)q * s->max_k, &o[(size_t)q * kmax], sizeof(FvHit) * out_cnt[q]);
        }
        if (device_ms) *device_ms = s->g->last_kernel_ms;
        return 0;
    }
    PV_CUDA_OK(cudaSetDevice(v->device), errbuf, errlen);
    PV_CUDA_OK(cudaEventRecord(s->e0, v->stream), errbuf, errlen);
    PV_CUDA_OK(cudaGraphLaunch(b->exec, v->stream), errbuf, errlen);
    PV_CUDA_OK(cudaEventRecord(s->e1, v->stream), errbuf, errlen);
    PV_CUDA_OK(cudaStreamSynchronize(v->stream), errbuf, errlen);
    v->tc_err = b->d_err;
    if (check_tc_watchdog(v, errbuf, errlen)) return -1;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->e0, s->e1);
    if (device_ms) *device_ms = ms;
    const char *oh = b->out_h.as<char>();
    const uint32_t *cnt = (const uint32_t *)(oh + b->o_cnt);
    for (int q = 0; q < nq; q++) {
        const uint32_t c = std::min(std::min(cnt[q], b->topb), k[q]);
        memcpy(out + (size_t)q * s->max_k, oh + (size_t)q * b->topb * sizeof(FvHit),
               sizeof(FvHit) * c);
        out_cnt[q] = c;
    }
    if (b->d_unc) {
        std::vector<uint8_t> unc(b->B);
        PV_CUDA_OK(cudaMemcpyAsync(unc.data(), b->d_unc, (size_t)b->B, cudaMemcpyDeviceToHost,
                                   v->stream),
                   errbuf, errlen);
        PV_CUDA_OK(cudaStreamSynchronize(v->stream), errbuf, errlen);
        int n = 0;
        for (int q = 0; q < nq; q++) n += unc[q] ? 1 : 0;
        if (n) {
            std::lock_guard<std::mutex> lg(s->g->mu);
            std::vector<FvHit> o((size_t)nq * b->topb);
            std::vector<uint32_t> oc(nq);
            std::vector<uint8_t> tr(nq);
            if (redo_flagged(s->g, nq, queries, pb, b->topb, unc.data(), o.data(), oc.data(),
                             tr.data(), errbuf, errlen))
                return -1;
            for (int q = 0; q < nq; q++)
                if (unc[q]) {
                    out_cnt[q] = std::min(oc[q], k[q]);
                    memcpy(out + (size_t)q * s->max_k, &o[(size_t)q * b->topb],
                           sizeof(FvHit) * out_cnt[q]);
                }
            s->last_uncertain = n;
        }
    }
    return 0;
}

extern "C" int pv_stream_info(PvStream *s, int i, int *B, uint32_t *topb, int *mode, int *epi,
                              int *ns, int *grow, float *tuned_ms) {
    if (!s) return -1;
    if (i < 0) return (int)s->buckets.size();
    if (i >= (int)s->buckets.size()) return -1;
    const Bucket *b = s->buckets[i];
    if (B) *B = b->B;
    if (topb) *topb = b->topb;
    if (mode) *mode = b->mode;
    if (epi) *epi = b->epi;
    if (ns) *ns = b->ns;
    if (grow) *grow = b->grow;
    if (tuned_ms) *tuned_ms = b->ms;
    return (int)s->buckets.size();
}

extern "C" int pv_stream_last(PvStream *s, int *uncertain, int *fallback) {
    if (!s) return -1;
    if (uncertain) *uncertain = s->last_uncertain;
    if (fallback) *fallback = s->last_fallback;
    return 0;
}
