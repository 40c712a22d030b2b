// arbiter.cpp — the GPU worker's micro-batch loop and its request slots,
// without PostgreSQL.
//
// Restates the protocol of extension/paves/src/arbiter.h:106-162,
// arbiter.c:108-269 and worker.c:149-598 with threads instead of processes:
//  * a fixed pool of slots with the state machine FREE -> FILLING ->
//    SUBMITTED -> RUNNING -> DONE | ERROR -> FREE (compare-and-swap, no
//    lock on the data path);
//  * backends fill a slot, mark it SUBMITTED, wake the worker and wait
//    (10 ms polls; a worker that is gone makes the backend reclaim its slot
//    and fall back, arbiter.c:210-251);
//  * the worker collects SUBMITTED slots, keeps the gathering window open
//    for up to wait_us (20 us polls) and leaves early after idle_us without
//    arrivals (worker.c:526-560), groups by (relid, strategy), orders graph
//    groups heaviest first (weight want / selectivity, worker.c:210-232),
//    runs one batch per group at the group's largest want, answers each
//    slot with its prefix min(cnt, want) translated to tids (out-of-range
//    ids dropped, worker.c:336-394), sets `more`, and updates the
//    per-(relid, strategy, selectivity bucket) service-time EWMAs
//    (worker.c:296-333).
// The batch itself goes through an executor: by default the drop-in C ABI
// (fv_gpu_brute_batch / fv_gpu_graph_batch); a host executor can be set
// for integration and for failure tests that must not involve a GPU.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "paves_ext.h"

namespace {

enum : uint32_t { S_FREE = 0, S_FILLING, S_SUBMITTED, S_RUNNING, S_DONE, S_ERROR };

int sel_bucket(int permille) {  // arbiter.h:50-60
    if (permille >= 200) return 0;
    if (permille >= 50) return 1;
    if (permille >= 10) return 2;
    if (permille >= 2) return 3;
    return 4;
}

struct Slot {
    std::atomic<uint32_t> state{S_FREE};
    // request
    uint32_t relid = 0;
    uint64_t ino = 0;
    int strategy = 0, dim = 0;
    uint32_t want = 0;
    uint64_t max_visited = 0;
    int sel_permille = 0;
    int nnodes = 0, nchildren = 0, ninvals = 0, nspans = 0, need_eval = 0, dedup = 0;
    float query[PV_ARB_MAX_DIM];
    FvGpuPredNode nodes[PV_ARB_MAX_NODES];
    int32_t children[PV_ARB_MAX_CHILDREN];
    double invals[PV_ARB_MAX_INVALS];
    FvGpuSpan spans[PV_ARB_MAX_SPANS];
    // response (FvHit.node carries the tid)
    uint32_t nresults = 0;
    uint8_t more = 0;
    FvHit results[PV_ARB_MAX_RESULTS];
};

struct Attached {
    uint32_t relid = 0;
    uint64_t ino = 0;
    FvGpuIndex *g = nullptr;
    const uint64_t *tids = nullptr;
    uint64_t count = 0;
    int dim = 0;
    // upper levels for the graph entry descent (may be absent)
    const float *vectors = nullptr;
    const uint64_t *upper_offs = nullptr;
    const uint32_t *upper = nullptr;
    uint32_t M = 0;
    int max_level = 0;
    uint64_t entry = 0;
};

struct Feedback {
    uint32_t relid = 0;
    std::atomic<uint32_t> q_us[2][5];
    std::atomic<uint32_t> batch_us[2];
    std::atomic<uint32_t> batch_n16[2];
    Feedback() {
        for (auto &r : q_us)
            for (auto &v : r) v = 0;
        for (auto &v : batch_us) v = 0;
        for (auto &v : batch_n16) v = 0;
    }
};

void ewma(std::atomic<uint32_t> &f, double sample, double alpha) {  // arbiter.h:237-245
    const uint32_t old = f.load();
    uint32_t nv = old == 0 ? (uint32_t)sample : (uint32_t)(old + alpha * (sample - old));
    f.store(nv > 1 ? nv : 1);
}

int default_exec(void *, const PvArbBatch *b) {
    char err[256];
    if (b->strategy == PV_STRAT_GPU_HNSW)
        return fv_gpu_graph_batch(b->g, b->nq, b->queries, b->qd, b->nodes, b->nnodes,
                                  b->children, b->nchildren, b->invals, b->ninvals, b->want,
                                  b->max_visited, b->out, b->out_cnt, b->flags, err,
                                  sizeof(err));
    return fv_gpu_brute_batch(b->g, b->nq, b->queries, b->qd, b->dedup, b->nodes, b->nnodes,
                              b->children, b->nchildren, b->invals, b->ninvals, b->spans,
                              b->nspans, b->spanoff, b->nspanoff, b->want, b->out, b->out_cnt,
                              b->flags, err, sizeof(err));
}

float l2sq(const float *a, const float *b, int d) {
    float s = 0.f;
    for (int i = 0; i < d; i++) {
        const float t = a[i] - b[i];
        s += t * t;
    }
    return s;
}

}  // namespace

struct PvArbiter {
    std::vector<Slot> slots;
    int batch_max, wait_us, idle_us;
    std::atomic<int> ready{0};
    std::atomic<int> stop{0};
    std::atomic<int> kill{0};  // injected failure: exit holding collected slots
    std::atomic<uint32_t> inflight{0};
    std::thread worker;
    std::mutex mu;  // wakeups only (data moves through the slot states)
    std::condition_variable wake_worker, wake_backends;
    std::mutex attach_mu;
    // a deque: push_back never moves its elements, so the pointer find()
    // hands the worker stays valid while pv_arbiter_attach adds indexes
    std::deque<Attached> indexes;
    std::vector<Feedback *> fb;
    pv_arb_exec_fn exec = default_exec;
    void *exec_ctx = nullptr;
    std::atomic<uint64_t> n_batches{0}, n_requests{0};

    explicit PvArbiter(int nslots) : slots(nslots) {}

    Feedback *feedback(uint32_t relid) {
        std::lock_guard<std::mutex> g(attach_mu);
        for (Feedback *f : fb)
            if (f->relid == relid) return f;
        Feedback *f = new Feedback();
        f->relid = relid;
        fb.push_back(f);
        return f;
    }

    const Attached *find(uint32_t relid) {
        std::lock_guard<std::mutex> g(attach_mu);
        for (const Attached &a : indexes)
            if (a.relid == relid) return &a;
        return nullptr;
    }

    int collect(std::vector<Slot *> &batch, int cap) {
        for (auto &s : slots) {
            if ((int)batch.size() >= cap) break;
            uint32_t e = S_SUBMITTED;
            if (s.state.compare_exchange_strong(e, S_RUNNING)) batch.push_back(&s);
        }
        return (int)batch.size();
    }

    void answer(Slot *s, uint32_t st) {
        s->state.store(st, std::memory_order_release);
        std::lock_guard<std::mutex> g(mu);
        wake_backends.notify_all();
    }

    void run_group(std::vector<Slot *> &grp);
    void run_batch(std::vector<Slot *> &batch) {
        while (!batch.empty()) {
            Slot *s0 = batch[0];
            std::vector<Slot *> grp, rest;
            for (Slot *s : batch)
                (s->relid == s0->relid && s->strategy == s0->strategy ? grp : rest).push_back(s);
            run_group(grp);
            batch.swap(rest);
        }
    }
    void loop();
};

void PvArbiter::run_group(std::vector<Slot *> &grp) {
    const Attached *ix = find(grp[0]->relid);
    std::vector<Slot *> ok;
    for (Slot *s : grp) {
        // dimension and index-file identity (worker.c:176-196)
        if (!ix || s->dim != ix->dim || s->ino != ix->ino) answer(s, S_ERROR);
        else ok.push_back(s);
    }
    if (ok.empty()) return;
    const int strategy = ok[0]->strategy;
    const int n = (int)ok.size();
    uint32_t want_max = 0;
    uint64_t mv_max = 0;
    for (Slot *s : ok) {
        want_max = std::max(want_max, s->want);
        mv_max = std::max(mv_max, s->max_visited);
    }
    auto weight = [](const Slot *s) { return (double)s->want * 1000.0 / std::max(s->sel_permille, 1); };
    if (strategy == PV_STRAT_GPU_HNSW && n > 2)
        std::stable_sort(ok.begin(), ok.end(),
                         [&](const Slot *a, const Slot *b) { return weight(a) > weight(b); });

    // concatenate and rebase the slots' predicate slices (engine.cpp:1232-1282)
    const int dim = ix->dim;
    std::vector<float> queries((size_t)n * dim);
    std::vector<FvGpuQueryDesc> qd(n);
    std::vector<uint8_t> dedup(n);
    std::vector<FvGpuPredNode> nodes;
    std::vector<int32_t> children;
    std::vector<double> invals;
    std::vector<FvGpuSpan> spans;
    std::vector<uint64_t> soff;
    const auto t0 = std::chrono::steady_clock::now();  // descent + batch (worker.c:258-279)
    for (int i = 0; i < n; i++) {
        const Slot *s = ok[i];
        memcpy(&queries[(size_t)i * dim], s->query, sizeof(float) * dim);
        FvGpuQueryDesc &d = qd[i];
        memset(&d, 0, sizeof(d));
        const int32_t bn = (int32_t)nodes.size(), bc = (int32_t)children.size(),
                      bv = (int32_t)invals.size();
        d.proot = s->nnodes > 0 ? bn : -1;
        d.need_eval = s->need_eval;
        dedup[i] = (uint8_t)s->dedup;
        for (int j = 0; j < s->nnodes; j++) {
            FvGpuPredNode x = s->nodes[j];
            x.child0 += bc;
            x.val0 += bv;
            nodes.push_back(x);
        }
        for (int j = 0; j < s->nchildren; j++) children.push_back(s->children[j] + bn);
        invals.insert(invals.end(), s->invals, s->invals + s->ninvals);
        d.span0 = (int32_t)spans.size();
        d.nspans = s->nspans;
        d.soff0 = (int32_t)soff.size();
        if (s->nspans > 0) {
            uint64_t tot = 0;
            for (int j = 0; j < s->nspans; j++) {
                soff.push_back(tot);
                tot += s->spans[j].hi - s->spans[j].lo;
                spans.push_back(s->spans[j]);
            }
            soff.push_back(tot);
            d.total = tot;
        } else {
            d.soff0 = 0;
            d.total = ix->count;
        }
        if (strategy == PV_STRAT_GPU_HNSW) {
            uint64_t ep = ix->entry;
            if (ix->vectors && ix->upper_offs && ix->upper) {
                const float *q = s->query;
                for (int lc = ix->max_level; lc >= 1; lc--) {
                    float dd = l2sq(q, ix->vectors + ep * dim, dim);
                    for (bool moved = true; moved;) {
                        moved = false;
                        const uint32_t *L =
                            ix->upper + ix->upper_offs[ep] + (uint64_t)(lc - 1) * (ix->M + 1);
                        for (uint32_t k = 0; k < L[0]; k++) {
                            const float nd = l2sq(q, ix->vectors + (uint64_t)L[1 + k] * dim, dim);
                            if (nd < dd) {
                                dd = nd;
                                ep = L[1 + k];
                                moved = true;
                            }
                        }
                    }
                }
            }
            d.entry = (uint32_t)ep;
        }
    }
    std::vector<FvHit> out((size_t)n * want_max);
    std::vector<uint32_t> cnt(n, 0);
    std::vector<uint8_t> flags(n, 0);
    PvArbBatch b;
    memset(&b, 0, sizeof(b));
    b.g = ix->g;
    b.strategy = strategy;
    b.nq = n;
    b.dim = dim;
    b.queries = queries.data();
    b.qd = qd.data();
    b.dedup = dedup.data();
    b.nodes = nodes.data();
    b.nnodes = (int)nodes.size();
    b.children = children.data();
    b.nchildren = (int)children.size();
    b.invals = invals.data();
    b.ninvals = (int)invals.size();
    b.spans = spans.data();
    b.nspans = (int)spans.size();
    b.spanoff = soff.data();
    b.nspanoff = (int)soff.size();
    b.want = want_max;
    b.max_visited = mv_max;
    b.out = out.data();
    b.out_cnt = cnt.data();
    b.flags = flags.data();
    const int rc = exec(exec_ctx, &b);
    const double T =
        std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    if (kill.load()) return;  // injected failure: die holding the RUNNING slots

    // service-time feedback per selectivity bucket, attributed by weight
    {
        Feedback *f = feedback(ix->relid);
        const int si = strategy == PV_STRAT_GPU_HNSW ? 1 : 0;
        double wmax = 0, wsum[5] = {0, 0, 0, 0, 0};
        int nb[5] = {0, 0, 0, 0, 0};
        for (Slot *s : ok) {
            const double w = si ? weight(s) : 1.0;
            wmax = std::max(wmax, w);
            const int bk = sel_bucket(s->sel_permille);
            wsum[bk] += w;
            nb[bk]++;
        }
        for (int bk = 0; bk < 5; bk++)
            if (nb[bk])
                ewma(f->q_us[si][bk], (T / std::max(wmax, 1e-9)) * (wsum[bk] / nb[bk]),
                     (double)nb[bk] / (nb[bk] + 64.0));
        ewma(f->batch_us[si], T, 0.125);
        ewma(f->batch_n16[si], n * 16.0, 0.125);
    }

    for (int i = 0; i < n; i++) {
        Slot *s = ok[i];
        if (rc < 0) {
            answer(s, S_ERROR);
            continue;
        }
        const uint32_t c = cnt[i];
        const uint32_t give = std::min(c, s->want);
        const FvHit *src = out.data() + (size_t)i * want_max;
        uint32_t kept = 0;
        for (uint32_t j = 0; j < give; j++) {
            if (src[j].node >= ix->count) continue;  // out-of-range row: dropped
            s->results[kept].node = ix->tids ? ix->tids[src[j].node] : src[j].node;
            s->results[kept].dist = src[j].dist;
            kept++;
        }
        s->nresults = kept;
        if (strategy == PV_STRAT_GPU_HNSW)
            s->more = (flags[i] == 0 || c > kept) ? 1 : 0;
        else
            s->more = (flags[i] != 0 || c > kept) ? 1 : 0;
        answer(s, S_DONE);
    }
}

void PvArbiter::loop() {
    ready.store(1);
    std::vector<Slot *> batch;
    while (!stop.load()) {
        batch.clear();
        int n = collect(batch, batch_max);
        if (n == 0) {
            std::unique_lock<std::mutex> lk(mu);
            wake_worker.wait_for(lk, std::chrono::milliseconds(100));
            continue;
        }
        // gathering window with early departure after idle_us
        if (wait_us > 0 && n < batch_max) {
            int waited = 0, idle = 0;
            while (waited < wait_us && n < batch_max) {
                std::this_thread::sleep_for(std::chrono::microseconds(20));
                waited += 20;
                const int got = collect(batch, batch_max);
                if (idle_us > 0) {
                    idle = got > n ? 0 : idle + 20;
                    if (idle >= idle_us) {
                        n = got;
                        break;
                    }
                }
                n = got;
            }
        }
        n_requests += (uint64_t)n;
        n_batches++;
        run_batch(batch);
        if (kill.load()) break;
    }
    ready.store(0);
    std::lock_guard<std::mutex> g(mu);
    wake_backends.notify_all();
}

extern "C" PvArbiter *pv_arbiter_create(int nslots, int batch_max, int wait_us, int idle_us) {
    if (nslots < 1 || nslots > 65536 || batch_max < 1) return nullptr;
    PvArbiter *a = new PvArbiter(nslots);
    a->batch_max = std::min(batch_max, FV_GPU_MAX_BATCH);
    a->wait_us = std::max(0, wait_us);
    a->idle_us = std::max(0, idle_us);
    a->worker = std::thread([a] { a->loop(); });
    while (!a->ready.load()) std::this_thread::yield();
    return a;
}

extern "C" int pv_arbiter_attach(PvArbiter *a, uint32_t relid, uint64_t ino, FvGpuIndex *g,
                                 const uint64_t *tids, uint64_t count, int dim,
                                 const float *vectors, const uint64_t *upper_offs,
                                 const uint32_t *upper, uint32_t M, int max_level,
                                 uint64_t entry) {
    if (!a || dim <= 0 || dim > PV_ARB_MAX_DIM || count == 0) return -1;
    std::lock_guard<std::mutex> gd(a->attach_mu);
    for (Attached &x : a->indexes)
        if (x.relid == relid) return -1;
    Attached x;
    x.relid = relid;
    x.ino = ino;
    x.g = g;
    x.tids = tids;
    x.count = count;
    x.dim = dim;
    x.vectors = vectors;
    x.upper_offs = upper_offs;
    x.upper = upper;
    x.M = M;
    x.max_level = max_level;
    x.entry = entry;
    a->indexes.push_back(x);
    return 0;
}

extern "C" void pv_arbiter_set_executor(PvArbiter *a, pv_arb_exec_fn fn, void *ctx) {
    if (!a) return;
    a->exec = fn ? fn : default_exec;
    a->exec_ctx = ctx;
}

extern "C" int pv_arbiter_submit(PvArbiter *a, uint32_t relid, uint64_t ino, int strategy,
                                 int dim, const float *query, const FvGpuPredNode *nodes,
                                 int nnodes, const int32_t *children, int nchildren,
                                 const double *invals, int ninvals, const FvGpuSpan *spans,
                                 int nspans, int need_eval, int dedup, uint32_t want,
                                 uint64_t max_visited, int sel_permille, FvHit *out,
                                 uint32_t *ncnt, uint8_t *more, int timeout_ms) {
    if (!a || a->ready.load() != 1) return 0;
    if (dim < 1 || dim > PV_ARB_MAX_DIM || want < 1 || want > PV_ARB_MAX_RESULTS ||
        nnodes > PV_ARB_MAX_NODES || nchildren > PV_ARB_MAX_CHILDREN ||
        ninvals > PV_ARB_MAX_INVALS || nspans > PV_ARB_MAX_SPANS || nnodes < 0 ||
        nchildren < 0 || ninvals < 0 || nspans < 0 ||
        (strategy != PV_STRAT_GPU_BRUTE && strategy != PV_STRAT_GPU_HNSW))
        return 0;  // capacity miss: caller keeps the query
    Slot *slot = nullptr;
    for (auto &s : a->slots) {
        uint32_t e = S_FREE;
        if (s.state.compare_exchange_strong(e, S_FILLING)) {
            slot = &s;
            break;
        }
    }
    if (!slot) return 0;  // queue full
    slot->relid = relid;
    slot->ino = ino;
    slot->strategy = strategy;
    slot->dim = dim;
    slot->want = want;
    slot->max_visited = max_visited;
    slot->sel_permille = sel_permille;
    slot->nnodes = nnodes;
    slot->nchildren = nchildren;
    slot->ninvals = ninvals;
    slot->nspans = nspans;
    slot->need_eval = need_eval;
    slot->dedup = dedup;
    memcpy(slot->query, query, sizeof(float) * dim);
    if (nnodes) memcpy(slot->nodes, nodes, sizeof(FvGpuPredNode) * nnodes);
    if (nchildren) memcpy(slot->children, children, sizeof(int32_t) * nchildren);
    if (ninvals) memcpy(slot->invals, invals, sizeof(double) * ninvals);
    if (nspans) memcpy(slot->spans, spans, sizeof(FvGpuSpan) * nspans);
    slot->state.store(S_SUBMITTED, std::memory_order_release);
    a->inflight++;
    {
        std::lock_guard<std::mutex> g(a->mu);
        a->wake_worker.notify_one();
    }
    const auto deadline = std::chrono::steady_clock::now() +
                          std::chrono::milliseconds(timeout_ms > 0 ? timeout_ms : 10000);
    bool lost = false;
    for (;;) {
        const uint32_t st = slot->state.load(std::memory_order_acquire);
        if (st == S_DONE || st == S_ERROR) break;
        const bool gone = a->ready.load() != 1;
        const bool late = std::chrono::steady_clock::now() > deadline;
        if (gone || late) {
            // reclaim: a slot the worker never picked up, or one it holds
            // while dead (arbiter.c:108-134, 216-236)
            uint32_t e = S_SUBMITTED;
            if (slot->state.compare_exchange_strong(e, S_FREE)) {
                lost = true;
                break;
            }
            if (gone && slot->state.load() == S_RUNNING) {
                slot->state.store(S_FREE);
                lost = true;
                break;
            }
        }
        std::unique_lock<std::mutex> lk(a->mu);
        a->wake_backends.wait_for(lk, std::chrono::milliseconds(10));
    }
    a->inflight--;
    if (lost) return 0;
    int ret;
    if (slot->state.load(std::memory_order_acquire) == S_DONE) {
        *ncnt = slot->nresults;
        *more = slot->more;
        memcpy(out, slot->results, sizeof(FvHit) * slot->nresults);
        ret = 1;
    } else {
        ret = -1;
    }
    slot->state.store(S_FREE, std::memory_order_release);
    return ret;
}

extern "C" int pv_arbiter_stats(PvArbiter *a, uint64_t *batches, uint64_t *requests,
                                uint32_t *inflight, int *worker_ready) {
    if (!a) return -1;
    if (batches) *batches = a->n_batches.load();
    if (requests) *requests = a->n_requests.load();
    if (inflight) *inflight = a->inflight.load();
    if (worker_ready) *worker_ready = a->ready.load();
    return 0;
}

extern "C" int pv_arbiter_feedback(PvArbiter *a, uint32_t relid, int strategy, uint32_t *q_us,
                                   uint32_t *batch_us, uint32_t *batch_n16) {
    if (!a) return -1;
    std::lock_guard<std::mutex> g(a->attach_mu);
    const int si = strategy == PV_STRAT_GPU_HNSW ? 1 : 0;
    for (Feedback *f : a->fb)
        if (f->relid == relid) {
            for (int b = 0; b < 5; b++)
                if (q_us) q_us[b] = f->q_us[si][b].load();
            if (batch_us) *batch_us = f->batch_us[si].load();
            if (batch_n16) *batch_n16 = f->batch_n16[si].load();
            return 0;
        }
    return -1;
}

extern "C" void pv_arbiter_kill_worker(PvArbiter *a) {
    if (a) a->kill.store(1);
}

extern "C" void pv_arbiter_destroy(PvArbiter *a) {
    if (!a) return;
    a->stop.store(1);
    {
        std::lock_guard<std::mutex> g(a->mu);
        a->wake_worker.notify_all();
    }
    if (a->worker.joinable()) a->worker.join();
    for (Feedback *f : a->fb) delete f;
    delete a;
}
