// hnsw_build.cpp — multi-threaded HNSW construction on the host.
//
// Produces the graph sections of the PAVES index file: per-node levels,
// level-0 lists of stride 2M+1 ([cnt, neighbours...]), upper-level slabs of
// M+1 per level, the entry node and its level. The construction follows the
// reference builder (extension/paves/src/engine/engine.cpp:698-919) step for
// step so that graphs have the same structure and files interoperate:
//   * node levels are a deterministic function of the row id (splitmix64 of
//     id * 0x5851F42D4C957F2D + 12345, level = floor(-ln(u) / ln(M)), <= 30);
//   * node 0 is inserted first, the rest in parallel (dynamic work claim);
//   * insertion = greedy descent through levels above the node's level,
//     then per level an ef_construction beam search, neighbour selection by
//     the "keep if closer to the node than to every kept neighbour" rule,
//     and bidirectional links; a full neighbour list is re-selected among
//     its members plus the new node.
// Per-node spinlocks guard the lists; each worker keeps its own epoch-tagged
// visited array.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <queue>
#include <thread>
#include <vector>

#include "paves_ext.h"

namespace {

inline float l2sq(const float *__restrict__ a, const float *__restrict__ b, int d) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    int i = 0;
    for (; i + 4 <= d; i += 4) {
        float t0 = a[i] - b[i], t1 = a[i + 1] - b[i + 1];
        float t2 = a[i + 2] - b[i + 2], t3 = a[i + 3] - b[i + 3];
        s0 += t0 * t0;
        s1 += t1 * t1;
        s2 += t2 * t2;
        s3 += t3 * t3;
    }
    for (; i < d; i++) {
        float t = a[i] - b[i];
        s0 += t * t;
    }
    return (s0 + s1) + (s2 + s3);
}

inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97f4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

struct Lock {
    std::atomic<uint32_t> v{0};
    void lock() {
        uint32_t z = 0;
        while (!v.compare_exchange_weak(z, 1, std::memory_order_acquire)) {
            z = 0;
#if defined(__x86_64__)
            __builtin_ia32_pause();
#endif
        }
    }
    void unlock() { v.store(0, std::memory_order_release); }
};

using Cand = std::pair<float, uint32_t>;  // (distance, node), ordered lexicographically

}  // namespace

struct PvHnsw {
    const float *vec = nullptr;
    int dim = 0;
    uint64_t n = 0;
    uint32_t M = 0, M0 = 0, efc = 0;
    std::vector<uint8_t> level;
    std::vector<uint32_t> l0;        // [n][M0 + 1]
    std::vector<uint64_t> upper_off;  // [n + 1], in u32 slots
    std::vector<uint32_t> upper;      // slabs of M + 1 per level >= 1
    std::vector<Lock> locks;
    std::atomic<uint64_t> entry{0};
    std::atomic<int> entry_level{-1};
    std::mutex entry_mu;

    const float *row(uint64_t i) const { return vec + i * (uint64_t)dim; }
    uint32_t *list(uint64_t node, int lvl) {
        if (lvl == 0) return &l0[node * (uint64_t)(M0 + 1)];
        return &upper[upper_off[node] + (uint64_t)(lvl - 1) * (M + 1)];
    }

    // copy of a node's list under its lock
    uint32_t snapshot(uint64_t node, int lvl, uint32_t *out) {
        locks[node].lock();
        const uint32_t *L = list(node, lvl);
        const uint32_t c = L[0];
        memcpy(out, L + 1, c * 4);
        locks[node].unlock();
        return c;
    }

    uint64_t descend(const float *q, uint64_t ep, int lvl) {
        float d = l2sq(q, row(ep), dim);
        uint32_t nb[256];
        for (bool moved = true; moved;) {
            moved = false;
            const uint32_t c = snapshot(ep, lvl, nb);
            for (uint32_t i = 0; i < c; i++) {
                const float nd = l2sq(q, row(nb[i]), dim);
                if (nd < d) {
                    d = nd;
                    ep = nb[i];
                    moved = true;
                }
            }
        }
        return ep;
    }

    // beam search at one level; out = up to ef results ascending
    void beam(const float *q, uint64_t ep, int lvl, uint32_t ef, std::vector<uint32_t> &tag,
              uint32_t epoch, std::vector<Cand> &out) {
        std::priority_queue<Cand, std::vector<Cand>, std::greater<Cand>> frontier;
        std::priority_queue<Cand> best;
        const float d0 = l2sq(q, row(ep), dim);
        frontier.push({d0, (uint32_t)ep});
        best.push({d0, (uint32_t)ep});
        tag[ep] = epoch;
        uint32_t nb[256];
        while (!frontier.empty()) {
            const Cand c = frontier.top();
            if (best.size() >= ef && c.first > best.top().first) break;
            frontier.pop();
            const uint32_t cnt = snapshot(c.second, lvl, nb);
            for (uint32_t i = 0; i < cnt; i++) {
                const uint32_t v = nb[i];
                if (tag[v] == epoch) continue;
                tag[v] = epoch;
                const float d = l2sq(q, row(v), dim);
                if (best.size() < ef || d < best.top().first) {
                    frontier.push({d, v});
                    best.push({d, v});
                    if (best.size() > ef) best.pop();
                }
            }
        }
        out.resize(best.size());
        for (size_t i = best.size(); i-- > 0;) {
            out[i] = best.top();
            best.pop();
        }
    }

    // keep a candidate (ascending) when it is closer to the node than to
    // every candidate already kept; at most m
    void prune(std::vector<Cand> &c, uint32_t m) {
        if (c.size() <= m) return;
        std::vector<Cand> kept;
        kept.reserve(m);
        for (const Cand &x : c) {
            if (kept.size() >= m) break;
            bool ok = true;
            for (const Cand &k : kept)
                if (l2sq(row(x.second), row(k.second), dim) < x.first) {
                    ok = false;
                    break;
                }
            if (ok) kept.push_back(x);
        }
        c.swap(kept);
    }

    void link(uint64_t node, uint32_t target, int lvl) {
        const uint32_t cap = lvl == 0 ? M0 : M;
        locks[node].lock();
        uint32_t *L = list(node, lvl);
        if (L[0] < cap) {
            L[1 + L[0]] = target;
            L[0]++;
            locks[node].unlock();
            return;
        }
        std::vector<Cand> c;
        c.reserve(cap + 1);
        c.push_back({l2sq(row(node), row(target), dim), target});
        for (uint32_t i = 0; i < L[0]; i++) c.push_back({l2sq(row(node), row(L[1 + i]), dim), L[1 + i]});
        std::sort(c.begin(), c.end());
        prune(c, cap);
        L[0] = (uint32_t)c.size();
        for (size_t i = 0; i < c.size(); i++) L[1 + i] = c[i].second;
        locks[node].unlock();
    }

    void insert(uint64_t node, std::vector<uint32_t> &tag, uint32_t &epoch) {
        const float *q = row(node);
        const int l = level[node];
        int el = entry_level.load(std::memory_order_acquire);
        uint64_t ep = entry.load(std::memory_order_acquire);
        if (el < 0) {
            std::lock_guard<std::mutex> g(entry_mu);
            if (entry_level.load() < 0) {
                entry.store(node);
                entry_level.store(l);
                return;
            }
            el = entry_level.load();
            ep = entry.load();
        }
        for (int lc = el; lc > l; lc--) ep = descend(q, ep, lc);
        std::vector<Cand> cand;
        for (int lc = std::min(el, l); lc >= 0; lc--) {
            epoch++;
            if (epoch == 0) {
                std::fill(tag.begin(), tag.end(), 0u);
                epoch = 1;
            }
            beam(q, ep, lc, efc, tag, epoch, cand);
            if (!cand.empty()) ep = cand[0].second;
            std::vector<Cand> sel = cand;
            prune(sel, M);
            locks[node].lock();
            uint32_t *L = list(node, lc);
            L[0] = (uint32_t)sel.size();
            for (size_t i = 0; i < sel.size(); i++) L[1 + i] = sel[i].second;
            locks[node].unlock();
            for (const Cand &s : sel) link(s.second, (uint32_t)node, lc);
        }
        if (l > entry_level.load(std::memory_order_acquire)) {
            std::lock_guard<std::mutex> g(entry_mu);
            if (l > entry_level.load()) {
                entry.store(node);
                entry_level.store(l);
            }
        }
    }
};

extern "C" PvHnsw *pv_hnsw_build(const float *vectors, uint64_t count, int dim, int M,
                                 int ef_construction, int threads, char *errbuf, size_t errlen) {
    if (!vectors || count == 0 || dim <= 0 || M < 2 || M > 120 || ef_construction < 1) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "hnsw: bad build parameters");
        return nullptr;
    }
    if (count >= 0xFFFFFFFFull) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "hnsw: too many rows");
        return nullptr;
    }
    PvHnsw *h = new PvHnsw();
    h->vec = vectors;
    h->dim = dim;
    h->n = count;
    h->M = (uint32_t)M;
    h->M0 = 2 * (uint32_t)M;
    h->efc = (uint32_t)ef_construction;
    h->level.resize(count);
    const double mult = 1.0 / log((double)M);
    h->upper_off.resize(count + 1);
    uint64_t slots = 0;
    for (uint64_t i = 0; i < count; i++) {
        double u = (double)(mix64(i * 0x5851F42D4C957F2DULL + 12345) >> 11) *
                   (1.0 / 9007199254740992.0);
        if (u < 1e-18) u = 1e-18;
        int lv = (int)(-log(u) * mult);
        if (lv > 30) lv = 30;
        h->level[i] = (uint8_t)lv;
        h->upper_off[i] = slots;
        slots += (uint64_t)lv * (M + 1);
    }
    h->upper_off[count] = slots;
    h->upper.assign(slots, 0);
    h->l0.assign(count * (uint64_t)(h->M0 + 1), 0);
    h->locks = std::vector<Lock>(count);

    {
        std::vector<uint32_t> tag(count, 0);
        uint32_t epoch = 0;
        h->insert(0, tag, epoch);
    }
    int T = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (T < 1) T = 1;
    std::atomic<uint64_t> next{1};
    auto work = [&]() {
        std::vector<uint32_t> tag(count, 0);
        uint32_t epoch = 0;
        for (;;) {
            const uint64_t i = next.fetch_add(1, std::memory_order_relaxed);
            if (i >= count) break;
            h->insert(i, tag, epoch);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return h;
}

namespace pv {

// Sections of a graph over count rows (levels drawn as above, zeroed lists)
// for builders that fill the lists themselves (the GPU builder).
PvHnsw *hnsw_sections(const float *vectors, uint64_t count, int dim, int M) {
    PvHnsw *h = new PvHnsw();
    h->vec = vectors;
    h->dim = dim;
    h->n = count;
    h->M = (uint32_t)M;
    h->M0 = 2 * (uint32_t)M;
    h->efc = 0;
    h->level.resize(count);
    const double mult = 1.0 / log((double)M);
    h->upper_off.resize(count + 1);
    uint64_t slots = 0;
    for (uint64_t i = 0; i < count; i++) {
        double u = (double)(mix64(i * 0x5851F42D4C957F2DULL + 12345) >> 11) *
                   (1.0 / 9007199254740992.0);
        if (u < 1e-18) u = 1e-18;
        int lv = (int)(-log(u) * mult);
        if (lv > 30) lv = 30;
        h->level[i] = (uint8_t)lv;
        h->upper_off[i] = slots;
        slots += (uint64_t)lv * (M + 1);
    }
    h->upper_off[count] = slots;
    h->upper.assign(slots, 0);
    h->l0.assign(count * (uint64_t)(h->M0 + 1), 0);
    return h;
}
const uint8_t *hnsw_levels(const PvHnsw *h) { return h->level.data(); }
uint32_t *hnsw_l0(PvHnsw *h) { return h->l0.data(); }
uint32_t *hnsw_upper_list(PvHnsw *h, uint64_t node, int level) { return h->list(node, level); }
void hnsw_set_entry(PvHnsw *h, uint64_t entry, int level, int efc) {
    h->entry.store(entry);
    h->entry_level.store(level);
    h->efc = (uint32_t)efc;
}

}  // namespace pv

extern "C" void pv_hnsw_free(PvHnsw *h) { delete h; }

extern "C" int pv_hnsw_info(const PvHnsw *h, uint32_t *M, int *max_level, uint64_t *entry,
                            uint64_t *upper_len) {
    if (!h) return -1;
    if (M) *M = h->M;
    if (max_level) *max_level = h->entry_level.load();
    if (entry) *entry = h->entry.load();
    if (upper_len) *upper_len = h->upper.size();
    return 0;
}

extern "C" int pv_hnsw_export(const PvHnsw *h, uint32_t *l0, uint8_t *levels,
                              uint64_t *upper_offs, uint32_t *upper) {
    if (!h) return -1;
    if (l0) memcpy(l0, h->l0.data(), h->l0.size() * 4);
    if (levels) memcpy(levels, h->level.data(), h->level.size());
    if (upper_offs) memcpy(upper_offs, h->upper_off.data(), h->upper_off.size() * 8);
    if (upper && !h->upper.empty()) memcpy(upper, h->upper.data(), h->upper.size() * 4);
    return 0;
}

// Greedy descent through the upper levels for each query (the level-0 entry
// point of a graph search; engine.cpp:1539-1559), parallel over queries.
extern "C" int pv_hnsw_entries(const float *vectors, int dim, const uint64_t *upper_offs,
                               const uint32_t *upper, uint32_t M, int max_level, uint64_t entry,
                               const float *queries, int nq, uint32_t *out, int threads) {
    if (!vectors || !queries || !out || nq < 0) return -1;
    auto one = [&](int qi) {
        const float *q = queries + (uint64_t)qi * dim;
        uint64_t ep = entry;
        for (int lc = max_level; lc >= 1; lc--) {
            float d = l2sq(q, vectors + ep * dim, dim);
            for (bool moved = true; moved;) {
                moved = false;
                const uint32_t *L = upper + upper_offs[ep] + (uint64_t)(lc - 1) * (M + 1);
                for (uint32_t i = 0; i < L[0]; i++) {
                    const float nd = l2sq(q, vectors + (uint64_t)L[1 + i] * dim, dim);
                    if (nd < d) {
                        d = nd;
                        ep = L[1 + i];
                        moved = true;
                    }
                }
            }
        }
        out[qi] = (uint32_t)ep;
    };
    int T = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (T < 1) T = 1;
    if (T > nq) T = nq > 0 ? nq : 1;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= nq) break;
            one(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return 0;
}
