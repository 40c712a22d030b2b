// graph.cu — batched filtered HNSW level-0 beam search.
//
// Replaces fv_graph_kernel / fv_gpu_graph_batch (gpu_engine.cu:1118-1485,
// 2338-2542) with the search semantics of the CPU HnswCursor
// (engine.cpp:1661-1713): traversal is unrestricted, only predicate-passing
// nodes enter the result list, the search stops when the best unexpanded
// candidate is farther than the worst of a full result list, when the
// frontier empties, or when max_visited nodes were visited.
//
// One CTA per query. Everything the search touches per step lives in
// shared memory:
//  * visited set: open-addressing hash of node ids; past half load it
//    spills into a per-query global bitmap that the kernel zeroes itself,
//    so there is no per-batch O(nq * N) memset;
//  * frontier and results: ascending key arrays (dist bits << 32 | node);
//    each step's new keys are placed by rank (a count among the new keys
//    plus a binary search in the old list), so no step sorts, and frontier
//    entries beyond the worst of a full result list are dropped;
//  * the step expands the best W frontier nodes at once (up to 16, fewer
//    only when the rest cannot beat the worst result), gathers their
//    neighbours from the fixed-width device adjacency, and computes
//    distances with 4 lanes per node (16-byte loads), so 128 rows are in
//    flight per CTA;
//  * the predicate is a bit of the batch bitmap, read only for candidates
//    that beat the current worst result.
#include <string.h>

#include <vector>

#include "pv_internal.h"

namespace pv {

constexpr int G_THREADS = 256;
constexpr int G_HC = 8192;   // visited hash slots (u32)
constexpr int G_FC = 8192;   // frontier capacity (selective filters grow it)
constexpr int G_RC = 512;    // result capacity (FV_GPU_MAX_EF)
constexpr int G_NB = 512;    // new entries per step (W * deg_cap <= G_NB)
constexpr uint32_t G_EMPTY = 0xFFFFFFFFu;

struct GraphArgs {
    const float *__restrict__ vecs;
    int dpad;
    uint64_t nrows;
    const uint32_t *__restrict__ adj;
    const uint16_t *__restrict__ deg;
    int deg_cap;
    int dc_shift;  // log2(deg_cap) when a power of two, else -1
    const float *__restrict__ queries;  // [nq][dpad]
    const uint32_t *__restrict__ entries;
    const int32_t *__restrict__ qprog;
    const uint32_t *__restrict__ bitmaps;
    uint64_t bm_words;
    int ef;
    const uint16_t *__restrict__ efq;  // optional per-query ef (<= ef)
    uint64_t max_visited;
    int wmax;
    uint32_t *visited_bits;  // [nq][bm_words], zeroed by the kernel on spill
    FvHit *out;              // [nq][ef]
    uint32_t *out_cnt;
    uint8_t *out_exh;
    uint32_t *stats;  // [nq][4]: steps, visited, predicate probes, results
};

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// A result/frontier key carries the node's predicate bit in bit 31 of the
// row half (rows < 2^31 are required), so one sort orders the keys and
// keeps each key's bit. Among passing keys the order is (dist, node).
constexpr uint32_t G_PASS = 0x80000000u;
__device__ __forceinline__ uint32_t grow_of(uint64_t k) { return (uint32_t)k & ~G_PASS; }

// Ascending bitonic sort of buf[0, n2) (n2 a power of two, 64 <= n2 <=
// 2 * G_THREADS). Only the n2 / 2 threads that own elements take part:
// thread t holds elements 2t and 2t + 1 in registers; partners at most 32
// elements away are exchanged by warp shuffles, farther ones through buf /
// alt alternately, with a named barrier over the participating warps. The
// caller synchronizes the block afterwards.
__device__ __forceinline__ void block_sort_pairs(uint64_t *buf, uint64_t *alt, int n2) {
    const int t = threadIdx.x;
    const int nact = n2 >> 1;  // a multiple of 32
    if (t >= nact) return;
    const int i0 = 2 * t, i1 = i0 + 1;
    uint64_t e0 = buf[i0], e1 = buf[i1];
    int which = 0;
    for (int k = 2; k <= n2; k <<= 1) {
        const bool asc = (i0 & k) == 0;  // same for i1: k >= 2
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j == 1) {
                const bool lt = e0 < e1;
                const uint64_t lo = lt ? e0 : e1, hi = lt ? e1 : e0;
                e0 = asc ? lo : hi;
                e1 = asc ? hi : lo;
                continue;
            }
            uint64_t o0, o1;
            if (j <= 32) {
                o0 = __shfl_xor_sync(0xffffffffu, e0, j >> 1);
                o1 = __shfl_xor_sync(0xffffffffu, e1, j >> 1);
            } else {
                uint64_t *bb = which ? alt : buf;
                which ^= 1;
                bb[i0] = e0;
                bb[i1] = e1;
                asm volatile("bar.sync 1, %0;" ::"r"(nact) : "memory");
                o0 = bb[i0 ^ j];
                o1 = bb[i1 ^ j];
            }
            const bool keep_min = ((i0 & j) == 0) == asc;  // same for i1: j >= 2
            e0 = ((e0 < o0) == keep_min) ? e0 : o0;
            e1 = ((e1 < o1) == keep_min) ? e1 : o1;
        }
    }
    asm volatile("bar.sync 1, %0;" ::"r"(nact) : "memory");
    buf[i0] = e0;
    buf[i1] = e1;
}

__global__ void __launch_bounds__(G_THREADS) graph_kernel(GraphArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *const fr0 = (uint64_t *)smem_raw;  // [2][G_FC] frontier ping-pong
    uint64_t *const rs0 = fr0 + 2 * G_FC;        // [2][G_RC] results ping-pong
    uint64_t *nfk = rs0 + 2 * G_RC;                // [G_NB] new keys (step order)
    uint64_t *salt = nfk + G_NB;                  // [G_NB] sort exchange buffer
    uint32_t *hash = (uint32_t *)(salt + G_NB);   // [G_HC]
    uint32_t *nid = hash + G_HC;                  // [G_NB] gathered neighbours
    int *rpos = (int *)(nid + G_NB);              // [G_NB] new results' places
    int *fpos = rpos + G_NB;                      // [G_NB] new frontier keys' places
    float *sq = (float *)(fpos + G_NB);           // [dpad] query

    __shared__ int s_nf, s_nr, s_head, s_cur_f, s_cur_r, s_nsel, s_nnew, s_nfk;
    __shared__ int s_wpass[G_THREADS / 32];
    __shared__ int s_stop, s_exh, s_spilled, s_hcount, s_dropped;
    __shared__ uint32_t s_sel[32];
    __shared__ unsigned long long s_visited;
    __shared__ unsigned int s_probes, s_steps;

    const int q = blockIdx.x;
    const int tid = threadIdx.x;
    // a per-query beam width of 0: the query is answered elsewhere (a mixed
    // routed batch scans it), nothing to search
    if (a.efq && a.efq[q] == 0) {
        if (tid == 0) {
            a.out_cnt[q] = 0;
            a.out_exh[q] = 0;
            if (a.stats)
                for (int i = 0; i < 4; i++) a.stats[q * 4 + i] = 0;
        }
        return;
    }
    // per-query beam width (never above the batch's, which is the output stride)
    const int ef = a.efq ? min((int)a.efq[q], a.ef) : a.ef;
    const int pg = a.qprog[q];
    const uint32_t *bm = pg >= 0 ? a.bitmaps + (uint64_t)pg * a.bm_words : nullptr;
    uint32_t *vb = a.visited_bits + (uint64_t)q * a.bm_words;
    const float *qv = a.queries + (uint64_t)q * a.dpad;

    for (int i = tid; i < a.dpad; i += blockDim.x) sq[i] = qv[i];
    for (int i = tid; i < G_HC; i += blockDim.x) hash[i] = G_EMPTY;
    if (tid == 0) {
        s_nf = 0; s_nr = 0; s_head = 0; s_cur_f = 0; s_cur_r = 0;
        s_stop = 0; s_exh = 0; s_spilled = 0; s_hcount = 0; s_dropped = 0;
        s_visited = 0; s_probes = 0; s_steps = 0;
    }
    __syncthreads();

    // seed: entry point (engine.cpp:1651-1656)
    {
        uint32_t ep = a.entries[q];
        if (ep >= a.nrows) ep = 0;
        const int warp = tid >> 5, lane = tid & 31;
        if (warp == 0) {
            float acc = 0.f;
            const float *x = a.vecs + (uint64_t)ep * a.dpad;
            for (int j = lane * 4; j < a.dpad; j += 128) {
                float4 v = __ldg((const float4 *)(x + j));
                float4 w = *(const float4 *)(sq + j);
                float d0 = v.x - w.x, d1 = v.y - w.y, d2 = v.z - w.z, d3 = v.w - w.w;
                acc = fmaf(d0, d0, acc); acc = fmaf(d1, d1, acc);
                acc = fmaf(d2, d2, acc); acc = fmaf(d3, d3, acc);
            }
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                hash[hash_u32(ep) & (G_HC - 1)] = ep;
                s_hcount = 1;
                s_visited = 1;
                const bool pass = !bm || ((bm[ep >> 5] >> (ep & 31)) & 1u);
                const uint64_t key = make_key(acc, ep | (pass ? G_PASS : 0u));
                fr0[0] = key;
                s_nf = 1;
                if (pass) {
                    rs0[0] = key;
                    s_nr = 1;
                }
            }
        }
    }
    __syncthreads();

    for (;;) {
        // ---- stop tests and selection (warp 0; the frontier is ascending):
        // the best W entries, cut at the first one beyond the worst result
        if (tid < 32) {
            const int lane = tid;
            const uint64_t *F = fr0 + s_cur_f * G_FC;
            const int head = s_head, avail = s_nf - head;
            const bool full = s_nr >= ef;
            const float worst = full ? key_dist(rs0[s_cur_r * G_RC + ef - 1]) : 0.f;
            const int w = avail < a.wmax ? avail : a.wmax;
            const uint64_t k = lane < w ? F[head + lane] : KEY_MAX;
            const bool ok = lane < w && (lane == 0 || !full || !(key_dist(k) > worst));
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            const int n = m == 0xffffffffu ? 32 : __ffs(~m) - 1;  // leading run of ok lanes
            int stop = 0;
            if (avail <= 0) stop = 1;
            else if (s_visited >= a.max_visited) stop = 2;
            else if (full && key_dist(F[head]) > worst) stop = 3;
            if (!stop && lane < n) s_sel[lane] = grow_of(k);
            if (lane == 0) {
                s_stop = stop;
                // an empty frontier is exhaustion unless entries were dropped
                // (they would still sit in an unbounded candidate queue)
                if (stop == 1) s_exh = s_dropped ? 0 : 1;
                if (stop == 2) s_exh = 1;
                if (!stop) {
                    s_head = head + n;
                    s_nsel = n;
                    s_nnew = 0;
                    s_nfk = 0;
                    s_steps++;
                }
            }
        }
        __syncthreads();
        if (s_stop) break;

        // ---- gather neighbours of the selected nodes, visited test-and-set
        const int nsel = s_nsel;
        const int dc = a.deg_cap;
        const int total = nsel * dc;
        const int lane = tid & 31;
        for (int base = 0; base < total; base += G_THREADS) {
            const int t = base + tid;
            bool fresh = false;
            uint32_t nb = 0;
            if (t < total) {
                const int s = a.dc_shift >= 0 ? t >> a.dc_shift : t / dc;
                const int i = t - s * dc;
                const uint32_t node = s_sel[s];
                // both loads in flight at once (the list is allocated to deg_cap)
                const int dg = (int)__ldg(a.deg + node);
                nb = __ldg(a.adj + (uint64_t)node * dc + i);
                if (i < dg && nb < a.nrows) {
                    if (s_spilled) {
                        const uint32_t m = 1u << (nb & 31);
                        fresh = (atomicOr(vb + (nb >> 5), m) & m) == 0;
                    } else {
                        uint32_t h = hash_u32(nb) & (G_HC - 1);
                        for (int probe = 0; probe < G_HC; probe++) {
                            const uint32_t old = atomicCAS(hash + h, G_EMPTY, nb);
                            if (old == G_EMPTY) { fresh = true; break; }
                            if (old == nb) break;
                            h = (h + 1) & (G_HC - 1);
                        }
                    }
                }
            }
            // one shared-memory atomic per warp for the appends
            const unsigned fm = __ballot_sync(0xffffffffu, fresh);
            int wb = 0;
            if (lane == 0 && fm) {
                wb = atomicAdd(&s_nnew, __popc(fm));
                if (!s_spilled) atomicAdd(&s_hcount, __popc(fm));
            }
            wb = __shfl_sync(0xffffffffu, wb, 0);
            if (fresh) nid[wb + __popc(fm & ((1u << lane) - 1u))] = nb;
        }
        __syncthreads();
        const int nnew = s_nnew;
        if (tid == 0) s_visited += (unsigned long long)nnew;

        // ---- distances: 4 lanes per node, two nodes per lane group, so
        // 128 rows (64 KB at d=128) are in flight per pass; the predicate
        // word of each row is fetched with the row. Admission as the
        // reference cursor: a node enters the frontier while results are
        // short or it beats the worst result (engine.cpp:1684-1690).
        const bool full = s_nr >= ef;
        const float worst = full ? key_dist(rs0[s_cur_r * G_RC + ef - 1]) : 0.f;
        {
            constexpr int GROUPS = G_THREADS / 4;  // lane groups of 4
            constexpr int RPG = 4;                 // rows per group per pass
            const int grp = tid >> 2, sub = tid & 3;
            for (int base = 0; base < nnew; base += RPG * GROUPS) {
                uint32_t nn[RPG], pw[RPG];
                bool okr[RPG];
                const float *xr[RPG];
                float acc[RPG];
#pragma unroll
                for (int r = 0; r < RPG; r++) {
                    const int i = base + grp + r * GROUPS;
                    okr[r] = i < nnew;
                    // rows past nnew re-read row nid[0] (valid) and are discarded
                    nn[r] = nid[okr[r] ? i : 0];
                    xr[r] = a.vecs + (uint64_t)nn[r] * a.dpad;
                    pw[r] = bm ? __ldg(bm + (nn[r] >> 5)) : ~0u;
                    acc[r] = 0.f;
                }
                // chunks of 64 dims: all loads of a chunk issue before use
                for (int c = 0; c < a.dpad; c += 64) {
                    float4 v[RPG][4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int j = c + u * 16 + sub * 4;
                        const bool in = j < a.dpad;
#pragma unroll
                        for (int r = 0; r < RPG; r++)
                            v[r][u] = in ? __ldg((const float4 *)(xr[r] + j))
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int j = c + u * 16 + sub * 4;
                        if (j >= a.dpad) break;
                        const float4 w = *(const float4 *)(sq + j);
#pragma unroll
                        for (int r = 0; r < RPG; r++) {
                            const float d0 = v[r][u].x - w.x, d1 = v[r][u].y - w.y;
                            const float d2 = v[r][u].z - w.z, d3 = v[r][u].w - w.w;
                            acc[r] = fmaf(d0, d0, acc[r]); acc[r] = fmaf(d1, d1, acc[r]);
                            acc[r] = fmaf(d2, d2, acc[r]); acc[r] = fmaf(d3, d3, acc[r]);
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < RPG; r++) {
                    acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 2);
                    acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], 1);
                }
                // admitted rows of this warp (lanes with sub == 0), appended
                // with one shared-memory atomic per warp
                unsigned m[RPG];
                bool ad[RPG];
                int tot = 0;
#pragma unroll
                for (int r = 0; r < RPG; r++) {
                    ad[r] = okr[r] && sub == 0 && (!full || acc[r] < worst);
                    m[r] = __ballot_sync(0xffffffffu, ad[r]);
                    tot += __popc(m[r]);
                }
                int wb = 0;
                if (lane == 0 && tot) {
                    wb = atomicAdd(&s_nfk, tot);
                    if (bm) atomicAdd(&s_probes, (unsigned)tot);
                }
                wb = __shfl_sync(0xffffffffu, wb, 0);
                const unsigned lt = (1u << lane) - 1u;
#pragma unroll
                for (int r = 0; r < RPG; r++) {
                    if (ad[r]) {
                        const bool pass = (pw[r] >> (nn[r] & 31)) & 1u;
                        nfk[wb + __popc(m[r] & lt)] = make_key(acc[r], nn[r] | (pass ? G_PASS : 0u));
                    }
                    wb += __popc(m[r]);
                }
            }
        }
        __syncthreads();
        const int nnf = s_nfk;

        // ---- sort the step's new keys, then merge them by rank: a new
        // key's place is its index among the sorted new keys plus a binary
        // search in the old list, and an old entry moves up by the number
        // of new keys placed before it (keys are unique: each node is
        // visited once).
        // Up to G_THREADS keys: each thread counts the keys below its own
        // (independent loads, no barrier chain); more: bitonic sort.
        uint64_t *srt = nfk;
        if (nnf <= G_THREADS) {
            if (tid < nnf) {
                const uint64_t key = nfk[tid];
                int r = 0;
                for (int i = 0; i < nnf; i++) r += nfk[i] < key;
                salt[r] = key;
            }
            srt = salt;
            __syncthreads();
        } else {
            int n2 = 64;
            while (n2 < nnf) n2 <<= 1;
            for (int i = nnf + tid; i < n2; i += blockDim.x) nfk[i] = KEY_MAX;
            __syncthreads();
            block_sort_pairs(nfk, salt, n2);
            __syncthreads();
        }
        // exclusive prefix of the pass bits over the sorted keys (thread t
        // owns sorted positions 2t, 2t + 1)
        const int i0 = 2 * tid;
        const uint64_t k0 = i0 < nnf ? srt[i0] : KEY_MAX;
        const uint64_t k1 = i0 + 1 < nnf ? srt[i0 + 1] : KEY_MAX;
        const int p0 = (i0 < nnf && ((uint32_t)k0 & G_PASS)) ? 1 : 0;
        const int p1 = (i0 + 1 < nnf && ((uint32_t)k1 & G_PASS)) ? 1 : 0;
        int incl = p0 + p1;
        {
            const int warp = tid >> 5;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (lane == 31) s_wpass[warp] = incl;
            __syncthreads();
            for (int w = 0; w < warp; w++) incl += s_wpass[w];
        }
        int nnr = 0;
        for (int w = 0; w < G_THREADS / 32; w++) nnr += s_wpass[w];
        const int cf = s_cur_f, cr = s_cur_r;
        const int head = s_head, nf = s_nf, nr = s_nr;
        const uint64_t *Rold = rs0 + cr * G_RC;
        uint64_t *Rnew = rs0 + (cr ^ 1) * G_RC;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            if (!(e ? p1 : p0)) continue;
            const uint64_t key = e ? k1 : k0;
            const int rr = incl - (e ? 1 : p1 + 1);  // exclusive rank among passing keys
            int lo = 0, hi = nr;  // first old result > key
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (Rold[mid] < key) lo = mid + 1; else hi = mid;
            }
            rpos[rr] = lo;
            if (rr + lo < ef) Rnew[rr + lo] = key;
        }
        __syncthreads();
        for (int i = tid; i < nr; i += blockDim.x) {
            int lo = 0, hi = nnr;  // new results placed at or before i
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (rpos[mid] <= i) lo = mid + 1; else hi = mid;
            }
            if (i + lo < ef) Rnew[i + lo] = Rold[i];
        }
        __syncthreads();
        // frontier entries beyond the worst of a full result list are never
        // expanded (the stop test would end the search first): drop them
        const int nr2 = min(nr + nnr, ef);
        const uint64_t kthr =
            nr2 >= ef ? (((uint64_t)__float_as_uint(key_dist(Rnew[ef - 1])) << 32) | 0xFFFFFFFFull)
                      : KEY_MAX;
        const uint64_t *Fold = fr0 + cf * G_FC + head;
        uint64_t *Fnew = fr0 + (cf ^ 1) * G_FC;
        int na, nk;
        {
            int lo = 0, hi = nf - head;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (Fold[mid] <= kthr) lo = mid + 1; else hi = mid;
            }
            na = lo;
            lo = 0;
            hi = nnf;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (srt[mid] <= kthr) lo = mid + 1; else hi = mid;
            }
            nk = lo;
        }
        for (int s = tid; s < nk; s += blockDim.x) {
            const uint64_t key = srt[s];
            int lo = 0, hi = na;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (Fold[mid] < key) lo = mid + 1; else hi = mid;
            }
            fpos[s] = lo;
            if (s + lo < G_FC) Fnew[s + lo] = key;
        }
        __syncthreads();
        {
            const int chunk = (na + G_THREADS - 1) / G_THREADS;
            const int a0 = tid * chunk, a1 = min(a0 + chunk, na);
            if (a0 < a1) {
                int lo = 0, hi = nk;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (fpos[mid] <= a0) lo = mid + 1; else hi = mid;
                }
                int sft = lo;
                for (int i = a0; i < a1; i++) {
                    while (sft < nk && fpos[sft] <= i) sft++;
                    if (i + sft < G_FC) Fnew[i + sft] = Fold[i];
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            if (na < nf - head || nk < nnf || na + nk > G_FC) s_dropped = 1;
            s_nf = min(na + nk, G_FC);
            s_head = 0;
            s_cur_f = cf ^ 1;
            s_nr = nr2;
            s_cur_r = cr ^ 1;
        }

        // ---- spill the visited set to the global bitmap at half load
        if (!s_spilled && s_hcount > G_HC / 2) {
            __syncthreads();
            for (uint64_t w = tid; w < a.bm_words; w += blockDim.x) vb[w] = 0u;
            __syncthreads();
            for (int i = tid; i < G_HC; i += blockDim.x) {
                const uint32_t v = hash[i];
                if (v != G_EMPTY) atomicOr(vb + (v >> 5), 1u << (v & 31));
            }
            __syncthreads();
            if (tid == 0) s_spilled = 1;
        }
        __syncthreads();
    }

    // ---- emit (ascending by (dist, node))
    const int nr = s_nr;
    const uint64_t *R = rs0 + s_cur_r * G_RC;
    for (int i = tid; i < nr; i += blockDim.x) {
        FvHit h;
        h.node = grow_of(R[i]);
        h.dist = key_dist(R[i]);
        a.out[(uint64_t)q * a.ef + i] = h;
    }
    if (tid == 0) {
        a.out_cnt[q] = (uint32_t)nr;
        a.out_exh[q] = (uint8_t)s_exh;
        if (a.stats) {
            a.stats[q * 4 + 0] = s_steps;
            a.stats[q * 4 + 1] = (uint32_t)s_visited;
            a.stats[q * 4 + 2] = s_probes;
            a.stats[q * 4 + 3] = (uint32_t)nr;
        }
    }
}

size_t graph_smem_bytes(int dpad) {
    return (size_t)(2 * G_FC + 2 * G_RC + 2 * G_NB) * 8 + (size_t)(G_HC + 3 * G_NB) * 4 +
           (size_t)dpad * 4;
}

cudaError_t launch_graph(const GraphArgs &a, int nq, cudaStream_t st) {
    const size_t smem = graph_smem_bytes(a.dpad);
    cudaError_t e = raise_smem_limit((const void *)graph_kernel, smem);
    if (e != cudaSuccess) return e;
    graph_kernel<<<nq, G_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace pv

using namespace pv;

extern "C" int fv_gpu_graph_batch(FvGpuIndex *g, int nq, const float *queries,
                                  const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes,
                                  int nnodes, const int32_t *children, int nchildren,
                                  const double *invals, int ninvals, uint32_t ef,
                                  uint64_t max_visited, FvHit *out, uint32_t *out_cnt,
                                  uint8_t *exhausted, char *errbuf, size_t errlen) {
    if (!g || !g->d_adj) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: graph not uploaded");
        return -1;
    }
    if (g->count >= (1ull << 31)) {  // keys keep the predicate bit in bit 31 of the row
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: graph search needs < 2^31 rows");
        return -1;
    }
    if (nq < 1 || nq > FV_GPU_MAX_BATCH || ef < 1 || ef > FV_GPU_MAX_EF || !queries || !qd ||
        !out || !out_cnt || !exhausted) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "gpu: bad graph batch (nq=%d ef=%u)", nq, ef);
        return -1;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return -1;
    std::vector<uint32_t> entries(nq);
    for (int q = 0; q < nq; q++) entries[q] = qd[q].entry;
    return graph_run_host(g, nq, queries, entries.data(), pb, ef, max_visited, out, out_cnt,
                          exhausted, errbuf, errlen);
}

namespace pv {

GraphOut graph_out_layout(int nq, uint32_t ef) {
    GraphOut lo;
    const size_t hit_bytes = (size_t)nq * ef * sizeof(FvHit);
    lo.off_cnt = (hit_bytes + 255) & ~(size_t)255;
    lo.off_exh = lo.off_cnt + (((size_t)nq * 4 + 255) & ~(size_t)255);
    lo.off_st = lo.off_exh + (((size_t)nq + 255) & ~(size_t)255);
    lo.bytes = lo.off_st + (size_t)nq * 16;
    return lo;
}

int graph_launch(FvGpuIndex *g, int nq, const float *d_q, const uint32_t *d_entries,
                 const int32_t *d_qprog, const uint16_t *d_efq, uint32_t ef,
                 uint64_t max_visited, char *od, const GraphOut &lo, char *errbuf,
                 size_t errlen, cudaStream_t st) {
    if (!st) st = g->stream;
    const uint64_t bm_words = (g->count + 31) / 32;
    GraphScratch &gs = g->graph;
    PV_CUDA_OK(gs.visited.ensure((size_t)nq * bm_words * 4), errbuf, errlen);
    GraphArgs a;
    a.vecs = g->d_vecs;
    a.dpad = g->dpad;
    a.nrows = g->count;
    a.adj = g->d_adj;
    a.deg = g->d_deg;
    a.deg_cap = g->deg_cap;
    a.dc_shift = -1;
    for (int sh = 0; sh < 16; sh++)
        if (g->deg_cap == (1 << sh)) a.dc_shift = sh;
    a.queries = d_q;
    a.entries = d_entries;
    a.qprog = d_qprog;
    a.bitmaps = g->scan.bitmaps.as<uint32_t>();
    a.bm_words = bm_words;
    a.ef = (int)ef;
    a.efq = d_efq;
    a.max_visited = max_visited;
    int wmax = G_NB / (g->deg_cap > 0 ? g->deg_cap : 1);
    if (wmax > 16) wmax = 16;
    if (wmax < 1) wmax = 1;
    a.wmax = wmax;
    a.visited_bits = gs.visited.as<uint32_t>();
    a.out = (FvHit *)od;
    a.out_cnt = (uint32_t *)(od + lo.off_cnt);
    a.out_exh = (uint8_t *)(od + lo.off_exh);
    a.stats = (uint32_t *)(od + lo.off_st);
    g->launches++;
    PV_CUDA_OK(launch_graph(a, nq, st), errbuf, errlen);
    return 0;
}

int graph_run_host(FvGpuIndex *g, int nq, const float *queries, const uint32_t *entries,
                   const PredBatch &pb, uint32_t ef, uint64_t max_visited, FvHit *out,
                   uint32_t *out_cnt, uint8_t *exhausted, char *errbuf, size_t errlen) {
    g->launches = 0;
    DevBatch db;
    db.stage_h = &g->scan.stage_h;
    db.stage_d = &g->scan.stage_d;
    for (int q = 0; q < nq; q++)
        if (entries[q] >= g->count) {
            snprintf(errbuf, errlen, "gpu: query %d entry %u out of range", q, entries[q]);
            return -1;
        }
    // entries ride in the extra section of the staging buffer
    if (brute_prepare(g, nq, queries, pb, db, (size_t)nq * 4, errbuf, errlen)) return -1;
    const size_t off_ent = db.off_extra;
    memcpy(db.stage_h->as<char>() + off_ent, entries, (size_t)nq * 4);
    if (brute_upload(g, db, errbuf, errlen)) return -1;
    char *d = db.stage_d->as<char>();
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;
    const int P = db.P;
    cudaEventRecord(g->ev0, g->stream);
    if (P > 0) {
        PV_CUDA_OK(s.bitmaps.ensure((size_t)P * bm_words * 4), errbuf, errlen);
        PV_CUDA_OK(s.popcnt.ensure((size_t)P * 8), errbuf, errlen);
        g->launches++;
        PV_CUDA_OK(launch_bitmaps(g->d_cols, g->count, (const PredInsn *)(d + db.off_insns),
                                  (const PredProg *)(d + db.off_progs),
                                  (const double *)(d + db.off_consts), P,
                                  s.bitmaps.as<uint32_t>(), bm_words,
                                  s.popcnt.as<unsigned long long>(), g->sm_count, g->stream,
                                  db.ninsns, db.nconsts, g->ncols, db.one_range),
                   errbuf, errlen);
    }
    const GraphOut lo = graph_out_layout(nq, ef);
    const size_t off_cnt = lo.off_cnt, off_exh = lo.off_exh, off_st = lo.off_st;
    const size_t obytes = lo.bytes;
    PV_CUDA_OK(s.out_d.ensure(obytes), errbuf, errlen);
    PV_CUDA_OK(s.out_h.ensure(obytes), errbuf, errlen);
    char *od = s.out_d.as<char>();
    if (graph_launch(g, nq, (const float *)(d + db.off_q), (const uint32_t *)(d + off_ent),
                     (const int32_t *)(d + db.off_qprog), nullptr, ef, max_visited, od, lo,
                     errbuf, errlen))
        return -1;
    cudaEventRecord(g->ev1, g->stream);
    PV_CUDA_OK(cudaMemcpyAsync(s.out_h.p, od, obytes, cudaMemcpyDeviceToHost, g->stream), errbuf,
               errlen);
    PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
    cudaEventElapsedTime(&g->last_kernel_ms, g->ev0, g->ev1);
    const char *oh = s.out_h.as<char>();
    const uint32_t *cnt = (const uint32_t *)(oh + off_cnt);
    for (int q = 0; q < nq; q++) {
        uint32_t c = cnt[q] > ef ? ef : cnt[q];
        memcpy(out + (size_t)q * ef, oh + (size_t)q * ef * sizeof(FvHit), c * sizeof(FvHit));
        out_cnt[q] = c;
    }
    memcpy(exhausted, oh + off_exh, (size_t)nq);
    g->graph_stats.resize((size_t)nq * 4);
    memcpy(g->graph_stats.data(), oh + off_st, (size_t)nq * 16);
    return 0;
}

}  // namespace pv
