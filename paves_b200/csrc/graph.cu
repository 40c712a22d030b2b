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
//  * frontier and results: ascending key arrays (dist bits << 32 | node)
//    kept sorted by merge-path merges of each step's sorted new entries;
//  * the step expands the best W frontier nodes at once (W adapts to the
//    frontier size), gathers their neighbours from the fixed-width device
//    adjacency, and computes distances with 8 lanes per node (16-byte
//    loads), so 32 rows are in flight per CTA;
//  * the predicate is a bit of the batch bitmap, read only for candidates
//    that beat the current worst result.
#include <string.h>

#include <vector>

#include "pv_internal.h"

namespace pv {

constexpr int G_THREADS = 256;
constexpr int G_HC = 4096;   // visited hash slots (u32)
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
    const float *__restrict__ queries;  // [nq][dpad]
    const uint32_t *__restrict__ entries;
    const int32_t *__restrict__ qprog;
    const uint32_t *__restrict__ bitmaps;
    uint64_t bm_words;
    int ef;
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

// Block-wide merge of ascending A[0,na) and B[0,nb) into C[0,min(na+nb,cap)).
__device__ __forceinline__ void merge_path(const uint64_t *A, int na, const uint64_t *B, int nb,
                                           uint64_t *C, int cap) {
    const int total = min(na + nb, cap);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int lo = max(0, i - nb), hi = min(i, na);
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (A[mid] < B[i - mid - 1]) lo = mid + 1; else hi = mid;
        }
        const int a = lo, b = i - lo;
        C[i] = (a < na && (b >= nb || A[a] < B[b])) ? A[a] : B[b];
    }
}

// Block-wide ascending bitonic sort of buf[0, n2), n2 a power of two.
__device__ __forceinline__ void bitonic_block(uint64_t *buf, int n2) {
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < (n2 >> 1); i += blockDim.x) {
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo | j;
                const uint64_t x = buf[lo], y = buf[hi];
                if ((x > y) == ((lo & k) == 0)) {
                    buf[lo] = y;
                    buf[hi] = x;
                }
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(G_THREADS) graph_kernel(GraphArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *const fr0 = (uint64_t *)smem_raw;  // [2][G_FC] frontier ping-pong
    uint64_t *const rs0 = fr0 + 2 * G_FC;        // [2][G_RC] results ping-pong
    uint64_t *nfk = rs0 + 2 * G_RC;                // [G_NB] new frontier keys
    uint64_t *nrk = nfk + G_NB;                   // [G_NB] new result keys
    uint32_t *hash = (uint32_t *)(nrk + G_NB);    // [G_HC]
    uint32_t *nid = hash + G_HC;                  // [G_NB] gathered neighbours
    float *sq = (float *)(nid + G_NB);            // [dpad] query

    __shared__ int s_nf, s_nr, s_head, s_cur_f, s_cur_r, s_nsel, s_nnew, s_nfk, s_nrk;
    __shared__ int s_stop, s_exh, s_spilled, s_hcount;
    __shared__ uint32_t s_sel[32];
    __shared__ unsigned long long s_visited;
    __shared__ unsigned int s_probes, s_steps;

    const int q = blockIdx.x;
    const int tid = threadIdx.x;
    const int ef = a.ef;
    const int pg = a.qprog[q];
    const uint32_t *bm = pg >= 0 ? a.bitmaps + (uint64_t)pg * a.bm_words : nullptr;
    uint32_t *vb = a.visited_bits + (uint64_t)q * a.bm_words;
    const float *qv = a.queries + (uint64_t)q * a.dpad;

    for (int i = tid; i < a.dpad; i += blockDim.x) sq[i] = qv[i];
    for (int i = tid; i < G_HC; i += blockDim.x) hash[i] = G_EMPTY;
    if (tid == 0) {
        s_nf = 0; s_nr = 0; s_head = 0; s_cur_f = 0; s_cur_r = 0;
        s_stop = 0; s_exh = 0; s_spilled = 0; s_hcount = 0;
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
                const uint64_t key = make_key(acc, ep);
                fr0[0] = key;
                s_nf = 1;
                const bool pass = !bm || ((bm[ep >> 5] >> (ep & 31)) & 1u);
                if (pass) {
                    rs0[0] = key;
                    s_nr = 1;
                }
            }
        }
    }
    __syncthreads();

    for (;;) {
        // ---- stop tests and selection (thread 0; frontier is ascending)
        if (tid == 0) {
            const uint64_t *F = (fr0 + s_cur_f * G_FC);
            const int avail = s_nf - s_head;
            int stop = 0;
            if (avail <= 0) {
                stop = 1;
                s_exh = 1;
            } else if (s_visited >= a.max_visited) {
                stop = 1;
                s_exh = 1;
            } else if (s_nr >= ef && key_dist(F[s_head]) > key_dist(rs0[s_cur_r * G_RC + ef - 1])) {
                stop = 1;
            }
            s_stop = stop;
            if (!stop) {
                int w = avail >> 6;
                if (w < 4) w = 4;
                if (w > a.wmax) w = a.wmax;
                if (w > avail) w = avail;
                const bool full = s_nr >= ef;
                const float worst = full ? key_dist(rs0[s_cur_r * G_RC + ef - 1]) : 0.f;
                int n = 0;
                for (int i = 0; i < w; i++) {
                    const uint64_t k = F[s_head + i];
                    if (i > 0 && full && key_dist(k) > worst) break;
                    s_sel[n++] = key_row(k);
                }
                s_head += n;
                s_nsel = n;
                s_nnew = 0;
                s_nfk = 0;
                s_nrk = 0;
                s_steps++;
            }
        }
        __syncthreads();
        if (s_stop) break;

        // ---- gather neighbours of the selected nodes, visited test-and-set
        const int nsel = s_nsel;
        const int dc = a.deg_cap;
        for (int t = tid; t < nsel * dc; t += blockDim.x) {
            const int s = t / dc, i = t - s * dc;
            const uint32_t node = s_sel[s];
            if (i >= (int)a.deg[node]) continue;
            const uint32_t nb = a.adj[(uint64_t)node * dc + i];
            if (nb >= a.nrows) continue;
            bool fresh;
            if (s_spilled) {
                const uint32_t m = 1u << (nb & 31);
                fresh = (atomicOr(vb + (nb >> 5), m) & m) == 0;
            } else {
                uint32_t h = hash_u32(nb) & (G_HC - 1);
                fresh = false;
                for (int probe = 0; probe < G_HC; probe++) {
                    const uint32_t old = atomicCAS(hash + h, G_EMPTY, nb);
                    if (old == G_EMPTY) { fresh = true; break; }
                    if (old == nb) break;
                    h = (h + 1) & (G_HC - 1);
                }
                if (fresh) atomicAdd(&s_hcount, 1);
            }
            if (fresh) nid[atomicAdd(&s_nnew, 1)] = nb;
        }
        __syncthreads();
        const int nnew = s_nnew;
        if (tid == 0) s_visited += (unsigned long long)nnew;

        // ---- distances: 8 lanes per node, 32 nodes per pass
        const bool full = s_nr >= ef;
        const float worst = full ? key_dist(rs0[s_cur_r * G_RC + ef - 1]) : 0.f;
        {
            const int grp = tid >> 3, sub = tid & 7;
            for (int base = 0; base < nnew; base += G_THREADS / 8) {
                const int i = base + grp;
                const bool ok = i < nnew;
                const uint32_t node = ok ? nid[i] : 0;
                float acc = 0.f;
                if (ok) {
                    const float *x = a.vecs + (uint64_t)node * a.dpad;
                    for (int j = sub * 4; j < a.dpad; j += 32) {
                        float4 v = __ldg((const float4 *)(x + j));
                        float4 w = *(const float4 *)(sq + j);
                        float d0 = v.x - w.x, d1 = v.y - w.y, d2 = v.z - w.z, d3 = v.w - w.w;
                        acc = fmaf(d0, d0, acc); acc = fmaf(d1, d1, acc);
                        acc = fmaf(d2, d2, acc); acc = fmaf(d3, d3, acc);
                    }
                }
                acc += __shfl_xor_sync(0xffffffffu, acc, 4);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                if (ok && sub == 0 && (!full || acc < worst)) {
                    const uint64_t key = make_key(acc, node);
                    nfk[atomicAdd(&s_nfk, 1)] = key;
                    bool pass = true;
                    if (bm) {
                        atomicAdd(&s_probes, 1u);
                        pass = (__ldg(bm + (node >> 5)) >> (node & 31)) & 1u;
                    }
                    if (pass) nrk[atomicAdd(&s_nrk, 1)] = key;
                }
            }
        }
        __syncthreads();
        const int nnf = s_nfk, nnr = s_nrk;

        // ---- sort the step's new entries
        int n2 = 1;
        while (n2 < (nnf > nnr ? nnf : nnr)) n2 <<= 1;
        for (int i = tid; i < n2; i += blockDim.x) {
            if (i >= nnf) nfk[i] = KEY_MAX;
            if (i >= nnr) nrk[i] = KEY_MAX;
        }
        __syncthreads();
        if (n2 > 1) {
            // both arrays share the network (two independent sorts)
            for (int k = 2; k <= n2; k <<= 1) {
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int it = tid; it < n2; it += blockDim.x) {
                        uint64_t *buf = it < (n2 >> 1) ? nfk : nrk;
                        const int i = it < (n2 >> 1) ? it : it - (n2 >> 1);
                        const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                        const int hi = lo | j;
                        const uint64_t x = buf[lo], y = buf[hi];
                        if ((x > y) == ((lo & k) == 0)) {
                            buf[lo] = y;
                            buf[hi] = x;
                        }
                    }
                    __syncthreads();
                }
            }
        }

        // ---- merge into frontier and results (ping-pong buffers)
        const int cf = s_cur_f, cr = s_cur_r;
        const int head = s_head, nf = s_nf, nr = s_nr;
        merge_path(fr0 + cf * G_FC + head, nf - head, nfk, nnf, fr0 + (cf ^ 1) * G_FC, G_FC);
        merge_path(rs0 + cr * G_RC, nr, nrk, nnr, rs0 + (cr ^ 1) * G_RC, ef);
        __syncthreads();
        if (tid == 0) {
            s_nf = min(nf - head + nnf, G_FC);
            s_head = 0;
            s_cur_f = cf ^ 1;
            s_nr = min(nr + nnr, ef);
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
        h.node = key_row(R[i]);
        h.dist = key_dist(R[i]);
        a.out[(uint64_t)q * ef + i] = h;
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
    return (size_t)(2 * G_FC + 2 * G_RC + 2 * G_NB) * 8 + (size_t)(G_HC + G_NB) * 4 +
           (size_t)dpad * 4;
}

cudaError_t launch_graph(const GraphArgs &a, int nq, cudaStream_t st) {
    const size_t smem = graph_smem_bytes(a.dpad);
    cudaError_t e =
        cudaFuncSetAttribute(graph_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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

int graph_run_host(FvGpuIndex *g, int nq, const float *queries, const uint32_t *entries,
                   const PredBatch &pb, uint32_t ef, uint64_t max_visited, FvHit *out,
                   uint32_t *out_cnt, uint8_t *exhausted, char *errbuf, size_t errlen) {
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
    GraphScratch &gs = g->graph;
    const int P = db.P;
    cudaEventRecord(g->ev0, g->stream);
    if (P > 0) {
        PV_CUDA_OK(s.bitmaps.ensure((size_t)P * bm_words * 4), errbuf, errlen);
        PV_CUDA_OK(s.popcnt.ensure((size_t)P * 8), errbuf, errlen);
        PV_CUDA_OK(launch_bitmaps(g->d_cols, g->count, (const PredInsn *)(d + db.off_insns),
                                  (const PredProg *)(d + db.off_progs),
                                  (const double *)(d + db.off_consts), P,
                                  s.bitmaps.as<uint32_t>(), bm_words,
                                  s.popcnt.as<unsigned long long>(), g->sm_count, g->stream,
                                  db.ninsns, db.nconsts),
                   errbuf, errlen);
    }
    PV_CUDA_OK(gs.visited.ensure((size_t)nq * bm_words * 4), errbuf, errlen);
    const size_t hit_bytes = (size_t)nq * ef * sizeof(FvHit);
    const size_t off_cnt = (hit_bytes + 255) & ~(size_t)255;
    const size_t off_exh = off_cnt + (((size_t)nq * 4 + 255) & ~(size_t)255);
    const size_t off_st = off_exh + (((size_t)nq + 255) & ~(size_t)255);
    const size_t obytes = off_st + (size_t)nq * 16;
    PV_CUDA_OK(s.out_d.ensure(obytes), errbuf, errlen);
    PV_CUDA_OK(s.out_h.ensure(obytes), errbuf, errlen);
    char *od = s.out_d.as<char>();

    GraphArgs a;
    a.vecs = g->d_vecs;
    a.dpad = g->dpad;
    a.nrows = g->count;
    a.adj = g->d_adj;
    a.deg = g->d_deg;
    a.deg_cap = g->deg_cap;
    a.queries = (const float *)(d + db.off_q);
    a.entries = (const uint32_t *)(d + off_ent);
    a.qprog = (const int32_t *)(d + db.off_qprog);
    a.bitmaps = s.bitmaps.as<uint32_t>();
    a.bm_words = bm_words;
    a.ef = (int)ef;
    a.max_visited = max_visited;
    int wmax = G_NB / (g->deg_cap > 0 ? g->deg_cap : 1);
    if (wmax > 16) wmax = 16;
    if (wmax < 1) wmax = 1;
    a.wmax = wmax;
    a.visited_bits = gs.visited.as<uint32_t>();
    a.out = (FvHit *)od;
    a.out_cnt = (uint32_t *)(od + off_cnt);
    a.out_exh = (uint8_t *)(od + off_exh);
    a.stats = (uint32_t *)(od + off_st);
    PV_CUDA_OK(launch_graph(a, nq, g->stream), errbuf, errlen);
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
