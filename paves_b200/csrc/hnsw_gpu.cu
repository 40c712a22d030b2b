// hnsw_gpu.cu — HNSW graph construction on the GPU.
//
// No counterpart in the reference: its builder is a CPU thread pool that
// inserts rows one at a time (engine.cpp:698-1032). Here rows are inserted
// in batches of doubling size (64, then as many as are already in), and
// each batch takes exact candidates instead of insertion-time beam searches:
//   1. candidates: each new node's C nearest nodes among all nodes inserted
//      so far (its own batch included), exact, from this library's scans
//      with the new nodes as queries over the prefix of the rows (the BF16
//      tensor-core scan when its distances are certified exact, else the
//      exact FP32 scan). Rows are in random order, so the early batches are
//      sparse samples of the data and their lists carry the long-range
//      links an insertion order gives a navigable graph;
//   2. forward selection, one warp per new node: candidates in ascending
//      distance, a candidate is kept when it is closer to the node than to
//      every neighbour kept so far (the neighbour-selection heuristic of
//      the HNSW paper, Malkov & Yashunin, Algorithm 4), up to R; a list
//      left short is topped up with the closest rejected candidates;
//   3. reverse edges: every kept edge u -> v of a new node is offered to v
//      (in-degrees counted with atomics, a prefix sum, a scatter into
//      per-node runs);
//   4. re-selection, one warp per touched node: its current list and its
//      new reverse candidates sorted together (duplicates dropped) and
//      selected again by the same rule to R.
// Level 0 uses R = 2M over all rows, each level L >= 1 uses R = M over the
// nodes whose level is >= L (a sub-index of their rows). Node levels are
// drawn as the engine draws them (so upper levels have the usual sizes),
// the entry point is the lowest-numbered node of the top level. The result
// is a graph in the index-file layout (PvHnsw), searched by the same code
// as any other; its quality contract is search recall, not identity with
// the engine's graph.
#include <string.h>

#include <algorithm>
#include <vector>

#include "index.h"
#include "paves_ext.h"
#include "pv_internal.h"
#include "tc_core.cuh"

namespace pv {

constexpr int HG_CAP = 512;      // candidates per node in the final selection
constexpr int HG_WARPS = 8;      // warps per block of the selection kernels
constexpr int HG_RMAX = 128;     // largest R (2M with M <= 64)

// squared L2 of rows a and b of x (stride dpad), reduced across the warp;
// the a row is passed in registers (lane owns dims 4 lane + 128 i)
template <int NV>
__device__ __forceinline__ float hg_dist(const float4 (&ra)[NV], const float *x, uint64_t b,
                                         int dpad, int lane) {
    const float *pb = x + b * (uint64_t)dpad;
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const int j = i * 128 + lane * 4;
        if (j < dpad) {
            const float4 v = __ldg((const float4 *)(pb + j));
            const float d0 = ra[i].x - v.x, d1 = ra[i].y - v.y, d2 = ra[i].z - v.z,
                        d3 = ra[i].w - v.w;
            s = fmaf(d0, d0, s);
            s = fmaf(d1, d1, s);
            s = fmaf(d2, d2, s);
            s = fmaf(d3, d3, s);
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

template <int NV>
__device__ __forceinline__ void hg_row(float4 (&r)[NV], const float *x, uint64_t a, int dpad,
                                       int lane) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const int j = i * 128 + lane * 4;
        r[i] = j < dpad ? __ldg((const float4 *)(x + a * (uint64_t)dpad + j))
                        : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// The selection rule on n ascending candidate keys of node v (smem, warp
// private): keeps up to R candidates, topping up from rejected ones; kept[]
// receives their positions in ck. Returns the number kept. Keys of v
// itself are skipped.
template <int NV>
__device__ int hg_select(const uint64_t *ck, int n, uint32_t v, int R, const float *x, int dpad,
                         uint32_t *kept, uint32_t *rej, int lane) {
    int nk = 0, nr = 0;
    for (int i = 0; i < n && nk < R; i++) {
        const uint32_t c = key_row(ck[i]);
        if (c == v) continue;
        const float dc = key_dist(ck[i]);
        float4 rc[NV];
        hg_row<NV>(rc, x, c, dpad, lane);
        bool ok = true;
        for (int j = 0; j < nk && ok; j++)
            if (hg_dist<NV>(rc, x, key_row(ck[kept[j]]), dpad, lane) < dc) ok = false;
        if (lane == 0) {
            if (ok) kept[nk] = (uint32_t)i;
            else if (nr < R) rej[nr] = (uint32_t)i;
        }
        __syncwarp();
        if (ok) nk++;
        else if (nr < R) nr++;
    }
    // top up in ascending distance: merge of the kept and rejected positions
    // is not needed, the rejected ones come after (keys stay sorted only
    // within each group, and lists need no order)
    for (int i = 0; i < nr && nk < R; i++) {
        if (lane == 0) kept[nk] = rej[i];
        __syncwarp();
        nk++;
    }
    return nk;
}

// Step 2: forward selection for nodes [n0, n0 + nq) from their scan answers
// (cand [nq][topb] ascending, cnt [nq]); out: fwd keys [node][R] + counts.
template <int NV>
__global__ void __launch_bounds__(32 * HG_WARPS)
hg_forward_kernel(const FvHit *__restrict__ cand, const uint32_t *__restrict__ ccnt, int topb,
                  uint64_t n0, int nq, int R, const float *__restrict__ x, int dpad,
                  uint64_t *__restrict__ fwd, uint32_t *__restrict__ fwd_cnt) {
    __shared__ uint64_t s_ck[HG_WARPS][HG_CAP];
    __shared__ uint32_t s_kept[HG_WARPS][HG_RMAX], s_rej[HG_WARPS][HG_RMAX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * HG_WARPS + warp;
    if (q >= nq) return;
    const uint64_t v = n0 + q;
    const int n = min((int)ccnt[q], min(topb, HG_CAP));
    for (int i = lane; i < n; i += 32) {
        const FvHit h = cand[(uint64_t)q * topb + i];
        s_ck[warp][i] = make_key(h.dist, (uint32_t)h.node);
    }
    __syncwarp();
    const int nk = hg_select<NV>(s_ck[warp], n, (uint32_t)v, R, x, dpad, s_kept[warp],
                                 s_rej[warp], lane);
    for (int j = lane; j < nk; j += 32) fwd[v * R + j] = s_ck[warp][s_kept[warp][j]];
    if (lane == 0) fwd_cnt[v] = (uint32_t)nk;
}

// Step 3: in-degrees, then the scatter of reverse edges into per-node runs.
// (edges of the sources [u0, u0 + nu))
__global__ void hg_count_kernel(const uint64_t *__restrict__ fwd,
                                const uint32_t *__restrict__ fwd_cnt, uint64_t u0, uint64_t nu,
                                int R, uint32_t *__restrict__ in_cnt) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nu * (uint64_t)R) return;
    const uint64_t u = u0 + i / R;
    if ((uint32_t)(i % R) >= fwd_cnt[u]) return;
    atomicAdd(&in_cnt[key_row(fwd[u * R + i % R])], 1u);
}

__global__ void hg_scatter_kernel(const uint64_t *__restrict__ fwd,
                                  const uint32_t *__restrict__ fwd_cnt, uint64_t u0, uint64_t nu,
                                  int R, const uint64_t *__restrict__ in_off,
                                  uint32_t *__restrict__ cursor, uint64_t *__restrict__ rev) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nu * (uint64_t)R) return;
    const uint64_t u = u0 + i / R;
    if ((uint32_t)(i % R) >= fwd_cnt[u]) return;
    const uint64_t k = fwd[u * R + i % R];
    const uint32_t v = key_row(k);
    const uint32_t pos = atomicAdd(&cursor[v], 1u);
    rev[in_off[v] + pos] = make_key(key_dist(k), (uint32_t)u);
}

// Step 4: re-selection over a node's list and its new reverse candidates,
// for the nodes [0, n) touched by this batch (new nodes >= lo, or with
// reverse edges); the list (keys, in place) and its count are rewritten.
template <int NV>
__global__ void __launch_bounds__(32 * HG_WARPS)
hg_final_kernel(uint64_t *__restrict__ fwd, uint32_t *__restrict__ fwd_cnt,
                const uint64_t *__restrict__ rev, const uint64_t *__restrict__ in_off,
                const uint32_t *__restrict__ in_cnt, uint64_t n, uint64_t lo, int R,
                const float *__restrict__ x, int dpad) {
    __shared__ uint64_t s_ck[HG_WARPS][HG_CAP];
    __shared__ uint32_t s_kept[HG_WARPS][HG_RMAX], s_rej[HG_WARPS][HG_RMAX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t v = (uint64_t)blockIdx.x * HG_WARPS + warp;
    if (v >= n || (v < lo && in_cnt[v] == 0)) return;
    uint64_t *ck = s_ck[warp];
    const int nf = (int)fwd_cnt[v];
    // reverse runs longer than the buffer keep their first entries (rare:
    // in-degrees of a pruned neighbour graph stay a small multiple of R)
    const int nr = min((int)in_cnt[v], HG_CAP - nf);
    for (int i = lane; i < nf; i += 32) ck[i] = fwd[v * R + i];
    for (int i = lane; i < nr; i += 32) ck[nf + i] = rev[in_off[v] + i];
    const int n1 = nf + nr;
    int n2 = 1;
    while (n2 < n1) n2 <<= 1;
    for (int i = n1 + lane; i < n2; i += 32) ck[i] = KEY_MAX;
    __syncwarp();
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < (n2 >> 1); i += 32) {
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo | j;
                const uint64_t a = ck[lo], b = ck[hi];
                if ((a > b) == ((lo & k) == 0)) {
                    ck[lo] = b;
                    ck[hi] = a;
                }
            }
            __syncwarp();
        }
    // drop duplicates (an edge present both ways has one key: distances
    // are symmetric)
    int m = 0;
    uint64_t last = KEY_MAX;  // the previous chunk's last key (pads are beyond n1)
    for (int base = 0; base < n1; base += 32) {
        const int i = base + lane;
        const uint64_t k = i < n1 ? ck[i] : KEY_MAX;
        uint64_t p = __shfl_up_sync(0xffffffffu, k, 1);
        if (lane == 0) p = last;
        last = __shfl_sync(0xffffffffu, k, 31);
        const bool keep = i < n1 && k != p;
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        __syncwarp();  // every lane has read its keys before the compaction writes
        if (keep) ck[m + __popc(bal & ((1u << lane) - 1u))] = k;
        m += __popc(bal);
        __syncwarp();
    }
    const int nk = hg_select<NV>(ck, m, (uint32_t)v, R, x, dpad, s_kept[warp], s_rej[warp], lane);
    for (int j = lane; j < nk; j += 32) fwd[v * R + j] = ck[s_kept[warp][j]];
    if (lane == 0) fwd_cnt[v] = (uint32_t)nk;
}

// The lists in the file layout: [cnt, ids...] of stride R + 1.
__global__ void hg_export_kernel(const uint64_t *__restrict__ lst,
                                 const uint32_t *__restrict__ cnt, uint64_t n, int R,
                                 uint32_t *__restrict__ lists) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * (uint64_t)(R + 1)) return;
    const uint64_t v = i / (R + 1);
    const int j = (int)(i % (R + 1));
    const uint32_t c = cnt[v];
    lists[i] = j == 0 ? c : (uint32_t)(j - 1) < c ? key_row(lst[v * R + j - 1]) : 0u;
}

namespace {

struct DevArr {
    void *p = nullptr;
    ~DevArr() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
    template <typename T>
    T *as() const {
        return (T *)p;
    }
};

#define HG_OK(call)                                                                  \
    do {                                                                             \
        cudaError_t e__ = (call);                                                    \
        if (e__ != cudaSuccess) {                                                    \
            if (errbuf && errlen)                                                    \
                snprintf(errbuf, errlen, "hnsw gpu: %s: %s", #call,                  \
                         cudaGetErrorString(e__));                                   \
            return -1;                                                               \
        }                                                                            \
    } while (0)

template <int NV>
void launch_forward(const FvHit *cand, const uint32_t *ccnt, int topb, uint64_t n0, int nq, int R,
                    const float *x, int dpad, uint64_t *fwd, uint32_t *fwd_cnt, cudaStream_t st) {
    hg_forward_kernel<NV><<<(nq + HG_WARPS - 1) / HG_WARPS, 32 * HG_WARPS, 0, st>>>(
        cand, ccnt, topb, n0, nq, R, x, dpad, fwd, fwd_cnt);
}
template <int NV>
void launch_final(uint64_t *fwd, uint32_t *fwd_cnt, const uint64_t *rev, const uint64_t *in_off,
                  const uint32_t *in_cnt, uint64_t n, uint64_t lo, int R, const float *x,
                  int dpad, cudaStream_t st) {
    hg_final_kernel<NV><<<(unsigned)((n + HG_WARPS - 1) / HG_WARPS), 32 * HG_WARPS, 0, st>>>(
        fwd, fwd_cnt, rev, in_off, in_cnt, n, lo, R, x, dpad);
}

// Exact nearest neighbours of rows [r0, r0 + nq) of g among all rows of g:
// the tensor-core scan when its BF16 distances are certified exact for
// these rows, else the exact FP32 scan (queries read in place from g's f32
// rows). out [nq][topb] ascending, cnt [nq].
int knn_batch(FvGpuIndex *g, uint64_t r0, int nq, uint32_t topb, const int32_t *d_qprog,
              const unsigned long long *d_popcnt, FvHit *d_out, uint32_t *d_cnt, uint8_t *d_tr,
              char *errbuf, size_t errlen) {
    const float *d_q = g->d_vecs + r0 * (uint64_t)g->dpad;
    const uint64_t bm_words = (g->count + 31) / 32;
    // (lists of at most 64 keys hold the whole answer: no certification)
    if (g->precision != FV_GPU_PREC_FP32 && tc_supported(g) && topb <= 64 &&
        tc_superset(g, topb, g->row_amax) == (int)topb) {
        return launch_scan_tc(g, nq, g->row_amax, d_q, d_qprog, nullptr, bm_words, d_popcnt,
                              topb, d_out, d_cnt, d_tr, nullptr, errbuf, errlen);
    }
    ScanPlan pl;
    const bool tiled = plan_scan_f32t(g->count, g->dpad, nq, (int)topb, g->sm_count, pl);
    if (!tiled && !plan_scan_f32(g->count, g->dpad, nq, (int)topb, g->sm_count, pl)) {
        snprintf(errbuf, errlen, "hnsw gpu: dimension %d not supported by the scan", g->dim);
        return -1;
    }
    ScanScratch &s = g->scan;
    PV_CUDA_OK(s.tau.ensure((size_t)nq * 8), errbuf, errlen);
    PV_CUDA_OK(s.part.ensure((size_t)nq * pl.grow * topb * 8), errbuf, errlen);
    PV_CUDA_OK(s.part_cnt.ensure((size_t)nq * pl.grow * 4), errbuf, errlen);
    PV_CUDA_OK(cudaMemsetAsync(s.tau.p, 0xFF, (size_t)nq * 8, g->stream), errbuf, errlen);
    ScanF32Args a;
    a.vecs = g->d_vecs;
    a.nrows = g->count;
    a.dpad = g->dpad;
    a.queries = d_q;
    a.nq = nq;
    a.bitmaps = nullptr;
    a.bm_words = bm_words;
    a.qprog = d_qprog;
    a.K = (int)topb;
    a.S = pl.S;
    a.CB = pl.CB;
    a.rows_per_cta = pl.rows_per_cta;
    a.grow = pl.grow;
    a.qtiles = pl.qtiles;
    a.tau = s.tau.as<unsigned long long>();
    a.part = s.part.as<uint64_t>();
    a.part_cnt = s.part_cnt.as<uint32_t>();
    PV_CUDA_OK(tiled ? launch_scan_f32t(a, pl, g->stream) : launch_scan_f32(a, pl, g->stream),
               errbuf, errlen);
    PV_CUDA_OK(launch_merge(a.part, a.part_cnt, pl.grow, (int)topb, pl, a.tau, d_qprog, d_popcnt,
                            g->count, nq, d_out, d_cnt, d_tr, g->stream),
               errbuf, errlen);
    return 0;
}

// One level over the rows of g by batched insertion: lists [count][R + 1]
// (device) of local ids.
int build_level(FvGpuIndex *g, int R, int C, uint32_t *d_lists, char *errbuf, size_t errlen) {
    const uint64_t n = g->count;
    const int dpad = g->dpad;
    const int NVn = (dpad + 127) / 128;
    const int B = 2048;          // scan batch (queries per call)
    // first insertion batch: a few rows spread over the whole data set, so
    // the earliest lists link distant regions (then doubling batches)
    const uint64_t first = 64;
    cudaStream_t st = g->stream;
    // the rows' tensor map covers all rows, whatever prefix is scanned
    if (g->precision != FV_GPU_PREC_FP32 && !g->tmap_x_ok) {
        CUtensorMap m;
        if (!tc_make_tmap(&m, g->d_vlow, g->precision == FV_GPU_PREC_FP8 ? TCK_FP8 : TCK_BF16,
                          (uint64_t)g->kpad,
                          g->count)) {
            snprintf(errbuf, errlen, "hnsw gpu: tensor map encoding failed");
            return -1;
        }
        memcpy(g->tmap_x, &m, sizeof(m));
        g->tmap_x_ok = true;
    }
    DevArr qprog, popcnt, out, cnt, tr, lst, lcnt, in_cnt, in_off, cursor, rev;
    const int topb_max = (int)std::min<uint64_t>((uint64_t)C + 1, n);  // self included
    HG_OK(qprog.alloc((size_t)B * 4));
    HG_OK(cudaMemsetAsync(qprog.p, 0xFF, (size_t)B * 4, st));  // no filter
    HG_OK(popcnt.alloc(8));
    HG_OK(out.alloc((size_t)B * topb_max * sizeof(FvHit)));
    HG_OK(cnt.alloc((size_t)B * 4));
    HG_OK(tr.alloc((size_t)B));
    HG_OK(lst.alloc((size_t)n * R * 8));
    HG_OK(lcnt.alloc((size_t)n * 4));
    HG_OK(in_cnt.alloc((size_t)n * 4));
    HG_OK(cursor.alloc((size_t)n * 4));
    HG_OK(in_off.alloc((size_t)(n + 1) * 8));
    HG_OK(cudaMemsetAsync(lcnt.p, 0, (size_t)n * 4, st));
    std::vector<uint32_t> h_in;
    std::vector<uint64_t> h_off;
    size_t rev_cap = 0;
    int rc = 0;
    for (uint64_t lo = 0; lo < n && rc == 0;) {
        const uint64_t hi = lo == 0 ? std::min(n, first) : std::min(n, 2 * lo);
        // 1-2: candidates among the inserted prefix [0, hi), forward selection
        g->count = hi;
        const int topb = (int)std::min<uint64_t>((uint64_t)C + 1, hi);
        for (uint64_t r0 = lo; r0 < hi && rc == 0; r0 += B) {
            const int nq = (int)std::min<uint64_t>(B, hi - r0);
            rc = knn_batch(g, r0, nq, (uint32_t)topb, qprog.as<int32_t>(),
                           popcnt.as<unsigned long long>(), out.as<FvHit>(), cnt.as<uint32_t>(),
                           tr.as<uint8_t>(), errbuf, errlen);
            if (rc) break;
            if (NVn <= 1)
                launch_forward<1>(out.as<FvHit>(), cnt.as<uint32_t>(), topb, r0, nq, R, g->d_vecs,
                                  dpad, lst.as<uint64_t>(), lcnt.as<uint32_t>(), st);
            else if (NVn <= 2)
                launch_forward<2>(out.as<FvHit>(), cnt.as<uint32_t>(), topb, r0, nq, R, g->d_vecs,
                                  dpad, lst.as<uint64_t>(), lcnt.as<uint32_t>(), st);
            else
                launch_forward<4>(out.as<FvHit>(), cnt.as<uint32_t>(), topb, r0, nq, R, g->d_vecs,
                                  dpad, lst.as<uint64_t>(), lcnt.as<uint32_t>(), st);
            if (cudaGetLastError() != cudaSuccess) rc = -1;
        }
        g->count = n;
        if (rc) break;
        if ((rc = check_tc_watchdog(g, errbuf, errlen))) break;
        // 3: reverse edges of the new nodes' lists
        const uint64_t nu = hi - lo;
        HG_OK(cudaMemsetAsync(in_cnt.p, 0, (size_t)hi * 4, st));
        HG_OK(cudaMemsetAsync(cursor.p, 0, (size_t)hi * 4, st));
        const unsigned eb = (unsigned)((nu * R + 255) / 256);
        hg_count_kernel<<<eb, 256, 0, st>>>(lst.as<uint64_t>(), lcnt.as<uint32_t>(), lo, nu, R,
                                            in_cnt.as<uint32_t>());
        HG_OK(cudaGetLastError());
        h_in.resize(hi);
        h_off.resize(hi + 1);
        HG_OK(cudaMemcpyAsync(h_in.data(), in_cnt.p, (size_t)hi * 4, cudaMemcpyDeviceToHost, st));
        HG_OK(cudaStreamSynchronize(st));
        uint64_t tot = 0;
        for (uint64_t i = 0; i < hi; i++) {
            h_off[i] = tot;
            tot += h_in[i];
        }
        h_off[hi] = tot;
        HG_OK(cudaMemcpyAsync(in_off.p, h_off.data(), (size_t)(hi + 1) * 8,
                              cudaMemcpyHostToDevice, st));
        if (tot > rev_cap) {
            if (rev.p) {
                HG_OK(cudaStreamSynchronize(st));
                cudaFree(rev.p);
                rev.p = nullptr;
            }
            HG_OK(rev.alloc((size_t)tot * 8));
            rev_cap = tot;
        }
        hg_scatter_kernel<<<eb, 256, 0, st>>>(lst.as<uint64_t>(), lcnt.as<uint32_t>(), lo, nu, R,
                                              in_off.as<uint64_t>(), cursor.as<uint32_t>(),
                                              rev.as<uint64_t>());
        HG_OK(cudaGetLastError());
        // 4: re-selection of every touched list
        if (NVn <= 1)
            launch_final<1>(lst.as<uint64_t>(), lcnt.as<uint32_t>(), rev.as<uint64_t>(),
                            in_off.as<uint64_t>(), in_cnt.as<uint32_t>(), hi, lo, R, g->d_vecs,
                            dpad, st);
        else if (NVn <= 2)
            launch_final<2>(lst.as<uint64_t>(), lcnt.as<uint32_t>(), rev.as<uint64_t>(),
                            in_off.as<uint64_t>(), in_cnt.as<uint32_t>(), hi, lo, R, g->d_vecs,
                            dpad, st);
        else
            launch_final<4>(lst.as<uint64_t>(), lcnt.as<uint32_t>(), rev.as<uint64_t>(),
                            in_off.as<uint64_t>(), in_cnt.as<uint32_t>(), hi, lo, R, g->d_vecs,
                            dpad, st);
        HG_OK(cudaGetLastError());
        HG_OK(cudaStreamSynchronize(st));  // rev and the host offsets are reused next batch
        lo = hi;
    }
    g->count = n;
    if (rc) return -1;
    const uint64_t total = n * (uint64_t)(R + 1);
    hg_export_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        lst.as<uint64_t>(), lcnt.as<uint32_t>(), n, R, d_lists);
    HG_OK(cudaGetLastError());
    HG_OK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace
}  // namespace pv

using namespace pv;

extern "C" PvHnsw *pv_hnsw_build_gpu(const float *vectors, uint64_t count, int dim, int M,
                                     int candidates, int device, int precision, char *errbuf,
                                     size_t errlen) {
    if (!vectors || count == 0 || dim <= 0 || dim > 512 || M < 2 || M > HG_RMAX / 2 ||
        candidates < 2 * M || candidates > 1023 ||
        (precision != FV_GPU_PREC_FP32 && precision != FV_GPU_PREC_BF16)) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "hnsw gpu: bad build parameters");
        return nullptr;
    }
    if (count >= 0xFFFFFFFFull) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "hnsw gpu: too many rows");
        return nullptr;
    }
    PvHnsw *h = hnsw_sections(vectors, count, dim, M);
    const uint8_t *lev = hnsw_levels(h);
    int top = 0;
    uint64_t entry = 0;
    for (uint64_t i = 0; i < count; i++)
        if (lev[i] > top) {
            top = lev[i];
            entry = i;
        }
    auto fail = [&]() -> PvHnsw * {
        pv_hnsw_free(h);
        return nullptr;
    };
    // level 0: all rows, R = 2M
    {
        FvGpuIndex *g = fv_gpu_index_upload(vectors, nullptr, nullptr, nullptr, 0, count, dim, 0,
                                            device, precision, errbuf, errlen);
        if (!g) return fail();
        int rc = 0;
        uint32_t *d_lists = nullptr;
        const int R = 2 * M;
        {
            std::lock_guard<std::mutex> lk(g->mu);
            if (cudaMalloc(&d_lists, (size_t)count * (R + 1) * 4) != cudaSuccess) rc = -1;
            if (!rc) rc = build_level(g, R, candidates, d_lists, errbuf, errlen);
            if (!rc && cudaMemcpy(hnsw_l0(h), d_lists, (size_t)count * (R + 1) * 4,
                                  cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = -1;
        }
        if (d_lists) cudaFree(d_lists);
        fv_gpu_index_free(g);
        if (rc) {
            if (errbuf && errlen && !errbuf[0]) snprintf(errbuf, errlen, "hnsw gpu: level 0 failed");
            return fail();
        }
    }
    // levels 1..top: the nodes of each level, R = M
    for (int L = 1; L <= top; L++) {
        std::vector<uint32_t> ids;
        for (uint64_t i = 0; i < count; i++)
            if (lev[i] >= L) ids.push_back((uint32_t)i);
        const uint64_t n = ids.size();
        if (n < 2) continue;  // a single node has no neighbours
        std::vector<float> sub(n * (uint64_t)dim);
        for (uint64_t i = 0; i < n; i++)
            memcpy(&sub[i * dim], vectors + (uint64_t)ids[i] * dim, sizeof(float) * dim);
        FvGpuIndex *g = fv_gpu_index_upload(sub.data(), nullptr, nullptr, nullptr, 0, n, dim, 0,
                                            device, precision, errbuf, errlen);
        if (!g) return fail();
        const int R = M;
        // upper levels are small: twice the candidates (exact FP32 scans)
        const int C = (int)std::min<uint64_t>((uint64_t)std::min(2 * candidates + 1, 1023), n - 1);
        std::vector<uint32_t> lists(n * (R + 1));
        uint32_t *d_lists = nullptr;
        int rc = 0;
        {
            std::lock_guard<std::mutex> lk(g->mu);
            if (cudaMalloc(&d_lists, lists.size() * 4) != cudaSuccess) rc = -1;
            if (!rc) rc = build_level(g, R, C, d_lists, errbuf, errlen);
            if (!rc && cudaMemcpy(lists.data(), d_lists, lists.size() * 4,
                                  cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = -1;
        }
        if (d_lists) cudaFree(d_lists);
        fv_gpu_index_free(g);
        if (rc) return fail();
        for (uint64_t i = 0; i < n; i++) {
            uint32_t *dst = hnsw_upper_list(h, ids[i], L);
            const uint32_t *src = &lists[i * (R + 1)];
            dst[0] = src[0];
            for (uint32_t j = 0; j < src[0]; j++) dst[1 + j] = ids[src[1 + j]];
        }
    }
    hnsw_set_entry(h, entry, top, candidates);
    return h;
}
