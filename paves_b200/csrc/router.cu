// router.cu — the learned scan-vs-graph router: query features, and a
// 12 -> 64 -> 64 -> 5 MLP (ReLU) with bf16 weights and fp32 accumulation,
// trained on the GPU by the kernels in this file.
//
// No reference counterpart: the reference routes by its planner cost rule
// (extension/paves/src/planner.c:185-346) and picks the beam width by the
// selectivity rule of exec.c:415-424. This router predicts, per query, one
// of five actions — 0 = scan, 1..4 = graph search at ef 32/64/128/256 —
// from 12 features:
//   f0   log10(selectivity), selectivity = popcount of the query's
//        predicate bitmap / rows (1 without a predicate)
//   f1   |q|
//   f2-9 distances to the 8 nearest of the router's centroids, ascending
//   f10  log2(k)
//   f11  predicate kind: 0 none, 1 compare, 2 IN, 3 AND, 4 OR, 5 NOT (root)
// Inputs are standardized by a per-feature mean/std stored with the
// weights. Training: softmax cross-entropy weighted per sample, Adam on
// fp32 master weights; every forward (training and inference) multiplies
// by the bf16-rounded weights and accumulates in fp32, and the gradients
// are those of that forward.
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <random>
#include <vector>

#include "paves_ext.h"
#include "pv_internal.h"

namespace pv {

constexpr int NI = PV_MLP_IN, NH = PV_MLP_HIDDEN, NO = PV_MLP_OUT;
constexpr int P_W1 = 0;
constexpr int P_B1 = P_W1 + NI * NH;
constexpr int P_W2 = P_B1 + NH;
constexpr int P_B2 = P_W2 + NH * NH;
constexpr int P_W3 = P_B2 + NH;
constexpr int P_B3 = P_W3 + NH * NO;
constexpr int P_N = P_B3 + NO;
static_assert(P_N == PV_MLP_NPARAMS, "parameter layout");

// ---------------------------------------------------------------- features
// One CTA per query; each thread scores its share of the centroids (four
// rows at a time) and keeps a sorted top-8; each warp reduces its lanes'
// lists to a top-8 by 8 rounds of warp-wide minimum, and warp 0 does the
// same over the 8 warps' lists. Under 1 KB of shared memory, so the kernel
// can run beside a scan that holds most of each SM's.
__device__ __forceinline__ float pick8(const float (&t)[8], int i) {
    float v = INFINITY;
#pragma unroll
    for (int j = 0; j < 8; j++)
        if (j == i) v = t[j];
    return v;
}

__device__ __forceinline__ void warp_argmin(float &best, int &who) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int ow = __shfl_xor_sync(0xffffffffu, who, o);
        if (ov < best || (ov == best && ow < who)) {
            best = ov;
            who = ow;
        }
    }
}

__global__ void __launch_bounds__(256) router_features_kernel(
    const float *__restrict__ queries, int dpad, const float *__restrict__ cent, int ncent,
    const unsigned long long *__restrict__ popcnt, const int32_t *__restrict__ qprog,
    uint64_t nrows, const uint32_t *__restrict__ kq, const int32_t *__restrict__ kind,
    float *__restrict__ feats) {
    extern __shared__ float rsm[];
    float *sq = rsm;              // [dpad]
    __shared__ float cand[64];    // [8 warps][8]
    __shared__ float s_norm;
    const int q = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int j = tid; j < dpad; j += blockDim.x) sq[j] = queries[(uint64_t)q * dpad + j];
    __syncthreads();
    if (warp == 0) {
        float s = 0.f;
        for (int j = lane; j < dpad; j += 32) s = fmaf(sq[j], sq[j], s);
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) s_norm = sqrtf(s);
    }
    // thread-per-centroid: each thread walks whole centroid rows (several
    // rows' loads in flight), keeping its sorted top-8
    float top[8];
#pragma unroll
    for (int i = 0; i < 8; i++) top[i] = INFINITY;
    for (int c0 = tid; c0 < ncent; c0 += 4 * blockDim.x) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const float *x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int c = c0 + u * blockDim.x;
            x[u] = cent + (uint64_t)(c < ncent ? c : c0) * dpad;
        }
        for (int j = 0; j < dpad; j += 4) {
            const float4 w = *(const float4 *)(sq + j);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float4 v = __ldg((const float4 *)(x[u] + j));
                const float d0 = v.x - w.x, d1 = v.y - w.y, d2 = v.z - w.z, d3 = v.w - w.w;
                acc[u] = fmaf(d0, d0, acc[u]); acc[u] = fmaf(d1, d1, acc[u]);
                acc[u] = fmaf(d2, d2, acc[u]); acc[u] = fmaf(d3, d3, acc[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (c0 + u * (int)blockDim.x >= ncent || !(acc[u] < top[7])) continue;
            float v = acc[u];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const float t = top[i];
                const bool sw = v < t;
                top[i] = sw ? v : t;
                v = sw ? t : v;
            }
        }
    }
    // the warp's 8 smallest: 8 rounds of minimum over the lanes' list heads
    {
        int head = 0;
        float mine = INFINITY;
        for (int r = 0; r < 8; r++) {
            float best = head < 8 ? pick8(top, head) : INFINITY;
            int who = lane;
            warp_argmin(best, who);
            if (lane == who) head++;
            if (lane == r) mine = best;
        }
        if (lane < 8) cand[warp * 8 + lane] = mine;
    }
    __syncthreads();
    if (warp == 0) {
        float v0 = cand[lane], v1 = cand[lane + 32];
        float out = 0.f;
        for (int r = 0; r < 8; r++) {
            float best = fminf(v0, v1);
            int who = lane;
            warp_argmin(best, who);
            if (lane == who) {  // remove one occurrence of the minimum
                if (v0 <= v1) v0 = INFINITY; else v1 = INFINITY;
            }
            if (lane == r) out = best;
        }
        float *f = feats + (uint64_t)q * NI;
        if (lane < 8) f[2 + lane] = sqrtf(out);
        if (lane == 0) {
            const int pg = qprog[q];
            double sel = pg < 0 ? 1.0 : (double)popcnt[pg] / (double)nrows;
            f[0] = (float)log10(sel > 1e-6 ? sel : 1e-6);
            f[1] = s_norm;
            f[10] = log2f((float)(kq[q] > 0 ? kq[q] : 1));
            f[11] = (float)kind[q];
        }
    }
}

// ------------------------------------------------------------------ MLP
struct MlpDev {
    float *master = nullptr;   // [P_N] fp32
    __nv_bfloat16 *w = nullptr;  // [P_N] forward weights
    float *norm = nullptr;     // [2][NI] mean, std
    float *m = nullptr, *v = nullptr, *grad = nullptr;
};

__device__ __forceinline__ void load_weights(const __nv_bfloat16 *__restrict__ w,
                                             const float *__restrict__ norm, float *sw,
                                             float *snorm) {
    for (int i = threadIdx.x; i < P_N; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
    for (int i = threadIdx.x; i < 2 * NI; i += blockDim.x) snorm[i] = norm[i];
    __syncthreads();
}

// One thread per sample. idx (optional) maps sample s to the row of X.
// Stores the standardized input, both hidden activations (after ReLU) and
// the logits when the pointers are given.
__global__ void __launch_bounds__(128) mlp_forward_kernel(
    const float *__restrict__ X, const uint32_t *__restrict__ idx, const int *__restrict__ off_p,
    int n, const __nv_bfloat16 *__restrict__ w, const float *__restrict__ norm,
    float *__restrict__ Xn, float *__restrict__ H1, float *__restrict__ H2,
    float *__restrict__ Z3) {
    __shared__ float sw[P_N];
    __shared__ float snorm[2 * NI];
    load_weights(w, norm, sw, snorm);
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int off = off_p ? *off_p : 0;
    const uint64_t row = idx ? idx[off + s] : (uint64_t)s;
    float x[NI];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        x[i] = (X[row * NI + i] - snorm[i]) / snorm[NI + i];
        if (Xn) Xn[(uint64_t)s * NI + i] = x[i];
    }
    float h1[NH];
#pragma unroll
    for (int j = 0; j < NH; j++) h1[j] = sw[P_B1 + j];
#pragma unroll
    for (int i = 0; i < NI; i++)
#pragma unroll
        for (int j = 0; j < NH; j++) h1[j] = fmaf(x[i], sw[P_W1 + i * NH + j], h1[j]);
#pragma unroll
    for (int j = 0; j < NH; j++) {
        h1[j] = fmaxf(h1[j], 0.f);
        if (H1) H1[(uint64_t)s * NH + j] = h1[j];
    }
    float z3[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) z3[o] = sw[P_B3 + o];
    // second layer one unit at a time keeps the register count bounded
    for (int j = 0; j < NH; j++) {
        float h = sw[P_B2 + j];
#pragma unroll
        for (int i = 0; i < NH; i++) h = fmaf(h1[i], sw[P_W2 + i * NH + j], h);
        h = fmaxf(h, 0.f);
        if (H2) H2[(uint64_t)s * NH + j] = h;
#pragma unroll
        for (int o = 0; o < NO; o++) z3[o] = fmaf(h, sw[P_W3 + j * NO + o], z3[o]);
    }
#pragma unroll
    for (int o = 0; o < NO; o++) Z3[(uint64_t)s * NO + o] = z3[o];
}

// Inference: one warp per sample, lanes over the hidden units, weights
// read through L1 (no shared memory, so it runs beside a scan). Its sums
// are ordered differently from mlp_forward_kernel's (training) ones.
__global__ void __launch_bounds__(256) mlp_infer_kernel(const float *__restrict__ X, int n,
                                                       const __nv_bfloat16 *__restrict__ w,
                                                       const float *__restrict__ norm,
                                                       float *__restrict__ Z3) {
    const int s = (int)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= n) return;
    const float xi =
        lane < NI ? (X[(uint64_t)s * NI + lane] - __ldg(norm + lane)) / __ldg(norm + NI + lane)
                  : 0.f;
    float h0 = __bfloat162float(w[P_B1 + lane]), h1 = __bfloat162float(w[P_B1 + lane + 32]);
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const float xb = __shfl_sync(0xffffffffu, xi, i);
        h0 = fmaf(xb, __bfloat162float(w[P_W1 + i * NH + lane]), h0);
        h1 = fmaf(xb, __bfloat162float(w[P_W1 + i * NH + lane + 32]), h1);
    }
    h0 = fmaxf(h0, 0.f);
    h1 = fmaxf(h1, 0.f);
    float g0 = __bfloat162float(w[P_B2 + lane]), g1 = __bfloat162float(w[P_B2 + lane + 32]);
#pragma unroll 8
    for (int i = 0; i < NH; i++) {
        const float hb = __shfl_sync(0xffffffffu, i < 32 ? h0 : h1, i & 31);
        g0 = fmaf(hb, __bfloat162float(w[P_W2 + i * NH + lane]), g0);
        g1 = fmaf(hb, __bfloat162float(w[P_W2 + i * NH + lane + 32]), g1);
    }
    g0 = fmaxf(g0, 0.f);
    g1 = fmaxf(g1, 0.f);
#pragma unroll
    for (int o = 0; o < NO; o++) {
        float p = g0 * __bfloat162float(w[P_W3 + lane * NO + o]);
        p = fmaf(g1, __bfloat162float(w[P_W3 + (lane + 32) * NO + o]), p);
#pragma unroll
        for (int x = 16; x; x >>= 1) p += __shfl_xor_sync(0xffffffffu, p, x);
        if (lane == 0) Z3[(uint64_t)s * NO + o] = p + __bfloat162float(w[P_B3 + o]);
    }
}

// Softmax cross-entropy: dZ3 = w_s (p - onehot) / W, W = sum of the batch's
// sample weights (computed by the block-0 reduction below into *wsum).
__global__ void mlp_loss_kernel(const float *__restrict__ Z3, const int32_t *__restrict__ labels,
                                const float *__restrict__ sw_in, const uint32_t *__restrict__ idx,
                                const int *__restrict__ off_p, int n, float *__restrict__ dZ3,
                                float *__restrict__ loss_acc) {
    __shared__ float red[256];
    const int off = off_p ? *off_p : 0;
    // every block computes the batch weight (n is small: one pass)
    float part = 0.f;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const uint64_t row = idx ? idx[off + s] : (uint64_t)s;
        part += sw_in ? sw_in[row] : 1.f;
    }
    red[threadIdx.x] = part;
    __syncthreads();
    for (int st = blockDim.x / 2; st; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    const float W = red[0] > 0.f ? red[0] : 1.f;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint64_t row = idx ? idx[off + s] : (uint64_t)s;
    const float ws = sw_in ? sw_in[row] : 1.f;
    const int y = labels[row];
    float z[NO], mx = -INFINITY;
#pragma unroll
    for (int o = 0; o < NO; o++) {
        z[o] = Z3[(uint64_t)s * NO + o];
        mx = fmaxf(mx, z[o]);
    }
    float se = 0.f;
#pragma unroll
    for (int o = 0; o < NO; o++) {
        z[o] = expf(z[o] - mx);
        se += z[o];
    }
#pragma unroll
    for (int o = 0; o < NO; o++) {
        const float p = z[o] / se;
        dZ3[(uint64_t)s * NO + o] = ws * (p - (o == y ? 1.f : 0.f)) / W;
    }
    if (loss_acc) atomicAdd(loss_acc, ws * (logf(se) - (Z3[(uint64_t)s * NO + y] - mx)) / W);
}

// dZ2 = (W3 dZ3) * [H2 > 0], dZ1 = (W2 dZ2) * [H1 > 0], one thread per sample.
__global__ void __launch_bounds__(128) mlp_backward_kernel(
    const __nv_bfloat16 *__restrict__ w, int n, const float *__restrict__ H1,
    const float *__restrict__ H2, const float *__restrict__ dZ3, float *__restrict__ dZ2,
    float *__restrict__ dZ1) {
    __shared__ float sw[P_N];
    for (int i = threadIdx.x; i < P_N; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float d3[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) d3[o] = dZ3[(uint64_t)s * NO + o];
    float d2[NH];
#pragma unroll
    for (int i = 0; i < NH; i++) {
        float acc = 0.f;
#pragma unroll
        for (int o = 0; o < NO; o++) acc = fmaf(sw[P_W3 + i * NO + o], d3[o], acc);
        d2[i] = H2[(uint64_t)s * NH + i] > 0.f ? acc : 0.f;
        dZ2[(uint64_t)s * NH + i] = d2[i];
    }
    for (int i = 0; i < NH; i++) {
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < NH; j++) acc = fmaf(sw[P_W2 + i * NH + j], d2[j], acc);
        dZ1[(uint64_t)s * NH + i] = H1[(uint64_t)s * NH + i] > 0.f ? acc : 0.f;
    }
}

// One thread per parameter: the sum over the batch of (input x delta).
__global__ void mlp_wgrad_kernel(int n, const float *__restrict__ Xn, const float *__restrict__ H1,
                                 const float *__restrict__ H2, const float *__restrict__ dZ1,
                                 const float *__restrict__ dZ2, const float *__restrict__ dZ3,
                                 float *__restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P_N) return;
    const float *A;
    const float *D;
    int na, nd, i, j;
    if (p < P_B1) { A = Xn; na = NI; D = dZ1; nd = NH; i = (p - P_W1) / NH; j = (p - P_W1) % NH; }
    else if (p < P_W2) { A = nullptr; na = 0; D = dZ1; nd = NH; i = 0; j = p - P_B1; }
    else if (p < P_B2) { A = H1; na = NH; D = dZ2; nd = NH; i = (p - P_W2) / NH; j = (p - P_W2) % NH; }
    else if (p < P_W3) { A = nullptr; na = 0; D = dZ2; nd = NH; i = 0; j = p - P_B2; }
    else if (p < P_B3) { A = H2; na = NH; D = dZ3; nd = NO; i = (p - P_W3) / NO; j = (p - P_W3) % NO; }
    else { A = nullptr; na = 0; D = dZ3; nd = NO; i = 0; j = p - P_B3; }
    float acc = 0.f;
    if (A)
        for (int s = 0; s < n; s++) acc = fmaf(A[(uint64_t)s * na + i], D[(uint64_t)s * nd + j], acc);
    else
        for (int s = 0; s < n; s++) acc += D[(uint64_t)s * nd + j];
    grad[p] = acc;
}

__global__ void mlp_adam_kernel(float *__restrict__ master, __nv_bfloat16 *__restrict__ w,
                                const float *__restrict__ grad, float *__restrict__ m,
                                float *__restrict__ v, const int *__restrict__ step, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P_N) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int t = *step + 1;
    const float g = grad[p];
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float mh = mm / (1.f - powf(b1, (float)t));
    const float vh = vv / (1.f - powf(b2, (float)t));
    const float nw = master[p] - lr * mh / (sqrtf(vh) + eps);
    master[p] = nw;
    w[p] = __float2bfloat16_rn(nw);
}

__global__ void mlp_step_kernel(int *step, int *off, int batch, int steps_per_epoch) {
    const int t = *step + 1;
    *step = t;
    *off = (t % steps_per_epoch) * batch;
}

__global__ void to_bf16_params_kernel(const float *__restrict__ src, __nv_bfloat16 *__restrict__ dst,
                                      int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

}  // namespace pv

using namespace pv;

struct PvRouter {
    int device = 0;
    int ncent = 0, dim = 0, dpad = 0;
    float *d_cent = nullptr;
    MlpDev mlp;
    cudaStream_t stream = nullptr;
    Buf scratch;  // training/inference activations
    Buf io;       // features / labels / weights / permutation
    Buf host{true};
    std::mutex mu;
};

#define RT_OK(x)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            if (errbuf && errlen) snprintf(errbuf, errlen, "router: %s (%s:%d)",   \
                                           cudaGetErrorString(e_), __FILE__, __LINE__); \
            return -1;                                                             \
        }                                                                          \
    } while (0)

extern "C" PvRouter *pv_router_create(int device, const float *centroids, int ncent, int dim,
                                      char *errbuf, size_t errlen) {
    if (!centroids || ncent < 8 || ncent > 65536 || dim < 1 || dim > 4096) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "router: bad centroids (%d x %d)", ncent, dim);
        return nullptr;
    }
    PvRouter *r = new PvRouter();
    r->device = device < 0 ? 0 : device;
    r->ncent = ncent;
    r->dim = dim;
    r->dpad = (dim + 3) & ~3;
    auto fail = [&](cudaError_t e) -> PvRouter * {
        if (errbuf && errlen) snprintf(errbuf, errlen, "router: %s", cudaGetErrorString(e));
        pv_router_free(r);
        return nullptr;
    };
    cudaError_t e = cudaSetDevice(r->device);
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    std::vector<float> pad((size_t)ncent * r->dpad, 0.f);
    for (int c = 0; c < ncent; c++)
        memcpy(&pad[(size_t)c * r->dpad], centroids + (size_t)c * dim, sizeof(float) * dim);
    if ((e = cudaMalloc(&r->d_cent, pad.size() * 4)) != cudaSuccess) return fail(e);
    // on r->stream, in order with the router's kernels (a non-blocking
    // stream does not wait for the legacy default stream)
    if ((e = cudaMemcpyAsync(r->d_cent, pad.data(), pad.size() * 4, cudaMemcpyHostToDevice,
                             r->stream)) != cudaSuccess)
        return fail(e);
    char *blk = nullptr;
    const size_t bytes = (size_t)P_N * (4 * 4 + 2) + 2 * NI * 4 + 256 * 6;
    if ((e = cudaMalloc(&blk, bytes)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(blk, 0, bytes, r->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaStreamSynchronize(r->stream)) != cudaSuccess) return fail(e);
    size_t o = 0;
    auto carve = [&](size_t n) { char *p = blk + o; o += (n + 255) & ~(size_t)255; return p; };
    r->mlp.master = (float *)carve((size_t)P_N * 4);
    r->mlp.m = (float *)carve((size_t)P_N * 4);
    r->mlp.v = (float *)carve((size_t)P_N * 4);
    r->mlp.grad = (float *)carve((size_t)P_N * 4);
    r->mlp.norm = (float *)carve(2 * NI * 4);
    r->mlp.w = (__nv_bfloat16 *)carve((size_t)P_N * 2);
    return r;
}

extern "C" void pv_router_free(PvRouter *r) {
    if (!r) return;
    cudaSetDevice(r->device);
    if (r->d_cent) cudaFree(r->d_cent);
    if (r->mlp.master) cudaFree(r->mlp.master);  // start of the parameter block
    r->scratch.release();
    r->io.release();
    r->host.release();
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
}

extern "C" int pv_router_set_params(PvRouter *r, const float *params, const float *feat_mean,
                                    const float *feat_std, char *errbuf, size_t errlen) {
    if (!r || !params || !feat_mean || !feat_std) return -1;
    for (int i = 0; i < NI; i++)
        if (!(feat_std[i] > 0.f)) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "router: feature %d std must be > 0", i);
            return -1;
        }
    std::lock_guard<std::mutex> lk(r->mu);
    RT_OK(cudaSetDevice(r->device));
    float norm[2 * NI];
    memcpy(norm, feat_mean, NI * 4);
    memcpy(norm + NI, feat_std, NI * 4);
    RT_OK(cudaMemcpyAsync(r->mlp.master, params, (size_t)P_N * 4, cudaMemcpyHostToDevice, r->stream));
    RT_OK(cudaMemcpyAsync(r->mlp.norm, norm, sizeof(norm), cudaMemcpyHostToDevice, r->stream));
    RT_OK(cudaMemsetAsync(r->mlp.m, 0, (size_t)P_N * 4, r->stream));
    RT_OK(cudaMemsetAsync(r->mlp.v, 0, (size_t)P_N * 4, r->stream));
    to_bf16_params_kernel<<<(P_N + 255) / 256, 256, 0, r->stream>>>(r->mlp.master, r->mlp.w, P_N);
    RT_OK(cudaGetLastError());
    RT_OK(cudaStreamSynchronize(r->stream));
    return 0;
}

extern "C" int pv_router_get_params(PvRouter *r, float *params, float *feat_mean,
                                    float *feat_std) {
    if (!r) return -1;
    std::lock_guard<std::mutex> lk(r->mu);
    if (cudaSetDevice(r->device) != cudaSuccess) return -1;
    float norm[2 * NI];
    if (params && cudaMemcpyAsync(params, r->mlp.master, (size_t)P_N * 4,
                                  cudaMemcpyDeviceToHost, r->stream) != cudaSuccess)
        return -1;
    if (cudaMemcpyAsync(norm, r->mlp.norm, sizeof(norm), cudaMemcpyDeviceToHost, r->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(r->stream) != cudaSuccess)
        return -1;
    if (feat_mean) memcpy(feat_mean, norm, NI * 4);
    if (feat_std) memcpy(feat_std, norm + NI, NI * 4);
    return 0;
}

namespace pv {

int router_kind(const FvGpuPredNode *nodes, int nnodes, int32_t root) {
    if (root < 0 || root >= nnodes) return 0;
    switch (nodes[root].kind) {
        case FV_NODE_CMP: return 1;
        case FV_NODE_IN: return 2;
        case FV_NODE_AND: return 3;
        case FV_NODE_OR: return 4;
        default: return 5;
    }
}

size_t router_features_smem(int dpad) { return (size_t)dpad * 4; }

cudaError_t launch_router_features(const PvRouter *r, const float *d_q, int dpad, int nq,
                                   const unsigned long long *popcnt, const int32_t *qprog,
                                   uint64_t nrows, const uint32_t *kq, const int32_t *kind,
                                   float *feats, cudaStream_t st) {
    if (dpad != r->dpad) return cudaErrorInvalidValue;
    const size_t smem = router_features_smem(dpad);
    cudaError_t e = raise_smem_limit((const void *)router_features_kernel, smem);
    if (e != cudaSuccess) return e;
    router_features_kernel<<<nq, 256, smem, st>>>(d_q, dpad, r->d_cent, r->ncent, popcnt, qprog,
                                                  nrows, kq, kind, feats);
    return cudaGetLastError();
}

cudaError_t launch_router_forward(const PvRouter *r, const float *feats, int n, float *Z3,
                                  cudaStream_t st) {
    mlp_infer_kernel<<<(n + 7) / 8, 256, 0, st>>>(feats, n, r->mlp.w, r->mlp.norm, Z3);
    return cudaGetLastError();
}

}  // namespace pv

extern "C" int pv_router_features(PvRouter *r, FvGpuIndex *g, int nq, const float *queries,
                                  const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes,
                                  int nnodes, const int32_t *children, int nchildren,
                                  const double *invals, int ninvals, const uint32_t *k,
                                  float *feats, char *errbuf, size_t errlen) {
    if (!r || !g || nq < 1 || nq > 65536 || !queries || !qd || !k || !feats) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "router: bad feature arguments");
        return -1;
    }
    if (g->dim != r->dim || g->device != r->device) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "router: index dim/device mismatch");
        return -1;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    RT_OK(cudaSetDevice(g->device));
    g->launches = 0;
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return -1;
    DevBatch db;
    db.stage_h = &g->scan.stage_h;
    db.stage_d = &g->scan.stage_d;
    const size_t extra = (size_t)nq * 8;
    if (brute_prepare(g, nq, queries, pb, db, extra, errbuf, errlen)) return -1;
    uint32_t *hk = (uint32_t *)(db.stage_h->as<char>() + db.off_extra);
    int32_t *hkind = (int32_t *)(hk + nq);
    for (int i = 0; i < nq; i++) {
        hk[i] = k[i];
        hkind[i] = router_kind(nodes, nnodes, qd[i].proot);
    }
    if (brute_upload(g, db, errbuf, errlen)) return -1;
    char *d = db.stage_d->as<char>();
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;
    const int P = db.P;
    RT_OK(s.popcnt.ensure((size_t)(P > 0 ? P : 1) * 8));
    if (P > 0) {
        RT_OK(s.bitmaps.ensure((size_t)P * bm_words * 4));
        g->launches++;
        RT_OK(launch_bitmaps(g->d_cols, g->count, (const PredInsn *)(d + db.off_insns),
                             (const PredProg *)(d + db.off_progs),
                             (const double *)(d + db.off_consts), P, s.bitmaps.as<uint32_t>(),
                             bm_words, s.popcnt.as<unsigned long long>(), g->sm_count, g->stream,
                             db.ninsns, db.nconsts, g->ncols, db.one_range));
    }
    const size_t fbytes = (size_t)nq * NI * 4;
    RT_OK(s.out_d.ensure(fbytes));
    g->launches++;
    RT_OK(launch_router_features(r, (const float *)(d + db.off_q), g->dpad, nq,
                                 s.popcnt.as<unsigned long long>(),
                                 (const int32_t *)(d + db.off_qprog), g->count,
                                 (const uint32_t *)(d + db.off_extra),
                                 (const int32_t *)(d + db.off_extra + (size_t)nq * 4),
                                 s.out_d.as<float>(), g->stream));
    RT_OK(cudaMemcpyAsync(feats, s.out_d.p, fbytes, cudaMemcpyDeviceToHost, g->stream));
    RT_OK(cudaStreamSynchronize(g->stream));
    return 0;
}

extern "C" int pv_router_forward(PvRouter *r, int n, const float *feats, float *logits,
                                 char *errbuf, size_t errlen) {
    if (!r || n < 1 || !feats || !logits) return -1;
    std::lock_guard<std::mutex> lk(r->mu);
    RT_OK(cudaSetDevice(r->device));
    const size_t fb = (size_t)n * NI * 4, zb = (size_t)n * NO * 4;
    RT_OK(r->io.ensure(fb + zb + 256));
    float *df = r->io.as<float>();
    float *dz = (float *)(r->io.as<char>() + ((fb + 255) & ~(size_t)255));
    RT_OK(cudaMemcpyAsync(df, feats, fb, cudaMemcpyHostToDevice, r->stream));
    RT_OK(launch_router_forward(r, df, n, dz, r->stream));
    RT_OK(cudaMemcpyAsync(logits, dz, zb, cudaMemcpyDeviceToHost, r->stream));
    RT_OK(cudaStreamSynchronize(r->stream));
    return 0;
}

namespace {

struct TrainBufs {
    float *Xn, *H1, *H2, *Z3, *dZ1, *dZ2, *dZ3, *loss;
    int *step, *off;
};

size_t train_bytes(int B, int epochs) {
    return (size_t)B * (NI + 4 * NH + 2 * NO) * 4 + (size_t)(epochs + 1) * 4 + 64 + 10 * 256;
}

TrainBufs carve_train(char *base, int B, int epochs) {
    TrainBufs t;
    size_t o = 0;
    auto c = [&](size_t n) { char *p = base + o; o += (n + 255) & ~(size_t)255; return p; };
    t.Xn = (float *)c((size_t)B * NI * 4);
    t.H1 = (float *)c((size_t)B * NH * 4);
    t.H2 = (float *)c((size_t)B * NH * 4);
    t.Z3 = (float *)c((size_t)B * NO * 4);
    t.dZ1 = (float *)c((size_t)B * NH * 4);
    t.dZ2 = (float *)c((size_t)B * NH * 4);
    t.dZ3 = (float *)c((size_t)B * NO * 4);
    t.loss = (float *)c((size_t)(epochs + 1) * 4);
    t.step = (int *)c(32);
    t.off = t.step + 1;
    return t;
}

// forward + loss + backward + weight gradient of one batch
cudaError_t one_batch(PvRouter *r, const TrainBufs &t, const float *X, const int32_t *lab,
                      const float *sw, const uint32_t *idx, const int *off, int B, float *loss,
                      cudaStream_t st) {
    const int g128 = (B + 127) / 128;
    mlp_forward_kernel<<<g128, 128, 0, st>>>(X, idx, off, B, r->mlp.w, r->mlp.norm, t.Xn, t.H1,
                                             t.H2, t.Z3);
    mlp_loss_kernel<<<(B + 255) / 256, 256, 0, st>>>(t.Z3, lab, sw, idx, off, B, t.dZ3, loss);
    mlp_backward_kernel<<<g128, 128, 0, st>>>(r->mlp.w, B, t.H1, t.H2, t.dZ3, t.dZ2, t.dZ1);
    mlp_wgrad_kernel<<<(P_N + 127) / 128, 128, 0, st>>>(B, t.Xn, t.H1, t.H2, t.dZ1, t.dZ2, t.dZ3,
                                                         r->mlp.grad);
    return cudaGetLastError();
}

}  // namespace

extern "C" int pv_router_grad(PvRouter *r, int n, const float *feats, const int32_t *labels,
                              const float *sample_w, float *grad, float *loss, char *errbuf,
                              size_t errlen) {
    if (!r || n < 1 || n > (1 << 20) || !feats || !labels || !grad) return -1;
    for (int i = 0; i < n; i++)
        if (labels[i] < 0 || labels[i] >= NO) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "router: label %d out of range", labels[i]);
            return -1;
        }
    std::lock_guard<std::mutex> lk(r->mu);
    RT_OK(cudaSetDevice(r->device));
    const size_t fb = ((size_t)n * NI * 4 + 255) & ~(size_t)255;
    const size_t lb = ((size_t)n * 4 + 255) & ~(size_t)255;
    RT_OK(r->io.ensure(fb + 2 * lb));
    char *io = r->io.as<char>();
    RT_OK(cudaMemcpyAsync(io, feats, (size_t)n * NI * 4, cudaMemcpyHostToDevice, r->stream));
    RT_OK(cudaMemcpyAsync(io + fb, labels, (size_t)n * 4, cudaMemcpyHostToDevice, r->stream));
    if (sample_w)
        RT_OK(cudaMemcpyAsync(io + fb + lb, sample_w, (size_t)n * 4, cudaMemcpyHostToDevice, r->stream));
    RT_OK(r->scratch.ensure(train_bytes(n, 0)));
    TrainBufs t = carve_train(r->scratch.as<char>(), n, 0);
    RT_OK(cudaMemsetAsync(t.loss, 0, 4, r->stream));
    RT_OK(one_batch(r, t, (const float *)io, (const int32_t *)(io + fb),
                    sample_w ? (const float *)(io + fb + lb) : nullptr, nullptr, nullptr, n,
                    t.loss, r->stream));
    RT_OK(cudaMemcpyAsync(grad, r->mlp.grad, (size_t)P_N * 4, cudaMemcpyDeviceToHost, r->stream));
    float l = 0.f;
    RT_OK(cudaMemcpyAsync(&l, t.loss, 4, cudaMemcpyDeviceToHost, r->stream));
    RT_OK(cudaStreamSynchronize(r->stream));
    if (loss) *loss = l;
    return 0;
}

extern "C" int pv_router_train(PvRouter *r, int n, const float *feats, const int32_t *labels,
                               const float *sample_w, int epochs, int batch, float lr,
                               uint64_t seed, float *epoch_loss, char *errbuf, size_t errlen) {
    if (!r || n < 1 || !feats || !labels || epochs < 1 || epochs > 100000 || batch < 1 ||
        batch > 65536 || batch > n || !(lr > 0.f)) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "router: bad training arguments");
        return -1;
    }
    for (int i = 0; i < n; i++)
        if (labels[i] < 0 || labels[i] >= NO) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "router: label %d out of range", labels[i]);
            return -1;
        }
    std::lock_guard<std::mutex> lk(r->mu);
    RT_OK(cudaSetDevice(r->device));
    const int spe = n / batch;  // steps per epoch (the remainder rotates in via shuffling)
    const size_t fb = ((size_t)n * NI * 4 + 255) & ~(size_t)255;
    const size_t lb = ((size_t)n * 4 + 255) & ~(size_t)255;
    RT_OK(r->io.ensure(fb + 3 * lb));
    char *io = r->io.as<char>();
    const float *dX = (const float *)io;
    const int32_t *dL = (const int32_t *)(io + fb);
    const float *dW = sample_w ? (const float *)(io + fb + lb) : nullptr;
    uint32_t *dperm = (uint32_t *)(io + fb + 2 * lb);
    RT_OK(cudaMemcpyAsync(io, feats, (size_t)n * NI * 4, cudaMemcpyHostToDevice, r->stream));
    RT_OK(cudaMemcpyAsync(io + fb, labels, (size_t)n * 4, cudaMemcpyHostToDevice, r->stream));
    if (sample_w)
        RT_OK(cudaMemcpyAsync(io + fb + lb, sample_w, (size_t)n * 4, cudaMemcpyHostToDevice, r->stream));
    RT_OK(r->scratch.ensure(train_bytes(batch, epochs)));
    TrainBufs t = carve_train(r->scratch.as<char>(), batch, epochs);
    RT_OK(cudaMemsetAsync(t.loss, 0, (size_t)(epochs + 1) * 4, r->stream));
    // step counter starts at -1 so the first mlp_step_kernel yields step 0, offset 0
    const int init[2] = {-1, 0};
    RT_OK(cudaMemcpyAsync(t.step, init, 8, cudaMemcpyHostToDevice, r->stream));
    RT_OK(cudaStreamSynchronize(r->stream));

    // one optimizer step as a CUDA graph: advance the step, forward,
    // loss, backward, weight gradient, Adam
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint32_t> perm(n);
    RT_OK(r->host.ensure((size_t)n * 4));
    uint32_t *hperm = r->host.as<uint32_t>();
    std::mt19937_64 rng(seed);
    for (int i = 0; i < n; i++) perm[i] = (uint32_t)i;
    cudaError_t err = cudaSuccess;
    for (int ep = 0; ep < epochs && err == cudaSuccess; ep++) {
        for (int i = n - 1; i > 0; i--) {
            const int j = (int)(rng() % (uint64_t)(i + 1));
            const uint32_t tmp = perm[i];
            perm[i] = perm[j];
            perm[j] = tmp;
        }
        memcpy(hperm, perm.data(), (size_t)n * 4);
        err = cudaMemcpyAsync(dperm, hperm, (size_t)n * 4, cudaMemcpyHostToDevice, r->stream);
        if (err != cudaSuccess) break;
        float *lacc = t.loss + ep;
        // the graph is rebuilt per epoch so that the loss accumulator moves
        if (exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        if (graph) {
            cudaGraphDestroy(graph);
            graph = nullptr;
        }
        err = cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal);
        if (err != cudaSuccess) break;
        mlp_step_kernel<<<1, 1, 0, r->stream>>>(t.step, t.off, batch, spe);
        one_batch(r, t, dX, dL, dW, dperm, t.off, batch, lacc, r->stream);
        mlp_adam_kernel<<<(P_N + 255) / 256, 256, 0, r->stream>>>(r->mlp.master, r->mlp.w,
                                                                  r->mlp.grad, r->mlp.m,
                                                                  r->mlp.v, t.step, lr);
        err = cudaStreamEndCapture(r->stream, &graph);
        if (err != cudaSuccess) break;
        err = cudaGraphInstantiate(&exec, graph, 0);
        if (err != cudaSuccess) break;
        for (int s = 0; s < spe && err == cudaSuccess; s++) err = cudaGraphLaunch(exec, r->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(r->stream);  // hperm is reused
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    RT_OK(err);
    std::vector<float> lh(epochs);
    RT_OK(cudaMemcpyAsync(lh.data(), t.loss, (size_t)epochs * 4, cudaMemcpyDeviceToHost,
                          r->stream));
    RT_OK(cudaStreamSynchronize(r->stream));
    // each step added its batch mean: report the epoch mean
    if (epoch_loss)
        for (int e = 0; e < epochs; e++) epoch_loss[e] = lh[e] / (float)spe;
    return 0;
}

// ------------------------------------------------------------ routed batch
namespace pv {

// Action per query from the MLP logits (or from a caller's plan): the most
// probable action, except that a graph action whose probability does not
// exceed the scan's by `margin` yields to the scan. Writes the beam width
// (0 = scan), never below k.
__global__ void router_decide_kernel(const float *__restrict__ Z3, int nq,
                                     const uint32_t *__restrict__ kq,
                                     const uint16_t *__restrict__ plan, float margin,
                                     uint16_t *__restrict__ efq) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int k = (int)kq[q];
    int ef;
    if (plan) {
        ef = plan[q];
    } else {
        float z[NO], mx = -INFINITY;
#pragma unroll
        for (int o = 0; o < NO; o++) {
            z[o] = Z3[(uint64_t)q * NO + o];
            mx = fmaxf(mx, z[o]);
        }
        int a = 0;
#pragma unroll
        for (int o = 1; o < NO; o++)
            if (z[o] > z[a]) a = o;
        // p_a < p_0 + margin  <=>  e^{z_a} - e^{z_0} < margin * sum e^z
        float se = 0.f;
#pragma unroll
        for (int o = 0; o < NO; o++) se += expf(z[o] - mx);
        if (a > 0 && expf(z[a] - mx) - expf(z[0] - mx) < margin * se) a = 0;
        const int efs[NO] = {0, 32, 64, 128, 256};
        ef = efs[a];
    }
    if (ef > 0 && ef < k) ef = k;
    if (ef > FV_GPU_MAX_EF) ef = 0;  // beyond the graph's result capacity: scan
    efq[q] = (uint16_t)ef;
}

// The routing decision of a batch in two short launches, for the routed
// batch call (the first beside the bitmaps, the second beside the start of
// the search). Same features, network and
// decision rule as router_features_kernel -> mlp_infer_kernel ->
// router_decide_kernel (the centroid distances summed in the same order,
// so the features are the same values).
//
// Step 1: squared distances of every (query, centroid) pair, dist[q][c],
// summed over the dimensions in order, four at a time - the order of
// router_features_kernel, so the features equal the training ones. A CTA
// takes a tile of 64 queries x 32 centroids through shared memory (rows
// padded by one word: the 32 centroid rows a warp reads fall in 32
// banks), 64 dimensions at a time; each thread owns 4 queries x 2
// centroids.
constexpr int RT_TQ = 64, RT_TC = 32, RT_TD = 64;

__global__ void __launch_bounds__(256) router_cent_kernel(const float *__restrict__ queries,
                                                          int nq, int dpad,
                                                          const float *__restrict__ cent,
                                                          int ncent, float *__restrict__ dist) {
    __shared__ float sq[RT_TQ][RT_TD + 1];
    __shared__ float sc[RT_TC][RT_TD + 1];
    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * RT_TC, q0 = blockIdx.y * RT_TQ;
    const int tq = (tid >> 4) * 4, tc = (tid & 15) * 2;
    float acc[4][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
    for (int d0 = 0; d0 < dpad; d0 += RT_TD) {
        const int dn = min(RT_TD, dpad - d0);
        __syncthreads();
        for (int i = tid; i < RT_TQ * RT_TD; i += 256) {
            const int r = i / RT_TD, j = i - r * RT_TD;
            sq[r][j] = (q0 + r < nq && j < dn) ? queries[(uint64_t)(q0 + r) * dpad + d0 + j] : 0.f;
        }
        for (int i = tid; i < RT_TC * RT_TD; i += 256) {
            const int r = i / RT_TD, j = i - r * RT_TD;
            sc[r][j] = (c0 + r < ncent && j < dn) ? cent[(uint64_t)(c0 + r) * dpad + d0 + j] : 0.f;
        }
        __syncthreads();
        for (int j = 0; j < dn; j++) {
            const float x0 = sc[tc][j], x1 = sc[tc + 1][j];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float u = sq[tq + k][j];
                const float e0 = x0 - u, e1 = x1 - u;
                acc[k][0] = fmaf(e0, e0, acc[k][0]);
                acc[k][1] = fmaf(e1, e1, acc[k][1]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
        for (int m = 0; m < 2; m++)
            if (q0 + tq + k < nq && c0 + tc + m < ncent)
                dist[(uint64_t)(q0 + tq + k) * ncent + c0 + tc + m] = acc[k][m];
}

// Step 2: one warp per query: the 8 smallest centroid distances, the
// features, the network and the decision.
__global__ void __launch_bounds__(256) router_route_kernel(
    const float *__restrict__ queries, int dpad, const float *__restrict__ dist,
    int ncent, const unsigned long long *__restrict__ popcnt, const int32_t *__restrict__ qprog,
    uint64_t nrows, const uint32_t *__restrict__ kq, const int32_t *__restrict__ kind,
    const __nv_bfloat16 *__restrict__ w, const float *__restrict__ norm, float margin, int nq,
    float *__restrict__ feats, float *__restrict__ Z3, uint16_t *__restrict__ efq) {
    const int lane = threadIdx.x & 31;
    const int q = (int)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5);
    if (q >= nq) return;
    const float *qv = queries + (uint64_t)q * dpad;
    // the 8 smallest of the query's centroid distances: each lane's sorted
    // top-8 of its strided share, then 8 rounds of warp-wide minimum
    float mine = INFINITY;
    {
        float top[8];
#pragma unroll
        for (int i = 0; i < 8; i++) top[i] = INFINITY;
        const float *dq = dist + (uint64_t)q * ncent;
        for (int c = lane; c < ncent; c += 32) {
            float v = dq[c];
            if (!(v < top[7])) continue;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const float t = top[i];
                const bool sw = v < t;
                top[i] = sw ? v : t;
                v = sw ? t : v;
            }
        }
        int head = 0;
        for (int r = 0; r < 8; r++) {
            float best = head < 8 ? pick8(top, head) : INFINITY;
            int who = lane;
            warp_argmin(best, who);
            if (lane == who) head++;
            if (lane == r) mine = best;
        }
    }
    // |q|
    float s = 0.f;
    for (int j = lane; j < dpad; j += 32) s = fmaf(qv[j], qv[j], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const float qnorm = sqrtf(s);
    // features: lane i holds feature i
    float f = 0.f;
    const float m2 = __shfl_sync(0xffffffffu, mine, (lane + 30) & 31);  // lane - 2
    if (lane >= 2 && lane < 10) f = sqrtf(m2);
    if (lane == 0) {
        const int pg = qprog[q];
        const double sel = pg < 0 ? 1.0 : (double)popcnt[pg] / (double)nrows;
        f = (float)log10(sel > 1e-6 ? sel : 1e-6);
    }
    if (lane == 1) f = qnorm;
    if (lane == 10) f = log2f((float)(kq[q] > 0 ? kq[q] : 1));
    if (lane == 11) f = (float)kind[q];
    if (feats && lane < NI) feats[(uint64_t)q * NI + lane] = f;
    // MLP (as mlp_infer_kernel): lanes over the hidden units
    const float xi = lane < NI ? (f - __ldg(norm + lane)) / __ldg(norm + NI + lane) : 0.f;
    float h0 = __bfloat162float(w[P_B1 + lane]), h1 = __bfloat162float(w[P_B1 + lane + 32]);
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const float xb = __shfl_sync(0xffffffffu, xi, i);
        h0 = fmaf(xb, __bfloat162float(w[P_W1 + i * NH + lane]), h0);
        h1 = fmaf(xb, __bfloat162float(w[P_W1 + i * NH + lane + 32]), h1);
    }
    h0 = fmaxf(h0, 0.f);
    h1 = fmaxf(h1, 0.f);
    float g0 = __bfloat162float(w[P_B2 + lane]), g1 = __bfloat162float(w[P_B2 + lane + 32]);
#pragma unroll 8
    for (int i = 0; i < NH; i++) {
        const float hb = __shfl_sync(0xffffffffu, i < 32 ? h0 : h1, i & 31);
        g0 = fmaf(hb, __bfloat162float(w[P_W2 + i * NH + lane]), g0);
        g1 = fmaf(hb, __bfloat162float(w[P_W2 + i * NH + lane + 32]), g1);
    }
    g0 = fmaxf(g0, 0.f);
    g1 = fmaxf(g1, 0.f);
    float z[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) {
        float p = g0 * __bfloat162float(w[P_W3 + lane * NO + o]);
        p = fmaf(g1, __bfloat162float(w[P_W3 + (lane + 32) * NO + o]), p);
#pragma unroll
        for (int x = 16; x; x >>= 1) p += __shfl_xor_sync(0xffffffffu, p, x);
        z[o] = p + __bfloat162float(w[P_B3 + o]);
    }
    if (lane == 0) {
        // the decision rule of router_decide_kernel
        float mx = -INFINITY;
#pragma unroll
        for (int o = 0; o < NO; o++) {
            if (Z3) Z3[(uint64_t)q * NO + o] = z[o];
            mx = fmaxf(mx, z[o]);
        }
        int a = 0;
#pragma unroll
        for (int o = 1; o < NO; o++)
            if (z[o] > z[a]) a = o;
        float se = 0.f;
#pragma unroll
        for (int o = 0; o < NO; o++) se += expf(z[o] - mx);
        if (a > 0 && expf(z[a] - mx) - expf(z[0] - mx) < margin * se) a = 0;
        const int efs[NO] = {0, 32, 64, 128, 256};
        int ef = efs[a];
        const int k = (int)kq[q];
        if (ef > 0 && ef < k) ef = k;
        if (ef > FV_GPU_MAX_EF) ef = 0;
        efq[q] = (uint16_t)ef;
    }
}

}  // namespace pv

extern "C" int pv_routed_batch(FvGpuIndex *g, PvRouter *r, int nq, const float *queries,
                               const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes, int nnodes,
                               const int32_t *children, int nchildren, const double *invals,
                               int ninvals, const uint32_t *k, uint32_t topb,
                               const uint16_t *plan, float margin, int split, FvHit *out,
                               uint32_t *out_cnt, uint16_t *decided, int *executed,
                               float *stage_ms, char *errbuf, size_t errlen) {
    if (!g || nq < 1 || nq > FV_GPU_MAX_BATCH || !queries || !qd || !k || !out || !out_cnt ||
        topb < 1 || topb > FV_GPU_MAX_TOPB || (!r && !plan)) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "routed: bad arguments");
        return -1;
    }
    for (int i = 0; i < nq; i++)
        if (k[i] < 1 || k[i] > topb) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "routed: k[%d]=%u outside 1..topb", i, k[i]);
            return -1;
        }
    if (r && (g->dim != r->dim || g->device != r->device)) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "routed: router/index mismatch");
        return -1;
    }
    const bool have_graph = g->d_adj != nullptr && g->count < (1ull << 31);
    if (have_graph)
        for (int i = 0; i < nq; i++)
            if (qd[i].entry >= g->count) {
                if (errbuf && errlen) snprintf(errbuf, errlen, "routed: query %d entry out of range", i);
                return -1;
            }
    std::lock_guard<std::mutex> lk(g->mu);
    std::unique_lock<std::mutex> lr;
    if (r) lr = std::unique_lock<std::mutex>(r->mu);
    RT_OK(cudaSetDevice(g->device));
    g->launches = 0;
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return -1;
    // staged extras: k, kind, entries (u32 each), plan (u16)
    DevBatch db;
    db.stage_h = &g->scan.stage_h;
    db.stage_d = &g->scan.stage_d;
    const size_t n4 = ((size_t)nq * 4 + 15) & ~(size_t)15;
    if (brute_prepare(g, nq, queries, pb, db, 3 * n4 + (size_t)nq * 2 + 16, errbuf, errlen))
        return -1;
    char *hx = db.stage_h->as<char>() + db.off_extra;
    uint32_t *hk = (uint32_t *)hx;
    int32_t *hkind = (int32_t *)(hx + n4);
    uint32_t *hent = (uint32_t *)(hx + 2 * n4);
    uint16_t *hplan = (uint16_t *)(hx + 3 * n4);
    for (int i = 0; i < nq; i++) {
        hk[i] = k[i];
        hkind[i] = router_kind(nodes, nnodes, qd[i].proot);
        hent[i] = qd[i].entry;
        hplan[i] = plan ? plan[i] : 0;
    }
    if (brute_upload(g, db, errbuf, errlen)) return -1;
    char *d = db.stage_d->as<char>();
    const char *dx = d + db.off_extra;
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;
    const int P = db.P;
    cudaEvent_t *ev = g->rev;
    for (int i = 0; i < 6; i++)
        if (!ev[i]) RT_OK(cudaEventCreate(&ev[i]));
    cudaStream_t side = g->stream2;
    // size every buffer first: an allocation later would wait for the work
    // already queued on both streams
    const size_t hit_bytes = (size_t)nq * topb * sizeof(FvHit);
    const size_t off_cnt = (hit_bytes + 255) & ~(size_t)255;
    const size_t off_tr = off_cnt + (((size_t)nq * 4 + 255) & ~(size_t)255);
    const size_t obytes = off_tr + (size_t)nq + 256;
    const size_t fb = ((size_t)nq * NI * 4 + 255) & ~(size_t)255;
    const size_t zb = ((size_t)nq * NO * 4 + 255) & ~(size_t)255;
    const size_t eb = ((size_t)nq * 2 + 255) & ~(size_t)255;
    const size_t pb8 = plan ? 0 : (size_t)nq * r->ncent * 4;  // centroid distances
    const size_t gbytes = have_graph ? graph_out_layout(nq, FV_GPU_MAX_EF).bytes : 0;
    RT_OK(s.out_d.ensure(obytes));
    RT_OK(s.out_h.ensure(obytes));
    RT_OK(g->graph.route.ensure(fb + zb + eb + pb8));
    RT_OK(g->graph.route_h.ensure(eb + gbytes));
    if (have_graph) RT_OK(g->graph.gout.ensure(gbytes));
    float *dfeat = g->graph.route.as<float>();
    float *dz = (float *)(g->graph.route.as<char>() + fb);
    uint16_t *defq = (uint16_t *)(g->graph.route.as<char>() + fb + zb);
    float *dpart = (float *)(g->graph.route.as<char>() + fb + zb + eb);
    uint16_t *hefq = g->graph.route_h.as<uint16_t>();
    if (!plan && g->dpad != r->dpad) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "routed: router dimension mismatch");
        return -1;
    }
    RT_OK(s.popcnt.ensure((size_t)(P > 0 ? P : 1) * 8));
    if (P > 0) RT_OK(s.bitmaps.ensure((size_t)P * bm_words * 4));
    RT_OK(cudaEventRecord(ev[0], g->stream));
    // Routing on the side stream, beside the bitmaps and then the search:
    // the centroid distances need only the queries (they run while the
    // bitmaps are built), the features, network and decision need the
    // bitmaps' counts (a few warps per query); the decisions are read back
    // into pinned memory while the search runs. (One CTA per query that
    // held its SM through the scan took issue slots from the scan's
    // epilogue; on the search stream, in series, it added its latency.)
    RT_OK(cudaStreamWaitEvent(side, ev[0], 0));
    g->launches += plan ? 1 : 2;
    if (!plan)
        router_cent_kernel<<<dim3((r->ncent + RT_TC - 1) / RT_TC, (nq + RT_TQ - 1) / RT_TQ), 256, 0,
                             side>>>((const float *)(d + db.off_q), nq, g->dpad, r->d_cent,
                                     r->ncent, dpart);
    if (P > 0) {
        g->launches++;
        RT_OK(launch_bitmaps(g->d_cols, g->count, (const PredInsn *)(d + db.off_insns),
                             (const PredProg *)(d + db.off_progs),
                             (const double *)(d + db.off_consts), P, s.bitmaps.as<uint32_t>(),
                             bm_words, s.popcnt.as<unsigned long long>(), g->sm_count, g->stream,
                             db.ninsns, db.nconsts, g->ncols, db.one_range));
    }
    // Speculative scan on the main stream meanwhile: a scan costs about the
    // same for one query as for the batch and is exact, so it runs unless
    // a caller's plan sends every query to the graph; the router's answer
    // only decides whether its results are replaced by the graph search's.
    bool plan_all_graph = plan != nullptr && have_graph;
    for (int i = 0; plan_all_graph && i < nq; i++) plan_all_graph = plan[i] > 0;
    const bool spec = !plan_all_graph;
    if (spec) {
        char *od = s.out_d.as<char>();
        const int mode = g->precision != FV_GPU_PREC_FP32 ? PV_MODE_LOW : PV_MODE_EXACT;
        // ev[1]: the bitmaps are complete (behind query prep, which the
        // tensor-core scan runs beside them); the routing waits for it
        if (brute_launch(g, db, topb, mode, (FvHit *)od, (uint32_t *)(od + off_cnt),
                         (uint8_t *)(od + off_tr), errbuf, errlen, nullptr, true, ev[1]))
            return -1;
        RT_OK(cudaEventRecord(ev[3], g->stream));
        RT_OK(cudaMemcpyAsync(s.out_h.p, od, obytes, cudaMemcpyDeviceToHost, g->stream));
        // the watchdog word rides behind the results (the spare tail of out_h)
        tc_watchdog_enqueue(g, (int *)(s.out_h.as<char>() + obytes - 64));
    } else {
        RT_OK(cudaEventRecord(ev[1], g->stream));
    }
    RT_OK(cudaStreamWaitEvent(side, ev[1], 0));
    if (!plan) {
        router_route_kernel<<<(nq + 7) / 8, 256, 0, side>>>(
            (const float *)(d + db.off_q), g->dpad, dpart, r->ncent,
            s.popcnt.as<unsigned long long>(), (const int32_t *)(d + db.off_qprog), g->count,
            (const uint32_t *)dx, (const int32_t *)(dx + n4), r->mlp.w, r->mlp.norm, margin, nq,
            dfeat, dz, defq);
    } else {
        router_decide_kernel<<<(nq + 127) / 128, 128, 0, side>>>(
            dz, nq, (const uint32_t *)dx, (const uint16_t *)(dx + 3 * n4), margin, defq);
    }
    RT_OK(cudaGetLastError());
    RT_OK(cudaEventRecord(ev[5], side));
    RT_OK(cudaMemcpyAsync(hefq, defq, (size_t)nq * 2, cudaMemcpyDeviceToHost, side));
    RT_OK(cudaEventRecord(ev[2], side));
    RT_OK(cudaEventSynchronize(ev[2]));
    // each query takes the route the router chose for it: the graph search
    // at its beam width (graph-routed queries, when the index has a graph)
    // or the scan; a batch whose every query went to the graph discards
    // the speculative scan
    int ngraph = 0;
    uint32_t efmax = 0;
    for (int i = 0; i < nq; i++) {
        if (!have_graph) hefq[i] = 0;
        if (hefq[i] > 0) ngraph++;
        efmax = hefq[i] > efmax ? hefq[i] : efmax;
    }
    const bool all_graph = have_graph && ngraph == nq;
    if (decided) memcpy(decided, hefq, (size_t)nq * 2);
    if (!split && !all_graph && spec) {
        // a batch that is scanned anyway answers every query from the scan
        // (exact, and already paid for); graph-routed queries in it would
        // only add the graph's time
        for (int i = 0; i < nq; i++) hefq[i] = 0;
        ngraph = 0;
    }
    if (executed) *executed = ngraph == 0 ? 0 : all_graph ? 1 : 2;
    if (!spec && !all_graph) {  // a plan sent every query to a graph the index lacks
        if (errbuf && errlen) snprintf(errbuf, errlen, "routed: no graph for the plan");
        return -1;
    }
    cudaEvent_t done = ev[3];
    const char *goh = nullptr;
    GraphOut glo{};
    if (ngraph > 0) {
        glo = graph_out_layout(nq, efmax);
        char *oh = g->graph.route_h.as<char>() + eb;
        char *od = g->graph.gout.as<char>();
        const uint64_t mv = (uint64_t)efmax * 400 > 200000 ? (uint64_t)efmax * 400 : 200000;
        if (graph_launch(g, nq, (const float *)(d + db.off_q), (const uint32_t *)(dx + 2 * n4),
                         (const int32_t *)(d + db.off_qprog), defq, efmax, mv, od, glo, errbuf,
                         errlen, side))
            return -1;
        RT_OK(cudaEventRecord(ev[4], side));
        RT_OK(cudaMemcpyAsync(oh, od, glo.bytes, cudaMemcpyDeviceToHost, side));
        RT_OK(cudaStreamSynchronize(side));
        goh = oh;
        g->graph_stats.resize((size_t)nq * 4);
        memcpy(g->graph_stats.data(), oh + glo.off_st, (size_t)nq * 16);
    }
    RT_OK(cudaStreamSynchronize(g->stream));  // the scan, if any
    if (spec && check_tc_watchdog(g, errbuf, errlen)) return -1;
    const char *soh = s.out_h.as<char>();
    const uint32_t *scnt = (const uint32_t *)(soh + off_cnt);
    const uint32_t *gcnt = goh ? (const uint32_t *)(goh + glo.off_cnt) : nullptr;
    for (int q = 0; q < nq; q++) {
        if (hefq[q] > 0) {
            const uint32_t c = gcnt[q] < k[q] ? gcnt[q] : k[q];
            memcpy(out + (size_t)q * topb, goh + (size_t)q * efmax * sizeof(FvHit),
                   c * sizeof(FvHit));
            out_cnt[q] = c;
        } else {
            const uint32_t c = scnt[q] < k[q] ? scnt[q] : k[q];
            memcpy(out + (size_t)q * topb, soh + (size_t)q * topb * sizeof(FvHit),
                   c * sizeof(FvHit));
            out_cnt[q] = c;
        }
    }
    if (spec && g->tc_unc && ngraph < nq) {
        // scan-routed queries whose reduced-precision superset the merge
        // could not certify are re-run exactly
        std::vector<uint8_t> unc(nq), tr(nq);
        RT_OK(cudaMemcpyAsync(unc.data(), g->tc_unc, (size_t)nq, cudaMemcpyDeviceToHost,
                              g->stream));
        RT_OK(cudaStreamSynchronize(g->stream));
        for (int q = 0; q < nq; q++)
            if (hefq[q] > 0) unc[q] = 0;
        if (redo_flagged(g, nq, queries, pb, topb, unc.data(), out, out_cnt, tr.data(), errbuf,
                         errlen))
            return -1;
        for (int q = 0; q < nq; q++)
            if (out_cnt[q] > k[q]) out_cnt[q] = k[q];
    }
    g->tc_unc = nullptr;
    if (ngraph > 0) done = ev[4];
    // device time of the batch: the bitmaps, then the search with the
    // routing's tail beside it (t[1]: the routing after the bitmaps; the
    // batch took t[0] + t[2])
    float t[3] = {0, 0, 0}, tot = 0.f;
    cudaEventElapsedTime(&t[0], ev[0], ev[1]);
    cudaEventElapsedTime(&t[1], ev[1], ev[5]);
    cudaEventElapsedTime(&tot, ev[0], done);
    if (ngraph > 0 && spec) {
        float a = 0.f;  // the scan may finish last
        cudaEventElapsedTime(&a, ev[0], ev[3]);
        if (a > tot) tot = a;
    }
    t[2] = tot - t[0];
    if (stage_ms) memcpy(stage_ms, t, sizeof(t));
    g->last_kernel_ms = tot;
    return 0;
}
