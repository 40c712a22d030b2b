// topk.cuh — block-level top-K maintenance shared by the scan kernels.
//
// Each CTA keeps, per query of its tile, one shared-memory region of S keys
// (S a power of two >= K + CB):
//   [0, K)      the CTA's current top-K keys, ascending, padded with KEY_MAX
//   [K, K+CB)   an append buffer of admitted candidates
//   [K+CB, S)   KEY_MAX padding
// A candidate is admitted when its key is below the query's threshold
// (min of the CTA's own K-th key and the grid-wide bound in global memory)
// and its predicate bit is set. When a buffer may overflow in the next step
// the whole region is sorted by a bitonic network and cut back to K.
// Keys are unique (row ids are), so the result is the canonical
// (dist, id)-ordered top-K.
#pragma once
#include "common.cuh"

namespace pv {

struct TopkSmem {
    uint64_t *region;        // [QT][S]
    int *nb;                 // [QT] buffer fill
    int *nt;                 // [QT] valid keys in [0, K)
    unsigned long long *tau; // [QT] admission threshold
    int *flush_list;         // [QT + 1]: [0] = count, then query slots
};

// Bitonic sort of the regions of the queries in flush_list, block-wide.
// All threads of the block must call it.
__device__ __forceinline__ void topk_flush(TopkSmem &t, int S, int K, int CB,
                                           int qt0, int nq,
                                           unsigned long long *__restrict__ g_tau) {
    const int nfl = t.flush_list[0];
    if (nfl == 0) return;
    // sort only the prefix that holds keys: [0, K) kept keys (KEY_MAX
    // padded) and [K, K + nb) appended ones; everything past is KEY_MAX
    int used = 0;
    for (int f = 0; f < nfl; f++) {
        const int nb = t.nb[t.flush_list[1 + f]];
        if (nb > used) used = nb;
    }
    int n2 = 2;
    while (n2 < K + used) n2 <<= 1;
    if (n2 > S) n2 = S;
    const int half = n2 >> 1;
    const int items = nfl * half;
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int it = threadIdx.x; it < items; it += blockDim.x) {
                const int f = it / half;
                const int i = it - f * half;
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo | j;
                uint64_t *r = t.region + (size_t)t.flush_list[1 + f] * S;
                const uint64_t a = r[lo], b = r[hi];
                const bool up = (lo & k) == 0;
                if ((a > b) == up) {
                    r[lo] = b;
                    r[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    // cut back to K, clear the buffer area, update thresholds
    const int tail = n2 > K ? n2 - K : 0;  // slots past the sorted prefix stay KEY_MAX
    for (int it = threadIdx.x; it < nfl * tail; it += blockDim.x) {
        const int f = it / tail;
        const int i = K + (it - f * tail);
        t.region[(size_t)t.flush_list[1 + f] * S + i] = KEY_MAX;
    }
    if (threadIdx.x < nfl) {
        const int qq = t.flush_list[1 + threadIdx.x];
        int n = t.nt[qq] + t.nb[qq];
        if (n > K) n = K;
        t.nt[qq] = n;
        t.nb[qq] = 0;
        if (n == K) {
            const unsigned long long kth = t.region[(size_t)qq * S + K - 1];
            if (kth < t.tau[qq]) t.tau[qq] = kth;
            const int qg = qt0 + qq;
            if (qg < nq) atomicMin(g_tau + qg, kth);
        }
    }
    __syncthreads();
}

}  // namespace pv
