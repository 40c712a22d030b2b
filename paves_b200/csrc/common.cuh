// common.cuh — shared definitions for the paves_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "paves_gpu.h"

namespace pv {

// Result keys pack (distance bits << 32 | row). For non-negative IEEE floats
// the bit pattern orders like the value, so unsigned key order equals the
// (dist, node) lexicographic order the reference sorts by
// (engine.cpp:1114-1116, gpu_engine.cu:583-584). NaN distances sort last.
__host__ __device__ inline uint64_t make_key(float d, uint32_t row) {
#ifdef __CUDA_ARCH__
    return ((uint64_t)__float_as_uint(d) << 32) | row;
#else
    uint32_t b;
    memcpy(&b, &d, 4);
    return ((uint64_t)b << 32) | row;
#endif
}
__host__ __device__ inline uint32_t key_row(uint64_t k) { return (uint32_t)k; }
__host__ __device__ inline float key_dist(uint64_t k) {
#ifdef __CUDA_ARCH__
    return __uint_as_float((uint32_t)(k >> 32));
#else
    uint32_t b = (uint32_t)(k >> 32);
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}
constexpr uint64_t KEY_MAX = ~0ull;

// Predicate program instruction: the per-query predicate tree re-serialized
// in post-order (children before parents) so a thread evaluates it with a
// bit stack, no recursion. Semantics follow FvPred::eval_node
// (engine.cpp:397-431): NaN compares false, NE is (v == v && v != c).
struct PredInsn {
    int32_t kind;    // FV_NODE_*
    int32_t col;     // CMP / IN
    int32_t op;      // CMP
    int32_t n;       // IN: number of values; AND/OR/NOT: number of children
    int32_t val0;    // IN: first value in the constant pool
    int32_t pad;
    double value;    // CMP constant
};
static_assert(sizeof(PredInsn) == 32, "PredInsn layout");

// Range form of a program (a single instruction of kind PV_NODE_RANGE):
// the AND of n per-column terms whose encodings sit in the constant pool
// from val0 on. An interval term is 3 doubles {meta, lo, hi}: lo <= v and
// v <= hi (open bounds were turned into closed ones on the host); an
// IN-set term over small integers is 2 doubles {meta, mask bits}: v is an
// integer b in [0, 64) with bit b of the mask set. meta = col | kind << 16.
// Both tests are the f64 comparisons of the nodes they replace (NaN fails
// every comparison), so results are identical.
constexpr int PV_NODE_RANGE = 16;
constexpr int PV_RANGE_MAX_TERMS = 4;
constexpr int PV_TERM_MASK = 1 << 16;

// One distinct predicate of a batch: instructions [insn0, insn0+ninsn).
struct PredProg {
    int32_t insn0;
    int32_t ninsn;
};

}  // namespace pv

#define PV_CUDA_OK(call, errbuf, errlen)                                   \
    do {                                                                   \
        cudaError_t e__ = (call);                                          \
        if (e__ != cudaSuccess) {                                          \
            if (errbuf && errlen)                                          \
                snprintf(errbuf, errlen, "gpu: %s failed: %s", #call,     \
                         cudaGetErrorString(e__));                         \
            return -1;                                                     \
        }                                                                  \
    } while (0)
