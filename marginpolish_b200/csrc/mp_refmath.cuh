// Device arithmetic of the reference's log-space pair HMM, shared by the kernels that reproduce
// its numbers bit for bit (the bubble scorer in mp_bubble.cu, the overlap posteriors in
// mp_refpost.cu): the approximate log-sum of impl/pairwiseAligner.c:279-299 and the term
// f + (e + t) of doTransitionForward / doTransitionBackward (:311-324), every operation rounded
// alone (__dadd_rn / __dmul_rn) so that no fused multiply-add changes a bit.
#pragma once

#include "mp_internal.h"

#include <cmath>
#include <cstdint>

namespace {

using mp::DevLogModel;

constexpr double kLogZero = -INFINITY;

// The cubic of impl/pairwiseAligner.c:282-293, piece by piece: (c3, c2), (c1, c0) for d <= 1,
// d <= 2.5, d <= 4.5 and beyond, the coefficients as the reference writes them (single-precision
// literals, widened to double).
__constant__ double2 kCubic[8] = {
    {(double) -0.009350833524763f, (double) 0.130659527668286f}, {(double) 0.498799810682272f, (double) 0.693203116424741f},
    {(double) -0.014532321752540f, (double) 0.139942324101744f}, {(double) 0.495635523139337f, (double) 0.692140569840976f},
    {(double) -0.004605031767994f, (double) 0.063427417320019f}, {(double) 0.695956496475118f, (double) 0.514272634594009f},
    {(double) -0.000458661602210f, (double) 0.009695946122598f}, {(double) 0.930734667215156f, (double) 0.168037164329057f},
};

// What a block keeps in shared memory: the cubic and both strands' models.
struct Tables {
    double2 cubic[8];
    DevLogModel models[2];
};

__device__ __forceinline__ void loadTables(Tables &T, const DevLogModel *models) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(models);
    uint32_t *dst = reinterpret_cast<uint32_t *>(T.models);
    for (int i = threadIdx.x; i < (int) (2 * sizeof(DevLogModel) / 4); i += blockDim.x) dst[i] = src[i];
    if (threadIdx.x < 8) T.cubic[threadIdx.x] = kCubic[threadIdx.x];
    __syncthreads();
}

// lookup() for 0 <= d < 7.5: the piece picked by comparisons (the reference's if-chain), its
// coefficients read from the table, every operation rounded alone.
__device__ __forceinline__ double lookupCubic(const Tables &T, double d) {
    const int piece = (d > (double) 1.00f) + (d > (double) 2.50f) + (d > (double) 4.50f);
    const double2 hi = T.cubic[2 * piece], lo = T.cubic[2 * piece + 1];
    double v = __dmul_rn(hi.x, d);
    v = __dadd_rn(v, hi.y);
    v = __dmul_rn(v, d);
    v = __dadd_rn(v, lo.x);
    v = __dmul_rn(v, d);
    return __dadd_rn(v, lo.y);
}

// logAdd of impl/pairwiseAligner.c:295-299 without branches: a is the term the reference keeps
// (y when x < y, else x), b the other; both of its branches compute lookup(a - b) + b.
__device__ __forceinline__ double logAdd(const Tables &T, double x, double y) {
    const bool lt = x < y;
    const double a = lt ? y : x, b = lt ? x : y;
    const double d = __dsub_rn(a, b);
    const double r = __dadd_rn(lookupCubic(T, d), b);
    return (b == kLogZero || d >= 7.5) ? a : r;
}

// f + (e + t): the term doTransitionForward adds (impl/pairwiseAligner.c:311-314).
__device__ __forceinline__ double term(double f, double e, double t) {
    return __dadd_rn(f, __dadd_rn(e, t));
}

__device__ __forceinline__ int baseOf(uint16_t s, int runLength) {
    const int b = runLength ? (s & 255) : s;
    return b >= 4 ? 4 : b;
}

}  // namespace
