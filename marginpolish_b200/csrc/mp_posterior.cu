// Posterior kernel of the realignment engine (sm_100a).
//
// Hot path: the anchored, banded 3-state pair-HMM forward / backward /
// posterior pass of MarginPolish (getPosteriorProbsWithBanding,
// impl/pairwiseAligner.c:687-808, over the split rectangles of :942-991; cell
// recurrence impl/stateMachine.c:559-581; posterior rules
// impl/pairwiseAligner.c:586-664), re-designed for warps that carry G = 32/L
// banded sub-problems ("tasks"), one per group of L lanes, persistent, fed
// from a length-sorted queue:
//
//  * The cells of anti-diagonal d of a task live in a window of S = L*C slots,
//    C consecutive slots per lane; slot i holds x-y = 2(Q+i) + (d&1). The
//    window origin Q moves only by whole lanes, when the 5-diagonal band hull
//    leaves it, so a diagonal step needs one shuffle per lane.
//  * The G tasks of a warp (neighbours in the length-sorted queue) run in
//    lockstep over anti-diagonals: the per-diagonal bookkeeping is issued once
//    for G tasks and every lane carries C independent cells. A group whose task
//    has ended is masked by predicates until the warp's longest task ends.
//  * FP32 probabilities (not logs), in push form: each cell sends its three
//    outgoing sums (to gap-x, gap-y and match successors); the receiving cell
//    multiplies by its emission. Emissions are zeroed outside the band, which
//    also masks every product built on them. Values are rescaled by exact
//    powers of two every K diagonals and the integer exponents are tracked per
//    block, so no log / exp is evaluated per cell; the FP64 log-likelihood is
//    ln(mantissa) + exponent*ln2 once per segment.
//  * The forward sweep stores one float4 per slot every K diagonals (the
//    checkpoint: outgoing gap sums of d-1 and match sums of d-1, d-2). The
//    forward values never depend on a traceback, so the reference's traceback
//    segments (intermediate points of impl/pairwiseAligner.c:722-737, then the
//    end) are all walked after the sweep, in the reference's order. A walk
//    recomputes each block of K diagonals into shared memory and runs the
//    backward recurrence and the posteriors over it, top block first,
//    prefetching the next block's checkpoint and band records into registers.
//  * Posterior tuples are ranked within the group (packed prefix sum) and
//    written from the top of the task's output region downwards: the region
//    then reads in the reference's order (ascending anti-diagonal, descending
//    x-y, later traceback segments first).
#include "mp_internal.h"

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <type_traits>

namespace mp {

#define FULL_MASK 0xffffffffu

// Dynamic shared memory of a posterior block. Fixed layout at the start:
//   [0, 200)    match emission tables, [model][x base][y base] (5 x 5 floats each)
//   [200, 240)  gap-x emissions [model][base]
//   [240, 280)  gap-y emissions [model][base]
//   [kRepBase)  run-length repeat tables, one per model (one when both strands share it)
// then the per-group workspaces. Table reads use byte offsets from the array start, so a
// lookup is one shared load with an immediate base.
extern __shared__ __align__(16) unsigned char mpSmem[];
constexpr uint32_t kMatchOff = 0, kGapXOff = 200, kGapYOff = 240, kRepBase = 384;

// Bytes of the table area (the per-group workspaces start 16-byte aligned after it).
__host__ __device__ constexpr size_t tableBytes(int nTables) {
    return ((size_t) kRepBase + (size_t) nTables * kRepTable * sizeof(float) + 15) & ~(size_t) 15;
}

__device__ __forceinline__ float ldsF(uint32_t off) {
    return *reinterpret_cast<const float *>(mpSmem + off);
}

// Shared-memory load / store at a byte offset from the start of the dynamic array.
template <typename T>
__device__ __forceinline__ T lds(uint32_t off) {
    return *reinterpret_cast<const T *>(mpSmem + off);
}

template <typename T>
__device__ __forceinline__ void sts(uint32_t off, const T &v) {
    *reinterpret_cast<T *>(mpSmem + off) = v;
}

template <int S>
struct RingSize {
    static constexpr int R = (S + 64 <= 128) ? 128 : ((S + 64 <= 256) ? 256 : 512);
};

__device__ __forceinline__ float pow2f(int k) {  // 2^k, k in [-126, 127]
    return __int_as_float((127 + k) << 23);
}

__device__ __forceinline__ int exponentOf(float m) {  // floor(log2 m) for normal m
    return ((__float_as_int(m) >> 23) & 0xff) - 127;
}

// Arithmetic of the scaled probabilities: FP32 for the production kernels, FP64 for the
// sub-problems whose dynamic range FP32 cannot hold (wide bands of weakly related
// sequences, detected by the total-probability check) and for the likelihood-only mode.
template <class V>
struct Num;

template <>
struct Num<float> {
    using V4 = float4;
    using V2 = float2;
    static constexpr int kMinExp = -126, kMaxExp = 127;
    __device__ static __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    __device__ static __forceinline__ float mx(float a, float b) { return fmaxf(a, b); }
    __device__ static __forceinline__ float pow2(int k) { return pow2f(k); }
    __device__ static __forceinline__ int expOf(float m) { return exponentOf(m); }
    __device__ static __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    __device__ static __forceinline__ float4 v4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
    __device__ static __forceinline__ float2 v2(float a, float b) { return make_float2(a, b); }
    __device__ static __forceinline__ int32_t weight(float p) {  // floor(min(p, 1) * 10^7)
        return (int32_t) floorf(fminf(p, 1.0f) * (float) kProbOne);
    }
};

template <>
struct Num<double> {
    using V4 = double4;
    using V2 = double2;
    static constexpr int kMinExp = -1022, kMaxExp = 1023;
    __device__ static __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    __device__ static __forceinline__ double mx(double a, double b) { return fmax(a, b); }
    __device__ static __forceinline__ double pow2(int k) { return __longlong_as_double((long long) (1023 + k) << 52); }
    __device__ static __forceinline__ int expOf(double m) {
        return (int) ((__double_as_longlong(m) >> 52) & 0x7ff) - 1023;
    }
    __device__ static __forceinline__ double div(double a, double b) { return a / b; }
    __device__ static __forceinline__ double4 v4(double a, double b, double c, double d) {
        return make_double4(a, b, c, d);
    }
    __device__ static __forceinline__ double2 v2(double a, double b) { return make_double2(a, b); }
    __device__ static __forceinline__ int32_t weight(double p) { return (int32_t) floor(fmin(p, 1.0) * (double) kProbOne); }
};

// Arithmetic over the C slots of a lane: r = a*b, r = a*s, r = fma(a, s, c) slot by slot
// (a scalar s is broadcast). In FP32 with an even C, slots 2p and 2p+1 go through one
// packed two-lane instruction (sm_100 FMUL2 / FFMA2: the same IEEE round-to-nearest
// products and fused multiply-adds as the scalar forms, half the issue slots).
template <int C, class V>
struct SlotMath {
    static constexpr bool kPacked = std::is_same<V, float>::value && (C % 2) == 0;
    __device__ static __forceinline__ void mul(V (&r)[C], const V (&a)[C], const V (&b)[C]) {
        if constexpr (kPacked) {
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const float2 v = __fmul2_rn(make_float2(a[j], a[j + 1]), make_float2(b[j], b[j + 1]));
                r[j] = v.x;
                r[j + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) r[j] = a[j] * b[j];
        }
    }
    __device__ static __forceinline__ void muls(V (&r)[C], const V (&a)[C], V s) {
        if constexpr (kPacked) {
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const float2 v = __fmul2_rn(make_float2(a[j], a[j + 1]), make_float2(s, s));
                r[j] = v.x;
                r[j + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) r[j] = a[j] * s;
        }
    }
    __device__ static __forceinline__ void fmas(V (&r)[C], const V (&a)[C], V s, const V (&c)[C]) {
        if constexpr (kPacked) {
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const float2 v =
                    __ffma2_rn(make_float2(a[j], a[j + 1]), make_float2(s, s), make_float2(c[j], c[j + 1]));
                r[j] = v.x;
                r[j + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) r[j] = Num<V>::fma(a[j], s, c[j]);
        }
    }
};

// Reductions within an aligned group of L lanes.
template <int L, class V>
__device__ __forceinline__ V groupMax(V v) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v = Num<V>::mx(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

// Maximum of non-negative values over the group. For non-negative FP32 values (never -0:
// every state value is a product or sum of positive factors, or +0) the order of the bit
// patterns is the order of the values, so a whole warp reduces in one redux.sync.
template <int L>
__device__ __forceinline__ float groupMaxNonNeg(float v) {
    if constexpr (L == 32) return __uint_as_float(__reduce_max_sync(FULL_MASK, __float_as_uint(v)));
    else return groupMax<L>(v);
}

template <int L>
__device__ __forceinline__ double groupMaxNonNeg(double v) {
    return groupMax<L>(v);
}

template <int L, class V>
__device__ __forceinline__ V groupSum(V v) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ int warpMaxInt(int v) {
    return __reduce_max_sync(FULL_MASK, v);
}

// Value held by lane gl+1 of the group (0 past the group's last lane).
template <int L, class V>
__device__ __forceinline__ V fromNext(V v, int gl) {
    const V r = __shfl_down_sync(FULL_MASK, v, 1, L);
    return gl == L - 1 ? V(0) : r;
}

// Value held by lane gl-1 of the group (0 before the group's first lane).
template <int L, class V>
__device__ __forceinline__ V fromPrev(V v, int gl) {
    const V r = __shfl_up_sync(FULL_MASK, v, 1, L);
    return gl == 0 ? V(0) : r;
}

// This group's bits of a warp ballot, shifted down to bit 0.
template <int L>
__device__ __forceinline__ unsigned groupBits(unsigned ballot, int g) {
    return L == 32 ? ballot : (ballot >> (g * L)) & ((1u << L) - 1u);
}

// 16-byte asynchronous copy into the dynamic shared array at byte offset `off`.
__device__ __forceinline__ void cpAsync16(uint32_t off, const void *gmem) {
    const unsigned s = (unsigned) __cvta_generic_to_shared(mpSmem) + off;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cpAsyncCommit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void cpAsyncWaitAllButOne() {
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Task context (identical over the lanes of a group)
// ---------------------------------------------------------------------------

template <class V>
struct Ctx {
    int gl;                 // lane within the group
    int g;                  // group within the warp
    int lx, ly, N;
    const uint16_t *xs;
    const uint16_t *ys;
    const int4 *band;       // (band lo, band hi, hull lo, hull hi) of d = 0..N, in window slots
    V t[9];                 // transitions from*3+to, in the arithmetic type
    uint32_t repOff;        // byte offset of the task's repeat table in shared memory
    uint32_t model;         // 0 forward strand, 1 reverse strand
    int rle;
    int strandFwd;
    int nTables;            // repeat tables in shared memory (1 when both strands share one)
};

// Decoded symbols: packed shared-memory byte offsets and the gap emission. For x, the low 17
// bits hold the offset of the repeat-table row (table, x base row, x repeat count) and the high
// bits the offset of the match-table row (model, x base); for y, the y repeat count and y base
// columns. The sum of an x and a y symbol therefore holds both cell offsets (the low part stays
// below 2^17, so it never carries). Positions outside the sequence decode to 'N' with repeat
// count 0, so every ring entry is a valid table offset.
template <class CT>
__device__ __forceinline__ uint2 decodeX(const CT &c, int pos, int &bad) {
    int b = 4, rc = 0;
    if (pos >= 0 && pos < c.lx) {
        uint32_t s = c.xs[pos];
        b = c.rle ? (int) (s & 255u) : (int) s;
        rc = c.rle ? (int) (s >> 8) : 0;
        b = b > 4 ? 4 : b;
        if (rc >= kMaxRepeat) {  // keeps the table lookup in bounds; reported as an argument error
            rc = kMaxRepeat - 1;
            bad = 1;
        }
    }
    int bb = b == 4 ? 0 : b;  // 'N' reads the A row of the repeat table (impl/polisher.c:1758)
    int row = c.strandFwd ? bb : 3 - bb;
    uint32_t pk = (c.repOff + (uint32_t) ((row * (kMaxRepeat * kMaxRepeat) + rc * kMaxRepeat) * 4)) |
                  ((kMatchOff + c.model * 100u + (uint32_t) (b * 20)) << 17);
    return make_uint2(pk, __float_as_uint(ldsF(kGapXOff + c.model * 20u + (uint32_t) b * 4u)));
}

template <class CT>
__device__ __forceinline__ uint2 decodeY(const CT &c, int pos, int &bad) {
    int b = 4, rc = 0;
    if (pos >= 0 && pos < c.ly) {
        uint32_t s = c.ys[pos];
        b = c.rle ? (int) (s & 255u) : (int) s;
        rc = c.rle ? (int) (s >> 8) : 0;
        b = b > 4 ? 4 : b;
        if (rc >= kMaxRepeat) {
            rc = kMaxRepeat - 1;
            bad = 1;
        }
    }
    uint32_t pk = (uint32_t) (rc * 4) | ((uint32_t) (b * 4) << 17);
    return make_uint2(pk, __float_as_uint(ldsF(kGapYOff + c.model * 20u + (uint32_t) b * 4u)));
}

__device__ __forceinline__ float matchEmission(uint32_t xpk, uint32_t ypk) {
    const uint32_t s = xpk + ypk;
    return ldsF(s & 0x1ffffu) * ldsF(s >> 17);
}

// Decoded symbols of a span of positions in shared memory (one ring per sequence and group).
template <int R>
struct Ring {
    uint32_t base;  // byte offset of the ring (R entries of 8 bytes)
    int lo;
    int bad;
    __device__ __forceinline__ uint32_t at(int pos) const { return base + ((uint32_t) (pos & (R - 1)) << 3); }
    __device__ __forceinline__ uint2 get(int pos) const { return lds<uint2>(at(pos)); }
};

// Decodes positions [newLo, newLo+R) into the group's ring where `doFill`; returns 1 if a
// symbol of this group's fill was out of range. Called by every lane of the warp.
template <int R, int L, bool IS_X, class CT>
__device__ __noinline__ int ringFillRaw(CT c, uint32_t base, int newLo, int doFill) {
    int bad = 0;
    if (doFill) {
#pragma unroll 4
        for (int k = 0; k < R / L; k++) {
            int p = newLo + k * L + c.gl;
            sts<uint2>(base + ((uint32_t) (p & (R - 1)) << 3), IS_X ? decodeX(c, p, bad) : decodeY(c, p, bad));
        }
    }
    const unsigned b = __ballot_sync(FULL_MASK, bad);
    __syncwarp();
    return groupBits<L>(b, c.g) ? 1 : 0;
}

// Makes positions [needLo, needHi] resident for the groups where `active`.
template <int R, int L, bool IS_X, class CT>
__device__ __forceinline__ void ringEnsure(const CT &c, Ring<R> &r, int needLo, int needHi, bool up, bool active) {
    const bool need = active && (needLo < r.lo || needHi >= r.lo + R);
    if (__any_sync(FULL_MASK, need)) {
        const int slack = R - (needHi - needLo + 1);
        const int newLo = up ? needLo - slack / 8 : needLo - (slack - slack / 8);
        r.bad |= ringFillRaw<R, L, IS_X, CT>(c, r.base, newLo, need ? 1 : 0);
        if (need) r.lo = newLo;
    }
}

// Makes the symbols of diagonal d resident in both rings (window Q) and returns the first
// diagonal after d whose symbols may leave them. While the window does not move, the x
// range [x0-1, x0+S-2] with x0 = Q + (d+1)/2 and the y range [y0-S, y0-1] with
// y0 = d/2 - Q only grow, so the rings stay valid until x0+S-2 or y0-1 passes the ring's
// top; a window shift forces a new check. Called by every lane of the warp.
template <int R, int L, int S, class CT>
__device__ __forceinline__ int ensureRings(const CT &c, Ring<R> &rx, Ring<R> &ry, int d, int Q, bool up,
                                           bool active) {
    const int x0 = Q + ((d + 1) >> 1), y0 = d - x0;
    ringEnsure<R, L, true, CT>(c, rx, x0 - 1, x0 + S - 2, up, active);
    ringEnsure<R, L, false, CT>(c, ry, y0 - S, y0 - 1, up, active);
    // x valid while (d'+1)/2 <= rx.lo + R + 1 - S - Q, y valid while d'/2 <= ry.lo + R + Q
    const int a = min(rx.lo + R + 1 - S - Q, 1 << 28), b = min(ry.lo + R + Q, 1 << 28);
    return min(2 * a, 2 * b + 1) + 1;
}

template <int C>
struct Slots {
    uint32_t xpk[C];
    float ex[C];
    uint32_t ypk[C];
    float ey[C];
};

// x of slot 0 at diagonal d in window Q
__device__ __forceinline__ int slotX0(int d, int Q) {
    return Q + ((d + 1) >> 1);
}

template <int C, int R>
__device__ __forceinline__ void loadSlots(int gl, const Ring<R> &rx, const Ring<R> &ry, int d, int Q, Slots<C> &s) {
    const int x0 = slotX0(d, Q), y0 = d - x0;
#pragma unroll
    for (int j = 0; j < C; j++) {
        const int i = gl * C + j;
        const uint2 vx = rx.get(x0 + i - 1);
        const uint2 vy = ry.get(y0 - i - 1);
        s.xpk[j] = vx.x;
        s.ex[j] = __uint_as_float(vx.y);
        s.ypk[j] = vy.x;
        s.ey[j] = __uint_as_float(vy.y);
    }
}

// Slot symbols from diagonal d-1 to d (window unchanged): entering odd d the x of
// every slot grows by one, entering even d the y of every slot grows by one. `fresh` is
// the sequence position that enters the window: x of the last slot (odd d) or y of the
// first slot (even d).
template <int C, int L, int R, int PAR>
__device__ __forceinline__ void stepSlotsAt(int gl, const Ring<R> &rx, const Ring<R> &ry, int freshPos,
                                            Slots<C> &s) {
    if (PAR) {
        const uint2 fresh = rx.get(freshPos);
        uint32_t npk = __shfl_down_sync(FULL_MASK, s.xpk[0], 1, L);
        float ne = __shfl_down_sync(FULL_MASK, s.ex[0], 1, L);
        if (gl == L - 1) {
            npk = fresh.x;
            ne = __uint_as_float(fresh.y);
        }
#pragma unroll
        for (int j = 0; j < C - 1; j++) {
            s.xpk[j] = s.xpk[j + 1];
            s.ex[j] = s.ex[j + 1];
        }
        s.xpk[C - 1] = npk;
        s.ex[C - 1] = ne;
    } else {
        const uint2 fresh = ry.get(freshPos);
        uint32_t npk = __shfl_up_sync(FULL_MASK, s.ypk[C - 1], 1, L);
        float ne = __shfl_up_sync(FULL_MASK, s.ey[C - 1], 1, L);
        if (gl == 0) {
            npk = fresh.x;
            ne = __uint_as_float(fresh.y);
        }
#pragma unroll
        for (int j = C - 1; j > 0; j--) {
            s.ypk[j] = s.ypk[j - 1];
            s.ey[j] = s.ey[j - 1];
        }
        s.ypk[0] = npk;
        s.ey[0] = ne;
    }
}

template <int C, int L, int R, int PAR>
__device__ __forceinline__ void stepSlots(int gl, const Ring<R> &rx, const Ring<R> &ry, int d, int Q, Slots<C> &s) {
    constexpr int S = L * C;
    stepSlotsAt<C, L, R, PAR>(gl, rx, ry, PAR ? slotX0(d, Q) + S - 2 : d - slotX0(d, Q) - 1, s);
}

// Forward state between diagonals: outgoing gap-x / gap-y sums of d-1 and
// outgoing match sums of d-1 and d-2 (even diagonals own mA, odd own mB).
template <int C, class V>
struct Fwd {
    V ox[C], oy[C], mA[C], mB[C];
};

// New lane gl takes old lane gl+dl of the group (values leaving the group become zero).
template <int C, int L, class V>
__device__ __forceinline__ void laneShift(V (&v)[C], int dl, int gl) {
    const int src = gl + dl;
    const bool ok = src >= 0 && src < L;
#pragma unroll
    for (int j = 0; j < C; j++) {
        const V w = __shfl_sync(FULL_MASK, v[j], src & (L - 1), L);
        v[j] = ok ? w : V(0);
    }
}

template <int C, int L, class V>
__device__ __forceinline__ void shiftFwd(Fwd<C, V> &f, int dl, int gl) {
    laneShift<C, L, V>(f.ox, dl, gl);
    laneShift<C, L, V>(f.oy, dl, gl);
    laneShift<C, L, V>(f.mA, dl, gl);
    laneShift<C, L, V>(f.mB, dl, gl);
}

// The window must contain the hull (in slots) of the bands of d-2..d+2; returns the
// lane shift (new Q = Q + C*shift). Shared by the sweep and the recompute, so both
// take the same decisions. Sets `bad` when the hull does not fit the window.
template <int C, int S>
__device__ __forceinline__ int windowShift(int Q, int needLo, int needHi, bool &bad) {
    if (needLo >= Q && needHi <= Q + S - 1) return 0;
    const int span = needHi - needLo + 1;
    if (span > S - 2 * C) {
        bad = true;
        return 0;
    }
    const int diff = needLo - (S - span) / 2 - Q;
    int dl = diff >= 0 ? diff / C : -((-diff + C - 1) / C);
    if (Q + C * dl + S - 1 < needHi) dl++;
    if (Q + C * dl > needLo) bad = true;
    return dl;
}

template <int S>
__device__ __forceinline__ int initialWindow(int needLo, int needHi) {
    return needLo - (S - (needHi - needLo + 1)) / 2;
}

// One diagonal's row of the block cache: per slot the masked forward values (fM, fX, fY)
// and the masked emissions (eM, eX, eY). FP32 with an even C keeps slot pairs adjacent,
// so that the packed arithmetic reads them without repacking: per pair p three float4,
// (fM, fM' fX, fX'), (fY, fY', eM, eM'), (eX, eX', eY, eY'), at [3p+q][lane]. Otherwise
// one (fM, fX, fY, eM) per slot in the A rows and one (eX, eY) in the B rows, [slot][lane].
// rowA / rowB are byte offsets of this lane's first entry in the diagonal's rows.
template <int C, int L, class V>
struct CacheRow {
    using N = Num<V>;
    using V4 = typename N::V4;
    using V2 = typename N::V2;
    static constexpr bool kPair = SlotMath<C, V>::kPacked;
    static constexpr uint32_t kRowA = kPair ? (uint32_t) (C * L * 24) : (uint32_t) (C * L * sizeof(V4));
    static constexpr uint32_t kRowB = kPair ? 0u : (uint32_t) (C * L * sizeof(V2));
    static constexpr uint32_t kStrideA = sizeof(V4);  // per lane
    static constexpr uint32_t kStrideB = sizeof(V2);

    __device__ static __forceinline__ void store(uint32_t rowA, uint32_t rowB, const V (&fM)[C], const V (&fX)[C],
                                                 const V (&fY)[C], const V (&eM)[C], const V (&eX)[C],
                                                 const V (&eY)[C]) {
        if constexpr (kPair) {
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const uint32_t o = rowA + (uint32_t) ((j / 2) * 3 * L * 16);
                sts<float4>(o, make_float4(fM[j], fM[j + 1], fX[j], fX[j + 1]));
                sts<float4>(o + L * 16, make_float4(fY[j], fY[j + 1], eM[j], eM[j + 1]));
                sts<float4>(o + 2 * L * 16, make_float4(eX[j], eX[j + 1], eY[j], eY[j + 1]));
            }
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) {
                sts<V4>(rowA + j * L * (uint32_t) sizeof(V4), N::v4(fM[j], fX[j], fY[j], eM[j]));
                sts<V2>(rowB + j * L * (uint32_t) sizeof(V2), N::v2(eX[j], eY[j]));
            }
        }
    }

    __device__ static __forceinline__ void load(uint32_t rowA, uint32_t rowB, V (&fM)[C], V (&fX)[C], V (&fY)[C],
                                                V (&eM)[C], V (&eX)[C], V (&eY)[C]) {
        if constexpr (kPair) {
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const uint32_t o = rowA + (uint32_t) ((j / 2) * 3 * L * 16);
                const float4 a = lds<float4>(o), b = lds<float4>(o + L * 16), e = lds<float4>(o + 2 * L * 16);
                fM[j] = a.x, fM[j + 1] = a.y, fX[j] = a.z, fX[j + 1] = a.w;
                fY[j] = b.x, fY[j + 1] = b.y, eM[j] = b.z, eM[j + 1] = b.w;
                eX[j] = e.x, eX[j + 1] = e.y, eY[j] = e.z, eY[j + 1] = e.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) {
                const V4 a = lds<V4>(rowA + j * L * (uint32_t) sizeof(V4));
                const V2 e = lds<V2>(rowB + j * L * (uint32_t) sizeof(V2));
                fM[j] = a.x, fX[j] = a.y, fY[j] = a.z, eM[j] = a.w;
                eX[j] = e.x, eY[j] = e.y;
            }
        }
    }

    // Once the backward has passed diagonal kk, its row holds the cells' posteriors, slot-major
    // per list: element (kk&1)*8 + k*kPStride + slot + (slot/32)*4 of the row (in V units). The
    // padding after every 32 slots and the shift of odd rows make both the owner lanes' stores
    // (consecutive slots) and the emitters' range reads (16 consecutive slots of two diagonals
    // per 8-lane phase) free of bank conflicts. `row` is the group's row of kk.
    static constexpr int kPStride = L * C + ((L * C) >> 5) * 4;
    static_assert((3 * kPStride + 8) * sizeof(V) <= kRowA, "the posteriors fit in the row they replace");
    __device__ static __forceinline__ uint32_t pAddr(uint32_t row, int kk, int slot, int k) {
        return row + (uint32_t) (((kk & 1) * 8 + k * kPStride + slot + (slot >> 5) * 4) * (int) sizeof(V));
    }
    __device__ static __forceinline__ void storeP(uint32_t row, int kk, int gl, const V (&pM)[C], const V (&pX)[C],
                                                  const V (&pY)[C]) {
        if constexpr (C == 2 && std::is_same<V, float>::value) {
            sts<float2>(pAddr(row, kk, 2 * gl, 0), make_float2(pM[0], pM[1]));
            sts<float2>(pAddr(row, kk, 2 * gl, 1), make_float2(pX[0], pX[1]));
            sts<float2>(pAddr(row, kk, 2 * gl, 2), make_float2(pY[0], pY[1]));
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) {
                sts<V>(pAddr(row, kk, gl * C + j, 0), pM[j]);
                sts<V>(pAddr(row, kk, gl * C + j, 1), pX[j]);
                sts<V>(pAddr(row, kk, gl * C + j, 2), pY[j]);
            }
        }
    }

    // forward values only (fM, fX, fY)
    __device__ static __forceinline__ void loadF(uint32_t rowA, V (&fM)[C], V (&fX)[C], V (&fY)[C]) {
        if constexpr (kPair) {
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const uint32_t o = rowA + (uint32_t) ((j / 2) * 3 * L * 16);
                const float4 a = lds<float4>(o);
                const float2 b = lds<float2>(o + L * 16);
                fM[j] = a.x, fM[j + 1] = a.y, fX[j] = a.z, fX[j + 1] = a.w;
                fY[j] = b.x, fY[j + 1] = b.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < C; j++) {
                const V4 a = lds<V4>(rowA + j * L * (uint32_t) sizeof(V4));
                fM[j] = a.x, fX[j] = a.y, fY[j] = a.z;
            }
        }
    }
};

// One forward anti-diagonal (PAR = d & 1). Emissions are zeroed outside the band
// [sLo, sHi], which zeroes the cell. With CACHE, the cell values and the masked
// emissions are written to the block cache row (rowA, rowB). With SYM, the cells'
// table offsets go to rowC (slot j at j*L entries). SW false: the model's switch
// transitions (gap-x -> gap-y, gap-y -> gap-x) are zero, and their products, which add
// exact zeros, are left out.
template <int C, int L, int PAR, bool CACHE, bool SYM, class V, bool SW = true>
__device__ __forceinline__ void forwardDiagonal(const Ctx<V> &c, Fwd<C, V> &st, const Slots<C> &sy, int sLo, int sHi,
                                                uint32_t rowA, uint32_t rowB, uint32_t rowC = 0) {
    using M = SlotMath<C, V>;
    V inX[C], inY[C], mIn[C];
    if (PAR) {  // odd d: gap-x source slot i, gap-y source slot i+1
        const V nb = fromNext<L>(st.oy[0], c.gl);
#pragma unroll
        for (int j = 0; j < C; j++) {
            inX[j] = st.ox[j];
            inY[j] = (j < C - 1) ? st.oy[j + 1] : nb;
            mIn[j] = st.mB[j];
        }
    } else {  // even d: gap-x source slot i-1, gap-y source slot i
        const V nb = fromPrev<L>(st.ox[C - 1], c.gl);
#pragma unroll
        for (int j = 0; j < C; j++) {
            inX[j] = (j > 0) ? st.ox[j - 1] : nb;
            inY[j] = st.oy[j];
            mIn[j] = st.mA[j];
        }
    }
    const int base = c.gl * C - sLo;
    const unsigned span = (unsigned) (sHi - sLo);
    V eM[C], eX[C], eY[C];
    if constexpr (M::kPacked) {
        // band mask as a 0/1 factor (emissions are finite, so the products are exact)
        V rp[C], mt[C], mk[C], gx[C], gy[C];
#pragma unroll
        for (int j = 0; j < C; j++) {
            const bool in = (unsigned) (base + j) <= span;
            const uint32_t s2 = sy.xpk[j] + sy.ypk[j];
            rp[j] = ldsF(s2 & 0x1ffffu);
            mt[j] = ldsF(s2 >> 17);
            mk[j] = in ? V(1) : V(0);
            gx[j] = sy.ex[j];
            gy[j] = sy.ey[j];
            if (SYM) sts<uint32_t>(rowC + j * L * 4, in ? s2 : 0xffffffffu);
        }
        M::mul(eM, rp, mt);
        M::mul(eM, eM, mk);
        M::mul(eX, gx, mk);
        M::mul(eY, gy, mk);
    } else {
#pragma unroll
        for (int j = 0; j < C; j++) {
            const bool in = (unsigned) (base + j) <= span;
            eM[j] = in ? (V) matchEmission(sy.xpk[j], sy.ypk[j]) : V(0);
            eX[j] = in ? (V) sy.ex[j] : V(0);
            eY[j] = in ? (V) sy.ey[j] : V(0);
            // the cell's table offsets (repeat | match << 17), for the adjoint's histograms
            if (SYM) sts<uint32_t>(rowC + j * L * 4, in ? sy.xpk[j] + sy.ypk[j] : 0xffffffffu);
        }
    }
    V fM[C], fX[C], fY[C], a[C];
    M::mul(fM, eM, mIn);
    M::mul(fX, eX, inX);
    M::mul(fY, eY, inY);
    // match: t00*fM + t10*fX + t20*fY; gap-x: t01, t11, t21; gap-y: t02, t22, t12 (in that order)
    M::muls(a, fM, c.t[0 * 3 + 0]);
    M::fmas(a, fX, c.t[1 * 3 + 0], a);
    if (PAR) M::fmas(st.mB, fY, c.t[2 * 3 + 0], a); else M::fmas(st.mA, fY, c.t[2 * 3 + 0], a);
    M::muls(a, fM, c.t[0 * 3 + 1]);
    if constexpr (SW) {
        M::fmas(a, fX, c.t[1 * 3 + 1], a);
        M::fmas(st.ox, fY, c.t[2 * 3 + 1], a);
    } else {
        M::fmas(st.ox, fX, c.t[1 * 3 + 1], a);
    }
    M::muls(a, fM, c.t[0 * 3 + 2]);
    if constexpr (SW) {
        M::fmas(a, fY, c.t[2 * 3 + 2], a);
        M::fmas(st.oy, fX, c.t[1 * 3 + 2], a);
    } else {
        M::fmas(st.oy, fY, c.t[2 * 3 + 2], a);
    }
    if (CACHE) CacheRow<C, L, V>::store(rowA, rowB, fM, fX, fY, eM, eX, eY);
}

// Diagonal 0: the start cell (x-y = 0) holds the start (or ragged-start) probabilities.
template <int C, int L, bool CACHE, class V>
__device__ __forceinline__ void forwardOrigin(const Ctx<V> &c, const float *startP, int Q, Fwd<C, V> &st,
                                              uint32_t rowA, uint32_t rowB) {
    using N = Num<V>;
    V fM[C], fX[C], fY[C], z[C];
#pragma unroll
    for (int j = 0; j < C; j++) {
        const bool here = c.gl * C + j == -Q;
        fM[j] = here ? (V) startP[0] : V(0);
        fX[j] = here ? (V) startP[1] : V(0);
        fY[j] = here ? (V) startP[2] : V(0);
        z[j] = V(0);
        st.mA[j] = N::fma(c.t[2 * 3 + 0], fY[j], N::fma(c.t[1 * 3 + 0], fX[j], c.t[0 * 3 + 0] * fM[j]));
        st.ox[j] = N::fma(c.t[2 * 3 + 1], fY[j], N::fma(c.t[1 * 3 + 1], fX[j], c.t[0 * 3 + 1] * fM[j]));
        st.oy[j] = N::fma(c.t[1 * 3 + 2], fX[j], N::fma(c.t[2 * 3 + 2], fY[j], c.t[0 * 3 + 2] * fM[j]));
        st.mB[j] = V(0);
    }
    if (CACHE) CacheRow<C, L, V>::store(rowA, rowB, fM, fX, fY, z, z, z);
}

// Rescales the carried forward state by a power of two; returns the exponent removed.
template <int C, int L, class V>
__device__ __forceinline__ int rescaleFwd(Fwd<C, V> &st) {
    using N = Num<V>;
    V m = V(0);
#pragma unroll
    for (int j = 0; j < C; j++) m = N::mx(m, N::mx(N::mx(st.ox[j], st.oy[j]), N::mx(st.mA[j], st.mB[j])));
    m = groupMaxNonNeg<L>(m);
    if (!(m > V(0))) return 0;
    const int k = N::expOf(m);
    const V sc = N::pow2(-k);
    using M = SlotMath<C, V>;
    M::muls(st.ox, st.ox, sc);
    M::muls(st.oy, st.oy, sc);
    M::muls(st.mA, st.mA, sc);
    M::muls(st.mB, st.mB, sc);
    return k;
}

// ---------------------------------------------------------------------------
// Output: ordered group compaction of one diagonal's tuples.
// ---------------------------------------------------------------------------

struct Out {
    int4 *t[3];   // the task's staging region of each list: (weight, x, y, 0)
    int top[3];
    int written[3];
    int xShift, yShift;
};

// ---------------------------------------------------------------------------
// Shared workspace of one group
// ---------------------------------------------------------------------------

// Adjoint histogram bins (floats): match posteriors by (model, x base, y base), gap-x by
// (model, x base), gap-y by (model, y base), state posteriors at the first and the last cell by
// (model, state); then the repeat tables (block-wide).
constexpr int kHistMatch = 0, kHistGapX = 50, kHistGapY = 60, kHistStart = 70, kHistEnd = 76, kHistSmall = 82;

template <int C, int L, int K, bool ADJ = false, class V = float>
struct GroupSmem {
    static constexpr int S = L * C;
    static constexpr int R = RingSize<S>::R;
    static constexpr size_t ringBytes = 2 * R * sizeof(uint2);
    static constexpr size_t bandRingBytes = 64 * sizeof(int4);
    static constexpr size_t walkBandBytes = K * sizeof(int4);
    static constexpr size_t cacheABytes = (size_t) K * CacheRow<C, L, V>::kRowA;
    static constexpr size_t cacheBBytes = (size_t) K * CacheRow<C, L, V>::kRowB;
    static constexpr size_t cacheCBytes = ADJ ? (size_t) K * S * sizeof(uint32_t) : 0;
    static constexpr size_t infoBytes = K * sizeof(int2);
    // adjoint only: the warp's own small histograms (no contention with the block's other warps)
    static constexpr size_t smallHistBytes = ADJ ? (((size_t) kHistSmall * sizeof(float) + 15) & ~(size_t) 15) : 0;
    static constexpr size_t bytes = ringBytes + bandRingBytes + walkBandBytes + cacheABytes + cacheBBytes +
                                    cacheCBytes + infoBytes + smallHistBytes;
};

template <int C, int L, int K>
struct GroupMem {
    Ring<RingSize<L * C>::R> rx, ry;
    uint32_t bandRing;  // byte offsets in shared memory: 64 band records (int4)
    uint32_t walkBand;  // K band records of the block being walked
    uint32_t cacheA;    // [K] rows of the block cache (CacheRow)
    uint32_t cacheB;    // [K] B rows of the block cache (empty in the paired layout)
    uint32_t cacheC;    // adjoint only: [K][S] uint32 table offsets of the cell
    uint32_t info;      // [K] int2: window, shift
    uint32_t hist;      // adjoint only: the block's histograms (its repeat tables at kHistSmall)
    uint32_t whist;     // adjoint only: the warp's small histograms (kHistSmall floats)
};

// Bytes of the block-wide adjoint histograms (the repeat tables start at bin kHistSmall).
__host__ __device__ constexpr size_t histBytes(int nTables) {
    return ((size_t) (kHistSmall + nTables * kRepTable) * sizeof(float) + 15) & ~(size_t) 15;
}

// Global slot of small-histogram bin i (see kExp* in mp_internal.h).
__device__ __forceinline__ int expectSlot(int i) {
    if (i < kHistGapX) return (i / 25) * kExpPerModel + kExpMatch + i % 25;
    if (i < kHistGapY) return ((i - kHistGapX) / 5) * kExpPerModel + kExpGapX + (i - kHistGapX) % 5;
    if (i < kHistStart) return ((i - kHistGapY) / 5) * kExpPerModel + kExpGapY + (i - kHistGapY) % 5;
    if (i < kHistEnd) return ((i - kHistStart) / 3) * kExpPerModel + kExpStart + (i - kHistStart) % 3;
    return ((i - kHistEnd) / 3) * kExpPerModel + kExpEnd + (i - kHistEnd) % 3;
}

template <class V>
struct Scratch {
    typename Num<V>::V4 *chk;  // checkpoints of the group's task: [block][C][L]
    int2 *scal;       // (exponent, window) per checkpoint
    int blocks;
};

template <int C, int L, class V>
__device__ __forceinline__ void storeFwd(typename Num<V>::V4 *p, int gl, const Fwd<C, V> &st) {
#pragma unroll
    for (int j = 0; j < C; j++) p[j * L + gl] = Num<V>::v4(st.ox[j], st.oy[j], st.mA[j], st.mB[j]);
}

template <int C, class V>
__device__ __forceinline__ void loadFwd(const typename Num<V>::V4 (&v)[C], Fwd<C, V> &st) {
#pragma unroll
    for (int j = 0; j < C; j++) {
        st.ox[j] = v[j].x;
        st.oy[j] = v[j].y;
        st.mA[j] = v[j].z;
        st.mB[j] = v[j].w;
    }
}

// ---------------------------------------------------------------------------
// Traceback walk over (tbTo, D] of every active group's task, in lockstep:
// iteration w processes block D/K - w of each group; every block is recomputed
// into the shared cache, then the backward recurrence and posteriors run over it.
// Block starts are multiples of K (even), so the parity of a block position is
// the same in every group.
// ---------------------------------------------------------------------------

// Posterior tuples of one walked block, written after the backward has stored the block's
// posteriors in the cache rows. The output order is the order of the walk: diagonals top
// down, slots (ascending x-y) within a diagonal, each list written from the top of its
// region downwards, so that the region reads in the reference's order. Lane gl of a group
// takes E = K*C consecutive entries of that order: slots [s0, s0+E) of diagonal kk (L/K lanes
// per diagonal). Its hits are ranked by one group-wide prefix sum per list. `emitMask` bit kk:
// diagonal dStart+kk emits (identical over the group's lanes). Called by every lane.
template <int C, int L, int K, class V>
__device__ __forceinline__ void emitBlock(int gl, const GroupMem<C, L, K> &gm, unsigned emitMask, int dStart,
                                          Out &o, V thr) {
    using CR = CacheRow<C, L, V>;
    constexpr int E = K * C, LPD = L / K;
    static_assert(L % K == 0 && E <= 32, "a lane's entries lie within one diagonal and one mask word");
    const int kk = K - 1 - gl / LPD;
    const int s0 = (gl % LPD) * E;
    const int d = dStart + kk;
    const bool on = (emitMask >> kk) & 1u;
    const int Q = lds<int2>(gm.info + kk * 8).x;
    const int x0 = slotX0(d, Q) + s0;  // x of the lane's first slot
    const int xo = x0 - 1 + o.xShift, yo = d - x0 - 1 + o.yShift;
    const uint32_t row = gm.cacheA + (uint32_t) kk * CR::kRowA;
    unsigned mask[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        unsigned m = 0;
        if constexpr (C == 2 && K == 8 && std::is_same<V, float>::value) {
            // 16 consecutive slots, 16-byte aligned and within one 32-slot stretch
            const uint32_t base = CR::pAddr(row, kk, s0, k);
#pragma unroll
            for (int i = 0; i < E / 4; i++) {
                const float4 v = lds<float4>(base + (uint32_t) (i * 16));
                if (v.x >= thr) m |= 1u << (4 * i);
                if (v.y >= thr) m |= 2u << (4 * i);
                if (v.z >= thr) m |= 4u << (4 * i);
                if (v.w >= thr) m |= 8u << (4 * i);
            }
        } else {
#pragma unroll
            for (int e = 0; e < E; e++)
                if (lds<V>(CR::pAddr(row, kk, s0 + e, k)) >= thr) m |= 1u << e;
        }
        mask[k] = on ? m : 0u;
    }
    // ranks: exclusive prefix sums of the lanes' hit counts over the group, the three lists
    // packed in 10-bit fields of one word when a group's total (at most K*S) fits
    int excl[3], total[3];
    if constexpr (K * L * C < 1024) {
        const unsigned cnt = (unsigned) __popc(mask[0]) | ((unsigned) __popc(mask[1]) << 10) |
                             ((unsigned) __popc(mask[2]) << 20);
        unsigned incl = cnt;
#pragma unroll
        for (int off = 1; off < L; off <<= 1) {
            const unsigned t = __shfl_up_sync(FULL_MASK, incl, off, L);
            if (gl >= off) incl += t;
        }
        const unsigned tot = __shfl_sync(FULL_MASK, incl, L - 1, L);
        const unsigned ex = incl - cnt;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            excl[k] = (int) ((ex >> (10 * k)) & 1023u);
            total[k] = (int) ((tot >> (10 * k)) & 1023u);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int cnt = __popc(mask[k]);
            int incl = cnt;
#pragma unroll
            for (int off = 1; off < L; off <<= 1) {
                const int t = __shfl_up_sync(FULL_MASK, incl, off, L);
                if (gl >= off) incl += t;
            }
            total[k] = __shfl_sync(FULL_MASK, incl, L - 1, L);
            excl[k] = incl - cnt;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        unsigned m = mask[k];
        int pos = o.top[k] - 1 - o.written[k] - excl[k];
        while (m) {
            const int e = __ffs(m) - 1;
            m &= m - 1;
            if (pos >= 0) {
                const V p = lds<V>(CR::pAddr(row, kk, s0 + e, k));
                o.t[k][pos] = make_int4(Num<V>::weight(p), xo + e, yo - e, 0);
            }
            pos--;
        }
        o.written[k] += total[k];
    }
}

struct Walk {
    int D, tbTo, tbFrom, atEnd, active, emit;
    const float *startP;
    const float *endP;
};

template <int C, int L, int K, bool ADJ, class V, bool SW>
__device__ __forceinline__ void walkSegment(const Ctx<V> &c, GroupMem<C, L, K> &gm, const Scratch<V> &sc,
                                            const Walk &wk, V thr, Out &o, double &logLik, bool &bad,
                                            bool &rangeBad, double (&accD)[9], double *expect) {
    static_assert(!ADJ || L == 32, "the adjoint runs one task per warp");
    static_assert(!ADJ || std::is_same<V, float>::value, "the adjoint accumulates in FP32");
    using N = Num<V>;
    using V4 = typename N::V4;
    using V2 = typename N::V2;
    using CR = CacheRow<C, L, V>;
    using M = SlotMath<C, V>;
    static_assert(K <= L && (K % 2) == 0, "band records of a block are held one per lane");
    static_assert(K <= 10, "a block holds at most one total refresh");
    constexpr bool kSolo = L == 32;  // one task per warp: per-task decisions are warp-uniform
    constexpr int S = L * C;
    constexpr int R = RingSize<S>::R;
    const int gl = c.gl;
    V gX[C], gY[C], gA[C], gB[C];  // backward u-values: gap-x / gap-y of d+1, match (even d in A, odd in B)
#pragma unroll
    for (int j = 0; j < C; j++) gX[j] = gY[j] = gA[j] = gB[j] = V(0);
    int Eb = 0, posts = 0, ET = 0, untilRefresh = 0;
    V Tm = V(0);
    V llTm = V(0);  // total of the first posterior diagonal of the final segment: the likelihood
    int llET = 0;
    bool llSet = false;
    const V endM = (V) wk.endP[0], endX = (V) wk.endP[1], endY = (V) wk.endP[2];
    const int bTop = wk.active ? wk.D / K : -1;
    const int bBot = wk.active ? (wk.tbTo + 1) / K : 0;
    const int nIter = warpMaxInt(wk.active ? bTop - bBot + 1 : 0);

    // register prefetch of a block's checkpoint and band records
    V4 pchk[C];
#pragma unroll
    for (int j = 0; j < C; j++) pchk[j] = N::v4(V(0), V(0), V(0), V(0));
    int2 pscal = make_int2(0, 0);
    int4 pband = make_int4(0, 0, 0, 0);
    auto prefetch = [&](int b, bool ok) {
        if (ok && b > 0) {
#pragma unroll
            for (int j = 0; j < C; j++) pchk[j] = sc.chk[((size_t) b * C + j) * L + gl];
            pscal = sc.scal[b];
        }
        const int dd = b * K + gl;
        if (ok && gl < K && dd <= c.N) pband = c.band[dd];
    };
    prefetch(bTop, bTop >= bBot);
    const uint32_t laneA = gm.cacheA + (uint32_t) gl * CR::kStrideA, laneB = gm.cacheB + (uint32_t) gl * CR::kStrideB;
    const uint32_t laneC = gm.cacheC + (uint32_t) gl * 4;

    for (int w = 0; w < nIter; w++) {
        const int b = bTop - w;
        const bool blockOn = b >= bBot;
        const int dStart = b * K;
        const int dEnd = min(dStart + K - 1, wk.D);
        Fwd<C, V> rs;
        V4 cchk[C];
#pragma unroll
        for (int j = 0; j < C; j++) cchk[j] = pchk[j];
        const int2 cscal = pscal;
        if (blockOn && gl < K) sts<int4>(gm.walkBand + gl * 16, pband);
        __syncwarp();
        prefetch(b - 1, blockOn && b - 1 >= bBot);

        float ta[9];  // adjoint: this block's transition sums
#pragma unroll
        for (int i = 0; i < 9; i++) ta[i] = 0.0f;
        // ---------------- recompute the block ----------------
        int Q;
        int Ef;
        V chkSM[C];
        loadFwd<C, V>(cchk, rs);
        Ef = cscal.x;
        Q = cscal.y;
#pragma unroll
        for (int j = 0; j < C; j++) chkSM[j] = rs.mB[j];
        if (blockOn && b == 0) {
            const int4 b0 = lds<int4>(gm.walkBand);
            Q = initialWindow<S>(b0.z, b0.w);
            Ef = 0;
#pragma unroll
            for (int j = 0; j < C; j++) chkSM[j] = V(0);
        }
        Slots<C> sy;
        // A whole block past diagonal 0 whose window does not move and whose symbols stay in
        // the rings is recomputed without checks or branches.
        const bool full = blockOn && b > 0 && dEnd == dStart + K - 1;
        // the slots of diagonal dStart-1 (window of the checkpoint) seed the block's first step
        int checkAt = ensureRings<R, L, S>(c, gm.rx, gm.ry, dStart - 1, Q, false, full);
        bool clear = full && dEnd < checkAt;
        if (gl < K) {
            const int4 bd = lds<int4>(gm.walkBand + gl * 16);
            clear = clear && bd.z >= Q && bd.w <= Q + S - 1;
        }
        const bool flat = __all_sync(FULL_MASK, clear);
        if (flat) {
            loadSlots<C, R>(gl, gm.rx, gm.ry, dStart - 1, Q, sy);
#pragma unroll 1
            for (int kk = 0; kk < K; kk += 2) {
                const int d = dStart + kk;
                const int2 b0 = lds<int2>(gm.walkBand + kk * 16);
                const int2 b1 = lds<int2>(gm.walkBand + (kk + 1) * 16);
                const uint32_t rowA = laneA + (uint32_t) kk * CR::kRowA, rowB = laneB + (uint32_t) kk * CR::kRowB;
                const uint32_t rowC = laneC + (uint32_t) (kk * S * 4);
                stepSlots<C, L, R, 0>(gl, gm.rx, gm.ry, d, Q, sy);
                forwardDiagonal<C, L, 0, true, ADJ, V, SW>(c, rs, sy, b0.x - Q, b0.y - Q, rowA, rowB, rowC);
                stepSlots<C, L, R, 1>(gl, gm.rx, gm.ry, d + 1, Q, sy);
                forwardDiagonal<C, L, 1, true, ADJ, V, SW>(c, rs, sy, b1.x - Q, b1.y - Q, rowA + CR::kRowA, rowB + CR::kRowB,
                                                       rowC + S * 4);
            }
            if (gl < K) sts<int2>(gm.info + gl * 8, make_int2(Q, 0));
        } else {
            checkAt = dStart;  // the rings are checked, and the slots loaded, at the block's first diagonal
#pragma unroll 1
            for (int k = 0; k < K; k += 2) {
#pragma unroll
                for (int par = 0; par < 2; par++) {
                    const int kk = k + par;
                    const int d = dStart + kk;
                    const bool on = blockOn && d <= dEnd;
                    const int4 bd = lds<int4>(gm.walkBand + kk * 16);
                    const bool move = on && d > 0 && (bd.z < Q || bd.w > Q + S - 1);
                    int dl = 0;
                    bool reload = kk == 0;
                    const bool rare = __any_sync(FULL_MASK, move || (on && d >= checkAt));
                    if (rare) {
                        dl = move ? windowShift<C, S>(Q, bd.z, bd.w, bad) : 0;
                        if (__any_sync(FULL_MASK, dl != 0)) {
                            shiftFwd<C, L, V>(rs, dl, gl);
                            if (dl != 0) {
                                Q += C * dl;
                                reload = true;
                            }
                        }
                        checkAt = ensureRings<R, L, S>(c, gm.rx, gm.ry, d, Q, false, on);
                    }
                    const int sLo = bd.x - Q, sHi = bd.y - Q;
                    const uint32_t rowA = laneA + (uint32_t) kk * CR::kRowA, rowB = laneB + (uint32_t) kk * CR::kRowB;
                    const uint32_t rowC = laneC + (uint32_t) (kk * S * 4);
                    if (par) {
                        stepSlots<C, L, R, 1>(gl, gm.rx, gm.ry, d, Q, sy);
                        if (rare && reload) loadSlots<C, R>(gl, gm.rx, gm.ry, d, Q, sy);
                        forwardDiagonal<C, L, 1, true, ADJ, V, SW>(c, rs, sy, sLo, sHi, rowA, rowB, rowC);
                    } else {
                        stepSlots<C, L, R, 0>(gl, gm.rx, gm.ry, d, Q, sy);
                        if (rare && reload) loadSlots<C, R>(gl, gm.rx, gm.ry, d, Q, sy);
                        forwardDiagonal<C, L, 0, true, ADJ, V, SW>(c, rs, sy, sLo, sHi, rowA, rowB, rowC);
                        if (d == 0) forwardOrigin<C, L, true, V>(c, wk.startP, Q, rs, rowA, rowB);
                    }
                    if (gl == 0) sts<int2>(gm.info + kk * 8, make_int2(Q, dl));
                }
            }
        }
        __syncwarp();

        // ---------------- backward over the block ----------------
        // Posterior of a cell = f * b * 2^(Ef + Eb - ET) / Tm: the factor changes only at a
        // total refresh and between blocks.
        auto scaleOf = [&]() {
            return Tm > V(0) ? N::div(N::pow2(max(N::kMinExp, min(N::kMaxExp, Ef + Eb - ET))), Tm) : V(0);
        };
        V postScale = scaleOf();
        unsigned emitMask = 0;  // diagonals of the block that emit tuples
        // Flat blocks: the posterior diagonals are kk <= pLim, the first processed is firstPost,
        // and the total is refreshed at kk = refreshKK (-1: none; at most one, as K <= 10);
        // the walk's counters are advanced once after the block.
        int pLim = 0, firstPost = -1, refreshKK = -1, posts0 = 0;
        // One diagonal (PAR = d & 1). FLAT: every diagonal of the block is on and no window
        // shift occurs, so the step has no votes or branches (the total is refreshed by
        // selection and tuples are written with predicated stores).
        auto back = [&](auto parity, auto flatTag, int kk) {
            constexpr int PAR = decltype(parity)::value;
            constexpr bool FLAT = decltype(flatTag)::value;
            const int d = dStart + kk;
            const bool on = FLAT || (blockOn && d <= dEnd && d > wk.tbTo);
            const int2 inf = FLAT ? make_int2(Q, 0) : lds<int2>(gm.info + kk * 8);
            V fM[C], fX[C], fY[C], eM[C], eX[C], eY[C];
            CR::load(laneA + (uint32_t) kk * CR::kRowA, laneB + (uint32_t) kk * CR::kRowB, fM, fX, fY, eM, eX, eY);
            V bM[C], bX[C], bY[C];
            V sX[C], sY[C], sM2[C];  // u-values of the gap-x, gap-y and match successors
            {
                if (PAR) {  // odd d: gap-x successor slot i+1, gap-y successor slot i
                    const V nb = fromNext<L>(gX[0], gl);
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        sX[j] = (j < C - 1) ? gX[j + 1] : nb;
                        sY[j] = gY[j];
                    }
                } else {  // even d: gap-x successor slot i, gap-y successor slot i-1
                    const V nb = fromPrev<L>(gY[C - 1], gl);
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        sX[j] = gX[j];
                        sY[j] = (j > 0) ? gY[j - 1] : nb;
                    }
                }
#pragma unroll
                for (int j = 0; j < C; j++) sM2[j] = PAR ? gB[j] : gA[j];
                // b_s = t_sX * uX + t_sY * uY + t_sM * uM, accumulated in that order
                V a[C];
                M::muls(a, sX, c.t[0 * 3 + 1]);
                M::fmas(a, sY, c.t[0 * 3 + 2], a);
                M::fmas(bM, sM2, c.t[0 * 3 + 0], a);
                M::muls(a, sX, c.t[1 * 3 + 1]);
                if constexpr (SW) M::fmas(a, sY, c.t[1 * 3 + 2], a);
                M::fmas(bX, sM2, c.t[1 * 3 + 0], a);
                if constexpr (SW) {
                    M::muls(a, sX, c.t[2 * 3 + 1]);
                    M::fmas(a, sY, c.t[2 * 3 + 2], a);
                } else {
                    M::muls(a, sY, c.t[2 * 3 + 2]);
                }
                M::fmas(bY, sM2, c.t[2 * 3 + 0], a);
                if (!FLAT && d == wk.D) {  // the walk's first diagonal holds the end probabilities
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        bM[j] = endM;
                        bX[j] = endX;
                        bY[j] = endY;
                    }
                }
            }
            const bool post = on && d <= wk.tbFrom;
            // total probability refresh: 1st, 11th, 21st ... posterior diagonal of the walk
            const bool refresh = FLAT ? kk == refreshKK : post && untilRefresh == 0;
            const int postsNow = FLAT ? posts0 + (firstPost - kk) : posts;  // posterior diagonals before d
            if ((FLAT && kSolo) ? refresh : __any_sync(FULL_MASK, refresh)) {
                // cells of d plus the match transitions crossing d (impl/pairwiseAligner.c:567-584)
                V sM1[C];
                if (kk > 0) {
                    V qM[C], qX[C], qY[C];
                    CR::loadF(laneA + (uint32_t) (kk - 1) * CR::kRowA, qM, qX, qY);
#pragma unroll
                    for (int j = 0; j < C; j++)
                        sM1[j] = N::fma(c.t[2 * 3 + 0], qY[j], N::fma(c.t[1 * 3 + 0], qX[j], c.t[0 * 3 + 0] * qM[j]));
                } else {
#pragma unroll
                    for (int j = 0; j < C; j++) sM1[j] = chkSM[j];
                }
                if (!FLAT) laneShift<C, L, V>(sM1, on ? inf.y : 0, gl);
                V part = V(0);
#pragma unroll
                for (int j = 0; j < C; j++) {
                    const V uMn = PAR ? gA[j] : gB[j];  // match u of d+1
                    part = N::fma(fM[j], bM[j], part);
                    part = N::fma(fX[j], bX[j], part);
                    part = N::fma(fY[j], bY[j], part);
                    part = N::fma(uMn, sM1[j], part);
                }
                const V T = groupSum<L>(part);
                const int ex = N::expOf(T);
                const V tm = T > V(0) ? T * N::pow2(-ex) : V(0);
                const int et = T > V(0) ? Ef + Eb + ex : 0;
                // The total through every diagonal of a walk is one quantity; a refresh that finds
                // no total, or one that disagrees with the walk's previous total, means the scaled
                // values lost their range (the host runs such sub-problems again in FP64).
                if (refresh) {
                    bool ok = tm > V(0);
                    if (ok && postsNow > 0 && Tm > V(0) && abs(et - ET) <= 1) {
                        const V r = N::div(tm * N::pow2(et - ET), Tm) - V(1);
                        ok = r <= V(1e-3) && r >= V(-1e-3);
                    } else if (postsNow > 0) {
                        ok = false;
                    }
                    rangeBad = rangeBad || !ok;
                }
                const bool first = refresh && wk.atEnd && postsNow == 0;
                llTm = first ? tm : llTm;
                llET = first ? et : llET;
                llSet = llSet || first;
                Tm = refresh ? tm : Tm;
                ET = refresh ? et : ET;
                postScale = scaleOf();
            }
            if constexpr (!FLAT) {
                untilRefresh = refresh ? 9 : untilRefresh - (post ? 1 : 0);
                posts += post ? 1 : 0;
            }
            const bool emit = post && Tm > V(0) && wk.emit;
            if constexpr (!ADJ) {
                // the row of d is not read again: it takes the posteriors (tuples after the block)
                if (FLAT || __any_sync(FULL_MASK, emit)) {
                    V p[3][C];
                    M::mul(p[0], fM, bM);
                    M::mul(p[1], fX, bX);
                    M::mul(p[2], fY, bY);
                    M::muls(p[0], p[0], postScale);
                    M::muls(p[1], p[1], postScale);
                    M::muls(p[2], p[2], postScale);
                    __syncwarp();  // every lane has read its part of the row
                    CR::storeP(gm.cacheA + (uint32_t) kk * CR::kRowA, kk, gl, p[0], p[1], p[2]);
                }
                emitMask |= emit ? 1u << kk : 0u;
            } else {
                (void) emit;
            }
            if constexpr (ADJ) {
                // expected counts: transitions out of the cells of d (f_from * u_to, scaled by 1/P)
                // and the emission posteriors of each state, binned by the cell's table entries
                const bool acc = post && Tm > V(0);
                if (FLAT || __any_sync(FULL_MASK, acc)) {
                    const int ex = max(N::kMinExp, min(N::kMaxExp, Ef + Eb - ET));
                    const float scale = acc ? N::div(N::pow2(ex), Tm) : 0.0f;
                    const int xl = slotX0(d, inf.x) + gl * C;
                    float *hs = reinterpret_cast<float *>(mpSmem + gm.hist);
                    float *ws = reinterpret_cast<float *>(mpSmem + gm.whist);
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        const float fm = fM[j] * scale, fx = fX[j] * scale, fy = fY[j] * scale;
                        ta[0] = __fmaf_rn(fm, sM2[j], ta[0]);
                        ta[1] = __fmaf_rn(fm, sX[j], ta[1]);
                        ta[2] = __fmaf_rn(fm, sY[j], ta[2]);
                        ta[3] = __fmaf_rn(fx, sM2[j], ta[3]);
                        ta[4] = __fmaf_rn(fx, sX[j], ta[4]);
                        ta[5] = __fmaf_rn(fx, sY[j], ta[5]);
                        ta[6] = __fmaf_rn(fy, sM2[j], ta[6]);
                        ta[7] = __fmaf_rn(fy, sX[j], ta[7]);
                        ta[8] = __fmaf_rn(fy, sY[j], ta[8]);
                        const float pm = fm * bM[j], px = fx * bX[j], py = fy * bY[j];
                        const uint32_t sym = lds<uint32_t>(laneC + (uint32_t) ((kk * S + j * L) * 4));
                        const int x = xl + j, y = d - x;
                        const uint32_t mb = sym >> 19;                                  // model*25 + xb*5 + yb
                        const uint32_t rb = ((sym & 0x1ffffu) - kRepBase) >> 2;         // repeat-table entry
                        // State posteriors below kTinyPosterior are left out of the emission
                        // histograms: even 1e8 such cells in one bin move it by < 1e-4, while
                        // the band's cells far from the alignment path stop costing a
                        // contended shared-memory atomic each.
                        constexpr float kTinyPosterior = 1e-12f;
                        if (sym != 0xffffffffu && mb < 50u) {
                            if (x > 0 && y > 0 && pm > kTinyPosterior) {
                                atomicAdd(ws + kHistMatch + mb, pm);
                                if (c.rle && rb < (uint32_t) (c.nTables * kRepTable))
                                    atomicAdd(hs + kHistSmall + rb, pm);
                            }
                            if (x > 0 && px > kTinyPosterior)
                                atomicAdd(ws + kHistGapX + (mb / 25) * 5 + (mb % 25) / 5, px);
                            if (y > 0 && py > kTinyPosterior) atomicAdd(ws + kHistGapY + (mb / 25) * 5 + mb % 5, py);
                        }
                        if (d == 0 || d == c.N) {  // the first / last cell: the start / end vectors
                            const int sb = (d == 0 ? kHistStart : kHistEnd) + (int) c.model * 3;
                            if (pm > 0.0f) atomicAdd(ws + sb, pm);
                            if (px > 0.0f) atomicAdd(ws + sb + 1, px);
                            if (py > 0.0f) atomicAdd(ws + sb + 2, py);
                        }
                    }
                }
            }
            // u-values of d (emissions are zero outside the band); kept when the diagonal is off
            if (FLAT) {
                M::mul(gX, eX, bX);
                M::mul(gY, eY, bY);
                if (PAR) M::mul(gB, eM, bM); else M::mul(gA, eM, bM);
            } else {
                V ux[C], uy[C], um[C];
                M::mul(ux, eX, bX);
                M::mul(uy, eY, bY);
                M::mul(um, eM, bM);
#pragma unroll
                for (int j = 0; j < C; j++) {
                    gX[j] = on ? ux[j] : gX[j];
                    gY[j] = on ? uy[j] : gY[j];
                    if (PAR) gB[j] = on ? um[j] : gB[j]; else gA[j] = on ? um[j] : gA[j];
                }
            }
            if (!FLAT) {
                // moving below d crosses the window shift met when entering d
                const int backShift = on ? -inf.y : 0;
                if (__any_sync(FULL_MASK, backShift != 0)) {
                    laneShift<C, L, V>(gX, backShift, gl);
                    laneShift<C, L, V>(gY, backShift, gl);
                    laneShift<C, L, V>(gA, backShift, gl);
                    laneShift<C, L, V>(gB, backShift, gl);
                }
            }
        };
        const auto odd = std::integral_constant<int, 1>{};
        const auto even = std::integral_constant<int, 0>{};
        if (flat && __all_sync(FULL_MASK, dStart > wk.tbTo && dEnd < wk.D)) {
            pLim = wk.tbFrom - dStart;
            firstPost = min(K - 1, pLim);
            const int nPost = firstPost >= 0 ? firstPost + 1 : 0;
            refreshKK = nPost > untilRefresh ? firstPost - untilRefresh : -1;
            posts0 = posts;
#pragma unroll 1
            for (int k = K - 2; k >= 0; k -= 2) {
                back(odd, std::true_type{}, k + 1);
                back(even, std::true_type{}, k);
            }
            // post diagonals after the refresh are kk = refreshKK-1 .. 0
            untilRefresh = refreshKK >= 0 ? 9 - refreshKK : untilRefresh - nPost;
            posts += nPost;
        } else {
#pragma unroll 1
            for (int k = K - 2; k >= 0; k -= 2) {
                back(odd, std::false_type{}, k + 1);
                back(even, std::false_type{}, k);
            }
        }
        if constexpr (!ADJ) {
            __syncwarp();
            if (__any_sync(FULL_MASK, emitMask != 0)) emitBlock<C, L, K, V>(gl, gm, emitMask, dStart, o, thr);
        }
        // rescale the carried backward state at the block boundary
        {
            V m = V(0);
#pragma unroll
            for (int j = 0; j < C; j++) m = N::mx(m, N::mx(N::mx(gX[j], gY[j]), N::mx(gA[j], gB[j])));
            m = groupMaxNonNeg<L>(m);
            if (blockOn && m > V(0)) {
                const int kx = N::expOf(m);
                const V s = N::pow2(-kx);
                M::muls(gX, gX, s);
                M::muls(gY, gY, s);
                M::muls(gA, gA, s);
                M::muls(gB, gB, s);
                Eb += kx;
            }
        }
        if constexpr (ADJ) {
#pragma unroll
            for (int i = 0; i < 9; i++) accD[i] += (double) ta[i];
            // the warp's small histograms go to FP64 in global memory after every block
            __syncwarp();
            float *ws = reinterpret_cast<float *>(mpSmem + gm.whist);
            for (int i = gl; i < kHistSmall; i += 32) {
                const float v = ws[i];
                ws[i] = 0.0f;
                if (v != 0.0f) atomicAdd(expect + expectSlot(i), (double) v);
            }
        }
        __syncwarp();
    }
    if (llSet) logLik += llTm > V(0) ? log((double) llTm) + (double) llET * 0.69314718055994530942 : -INFINITY;
}

// Next traceback point of a group's task: the first anti-diagonal d in [from, N) whose band
// is at most 2*diagonalExpansion+1 cells wide (impl/pairwiseAligner.c:722-724), else N.
// Called by every lane of the warp; groups with `searching` false return N.
template <int L, class CT>
__device__ __forceinline__ int nextTracePoint(const CT &c, int from, int maxWidth, bool searching) {
    int D = c.N;
    int pos = from;
    bool look = searching && pos < c.N;
    while (__any_sync(FULL_MASK, look)) {
        const int d = pos + c.gl;
        bool ok = false;
        if (look && d < c.N) {
            const int2 bd = *reinterpret_cast<const int2 *>(c.band + d);
            ok = bd.y - bd.x + 1 <= maxWidth;
        }
        const unsigned bits = groupBits<L>(__ballot_sync(FULL_MASK, ok), c.g);
        if (look) {
            if (bits) {
                D = pos + __ffs(bits) - 1;
                look = false;
            } else {
                pos += L;
                look = pos < c.N;
            }
        }
    }
    return D;
}

// ---------------------------------------------------------------------------
// One warp-load of G tasks: forward sweep with checkpoints, then the walks.
// ---------------------------------------------------------------------------

template <int C, int L, int K, bool ADJ, class V, bool SW>
__device__ __forceinline__ void runGroup(const DpArgs &a, int taskIndex, GroupMem<C, L, K> &gm, const Scratch<V> &sc) {
    constexpr int S = L * C;
    constexpr int R = RingSize<S>::R;
    constexpr bool kSolo = L == 32;  // one task per warp: every lane is always on
    const int lane = threadIdx.x & 31;
    const bool has = taskIndex >= 0;
    const Task *tk = a.tasks + (has ? taskIndex : 0);
    TaskOut *to = a.out + (has ? taskIndex : 0);
    Ctx<V> c;
    c.gl = lane & (L - 1);
    c.g = lane / L;
    c.lx = has ? tk->lx : 0;
    c.ly = has ? tk->ly : 0;
    c.N = c.lx + c.ly;
    c.xs = a.xs + tk->xOff;
    c.ys = a.ys + tk->yOff;
    c.band = reinterpret_cast<const int4 *>(a.band) + tk->bandOff;
    const int flags = has ? tk->flags : 0;
    const int model = (flags & 4) ? 0 : 1;
    const DevModel &dm = a.models[model];
#pragma unroll
    for (int k = 0; k < 9; k++) c.t[k] = (V) dm.t[k];
    c.model = (uint32_t) model;
    c.repOff = kRepBase + (a.sharedRepeat ? 0u : (uint32_t) model * (uint32_t) (kRepTable * sizeof(float)));
    c.rle = dm.runLength;
    c.strandFwd = dm.strand;
    c.nTables = a.sharedRepeat ? 1 : 2;
    const int status0 = has ? to->status : 0;
    const bool tooLong = has && c.N / K + 1 > sc.blocks;
    const bool live = has && c.N > 0 && (status0 & kTaskBand) == 0 && !tooLong;
    if (has && !live && c.gl == 0) {
        to->count[0] = to->count[1] = to->count[2] = 0;
        to->logLik = 0.0;
        if (tooLong) to->status = status0 | kTaskScratch;
    }
    const int myN = live ? c.N : 0;
    const int Nmax = warpMaxInt(myN);
    if (Nmax <= 0) return;

    Out o;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        o.t[k] = a.outT[k] + tk->outOff[k];
        o.top[k] = tk->cap[k];
        o.written[k] = 0;
    }
    o.xShift = tk->x1 + tk->xShift;
    o.yShift = tk->y1;
    Walk wk;
    wk.startP = (flags & 1) ? dm.raggedStart : dm.start;
    double logLik = 0.0;
    bool bad = false;
    bool rangeBad = false;
    gm.rx.bad = 0;
    gm.ry.bad = 0;
    gm.rx.lo = 1 << 30;  // nothing resident
    gm.ry.lo = 1 << 30;

    // band records: 32-diagonal chunks through cp.async into the group's ring of 64
    auto issueChunk = [&](int chunk) {
#pragma unroll
        for (int q = c.gl; q < 32; q += L) {
            const int dd = chunk * 32 + q;
            if (live && dd <= myN) cpAsync16(gm.bandRing + ((dd & 63) << 4), &c.band[dd]);
        }
        cpAsyncCommit();
    };
    issueChunk(0);
    issueChunk(1);
    cpAsyncWaitAllButOne();
    __syncwarp();

    Fwd<C, V> st;
    Slots<C> sy;
    int Q = 0;
    if (live) {
        const int4 b0 = lds<int4>(gm.bandRing);
        Q = initialWindow<S>(b0.z, b0.w);
    }
    int Ef = 0;
    {
        // every group fills its rings once, so that every entry is a valid decoded symbol
        const int x0 = slotX0(0, Q);
        ringEnsure<R, L, true>(c, gm.rx, x0 - 1 - 8, x0 + S - 2, true, true);
        ringEnsure<R, L, false>(c, gm.ry, -x0 - S - 8, -x0 - 1, true, true);
        forwardOrigin<C, L, false, V>(c, wk.startP, Q, st, 0, 0);
        loadSlots<C, R>(c.gl, gm.rx, gm.ry, 0, Q, sy);
    }
    int checkAt = 1;
    // One anti-diagonal of the sweep; the parity is a compile-time constant, and the band
    // chunk and checkpoint boundaries (multiples of 32 and of K) fall on even diagonals.
    // One anti-diagonal with the window and ring checks (PAR = d & 1).
    auto checkedStep = [&](auto parity, int d) {
        constexpr int PAR = decltype(parity)::value;
        const bool on = kSolo || d <= myN;
        const int4 bd = lds<int4>(gm.bandRing + ((d & 63) << 4));
        const bool move = on && (bd.z < Q || bd.w > Q + S - 1);
        const bool rare = __any_sync(FULL_MASK, move || (on && d >= checkAt));
        bool reload = false;
        if (rare) {
            const int dl = move ? windowShift<C, S>(Q, bd.z, bd.w, bad) : 0;
            if (__any_sync(FULL_MASK, dl != 0)) {
                shiftFwd<C, L, V>(st, dl, c.gl);
                if (dl != 0) {
                    Q += C * dl;
                    reload = true;
                }
            }
            checkAt = ensureRings<R, L, S>(c, gm.rx, gm.ry, d, Q, true, on);
        }
        stepSlots<C, L, R, PAR>(c.gl, gm.rx, gm.ry, d, Q, sy);
        if (rare && reload) loadSlots<C, R>(c.gl, gm.rx, gm.ry, d, Q, sy);
        forwardDiagonal<C, L, PAR, false, false, V, SW>(c, st, sy, bd.x - Q, bd.y - Q, 0, 0);
    };
    const auto odd = std::integral_constant<int, 1>{};
    const auto even = std::integral_constant<int, 0>{};
    // diagonals 1 .. K-1
    for (int d = 1; d < K && d <= Nmax; d++) {
        if (d & 1) checkedStep(odd, d); else checkedStep(even, d);
    }
    // Checkpoint blocks [d0, d0+K-1]. A block where no group's window moves, no ring runs
    // out and every group is on runs without checks or branches, so the diagonals' symbol
    // and emission loads overlap the previous diagonals' arithmetic.
    for (int d0 = K; d0 <= Nmax; d0 += K) {
        if ((d0 & 31) == 0) {
            issueChunk((d0 >> 5) + 1);
            cpAsyncWaitAllButOne();
            __syncwarp();
        }
        Ef += rescaleFwd<C, L, V>(st);
        if (kSolo || d0 <= myN) {
            storeFwd<C, L, V>(sc.chk + (size_t) (d0 / K) * S, c.gl, st);
            if (c.gl == 0) sc.scal[d0 / K] = make_int2(Ef, Q);
        }
        const int dLast = d0 + K - 1;
        // A ring that would run out inside the block is refilled for the whole block now
        // (positions needed at d0 .. dLast in the current window: x0-1 .. x0'+S-2 and
        // y0-S .. y0'-1, at most S + K/2 + 1 entries), so that the block can run flat.
        if (__any_sync(FULL_MASK, dLast >= checkAt && dLast <= myN)) {
            const bool on = kSolo || dLast <= myN;
            const int xa = slotX0(d0, Q), xb = slotX0(dLast, Q);
            ringEnsure<R, L, true>(c, gm.rx, xa - 1, xb + S - 2, true, on);
            ringEnsure<R, L, false>(c, gm.ry, d0 - xa - S, dLast - xb - 1, true, on);
            checkAt = ensureRings<R, L, S>(c, gm.rx, gm.ry, d0, Q, true, on);
        }
        bool clear = dLast <= myN && dLast < checkAt;
        if (c.gl < K) {
            const int4 bd = lds<int4>(gm.bandRing + (((d0 + c.gl) & 63) << 4));
            clear = clear && bd.z >= Q && bd.w <= Q + S - 1;
        }
        if (__all_sync(FULL_MASK, clear)) {
            // pairs (even, odd): one small loop body keeps the hot code in the instruction cache
#pragma unroll 1
            for (int d = d0; d < d0 + K; d += 2) {
                const int2 b0 = lds<int2>(gm.bandRing + ((d & 63) << 4));
                const int2 b1 = lds<int2>(gm.bandRing + (((d + 1) & 63) << 4));
                stepSlots<C, L, R, 0>(c.gl, gm.rx, gm.ry, d, Q, sy);
                forwardDiagonal<C, L, 0, false, false, V, SW>(c, st, sy, b0.x - Q, b0.y - Q, 0, 0);
                stepSlots<C, L, R, 1>(c.gl, gm.rx, gm.ry, d + 1, Q, sy);
                forwardDiagonal<C, L, 1, false, false, V, SW>(c, st, sy, b1.x - Q, b1.y - Q, 0, 0);
            }
        } else {
            for (int kk = 0; kk < K; kk += 2) {
                if (d0 + kk > Nmax) break;
                checkedStep(even, d0 + kk);
                if (d0 + kk + 1 > Nmax) break;
                checkedStep(odd, d0 + kk + 1);
            }
        }
    }
    // drain the band prefetch groups before the ring is reused
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();

    // Traceback segments in the reference's order: an intermediate point D is the first
    // anti-diagonal after the previous point with D >= tracedBackTo + minDiagsBetweenTraceBack
    // and a narrow band; its posteriors cover (tracedBackTo, D - traceBackDiagonals - 1].
    // The last segment ends at N and covers (tracedBackTo, N]. The likelihood-only mode
    // (computeForwardProbability) walks just the top diagonal; the adjoint walks the whole
    // lattice at once (no segments: the gradient of the full forward total).
    const bool fwdOnly = (flags & kFlagForwardOnly) != 0;
    const bool single = ADJ || fwdOnly;
    const int maxWidth = 2 * a.diagonalExpansion + 1;
    int prevD = 0, tb = 0;
    bool more = live;
    double accD[9];
#pragma unroll
    for (int i = 0; i < 9; i++) accD[i] = 0.0;
    while (__any_sync(FULL_MASK, more)) {
        const int from = max(prevD + 1, tb + a.minDiagsBetweenTraceBack);
        const int D = single ? c.N : nextTracePoint<L>(c, from, maxWidth, more && !single);
        const bool atEnd = D >= c.N;
        wk.D = c.N < D ? c.N : D;
        wk.tbTo = ADJ ? -1 : (fwdOnly ? c.N - 1 : tb);
        wk.tbFrom = atEnd ? wk.D : wk.D - (a.traceBackDiagonals + 1);
        wk.atEnd = atEnd ? 1 : 0;
        wk.active = more ? 1 : 0;
        wk.emit = single ? 0 : 1;
        wk.endP = (atEnd && (flags & 2)) ? dm.raggedEnd : dm.end;
        walkSegment<C, L, K, ADJ, V, SW>(c, gm, sc, wk, (V) a.threshold, o, logLik, bad, rangeBad, accD, a.expect);
        if (more) {
            tb = wk.tbFrom;
            prevD = wk.D;
            more = !atEnd;
        }
    }
    if constexpr (ADJ) {
        // transition sums of the task (FP64 warp reduction), then the repeat histograms
#pragma unroll
        for (int i = 0; i < 9; i++) {
            double v = accD[i];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(FULL_MASK, v, off);
            if (lane == 0 && live && !bad && v != 0.0)
                atomicAdd(a.expect + (size_t) model * kExpPerModel + kExpTrans + i, v);
        }
        float *hr = reinterpret_cast<float *>(mpSmem + gm.hist) + kHistSmall;
        for (int i = lane; i < c.nTables * kRepTable; i += 32) {
            const float v = atomicExch(hr + i, 0.0f);
            if (v != 0.0f) atomicAdd(a.expectRep + i, (double) v);
        }
    }
    if (live && c.gl == 0) {
        int s = status0;
        if (bad) s |= kTaskWindow;
        if (rangeBad) s |= kTaskRange;
        if (gm.rx.bad | gm.ry.bad) s |= kTaskSymbol;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            to->count[k] = bad ? 0 : o.written[k];
            if (!bad && o.written[k] > o.top[k]) s |= kTaskCapacity;
        }
        to->status = s;
        to->logLik = logLik;
    }
}

template <int C, int L, int K, int MAXW, bool ADJ, class V, bool SW>
__global__ void __launch_bounds__(MAXW * 32, 1) posteriorKernel(DpArgs a) {
    using GS = GroupSmem<C, L, K, ADJ, V>;
    constexpr int G = 32 / L;
    constexpr int R = RingSize<L * C>::R;
    const int nTables = a.sharedRepeat ? 1 : 2;
    float *sm = reinterpret_cast<float *>(mpSmem + kMatchOff);
    float *gx = reinterpret_cast<float *>(mpSmem + kGapXOff);
    float *gy = reinterpret_cast<float *>(mpSmem + kGapYOff);
    float *rp = reinterpret_cast<float *>(mpSmem + kRepBase);
    for (int i = threadIdx.x; i < nTables * kRepTable; i += blockDim.x) rp[i] = a.repeatProb[i];
    for (int i = threadIdx.x; i < 2 * 25; i += blockDim.x) sm[i] = a.models[i / 25].match[i % 25];
    for (int i = threadIdx.x; i < 2 * 5; i += blockDim.x) {
        gx[i] = a.models[i / 5].gapX[i % 5];
        gy[i] = a.models[i / 5].gapY[i % 5];
    }
    const uint32_t histOff = (uint32_t) tableBytes(nTables);
    if (ADJ) {
        float *h = reinterpret_cast<float *>(mpSmem + histOff);
        for (int i = threadIdx.x; i < kHistSmall + nTables * kRepTable; i += blockDim.x) h[i] = 0.0f;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int g = lane / L;
    const int gwarp = blockIdx.x * (blockDim.x >> 5) + warp;
    const uint32_t mine = histOff + (ADJ ? (uint32_t) histBytes(nTables) : 0u) + (uint32_t) ((warp * G + g) * GS::bytes);
    GroupMem<C, L, K> gm;
    gm.rx = Ring<R>{mine, 0, 0};
    gm.ry = Ring<R>{mine + (uint32_t) (R * sizeof(uint2)), 0, 0};
    gm.bandRing = mine + (uint32_t) GS::ringBytes;
    gm.walkBand = gm.bandRing + (uint32_t) GS::bandRingBytes;
    gm.cacheA = gm.walkBand + (uint32_t) GS::walkBandBytes;
    gm.cacheB = gm.cacheA + (uint32_t) GS::cacheABytes;
    gm.cacheC = gm.cacheB + (uint32_t) GS::cacheBBytes;
    gm.info = gm.cacheC + (uint32_t) GS::cacheCBytes;
    gm.hist = histOff;
    gm.whist = gm.info + (uint32_t) GS::infoBytes;
    if (ADJ) {
        float *w = reinterpret_cast<float *>(mpSmem + gm.whist);
        for (int i = lane; i < kHistSmall; i += 32) w[i] = 0.0f;
        __syncwarp();
    }
    Scratch<V> sc;
    sc.blocks = a.scratchBlocks;
    const size_t slot = (size_t) gwarp * G + g;  // one checkpoint area per task slot
    sc.chk = reinterpret_cast<typename Num<V>::V4 *>(a.scratch) + slot * a.scratchBlocks * (size_t) (C * L);
    sc.scal = a.scratchScalars + slot * a.scratchBlocks;

    const int nLoads = (a.nTasks + G - 1) / G;
    while (true) {
        int q = 0;
        if (lane == 0) q = atomicAdd(a.queue, 1);
        q = __shfl_sync(FULL_MASK, q, 0);
        if (q >= nLoads) break;
        const int t = q * G + g;
        runGroup<C, L, K, ADJ, V, SW>(a, t < a.nTasks ? a.order[t] : -1, gm, sc);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------


template <int C, int L, int K, bool ADJ = false, class V = float>
static size_t smemFor(int warps, int nTables) {
    return tableBytes(nTables) + (ADJ ? histBytes(nTables) : 0) +
           (size_t) warps * (32 / L) * GroupSmem<C, L, K, ADJ, V>::bytes;
}

template <int C, int L, int K, int MAXW, bool ADJ, class V, bool SW>
static cudaError_t launchSW(const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    const size_t smem = smemFor<C, L, K, ADJ, V>(warps, a.sharedRepeat ? 1 : 2);
    // the shared-memory limit of the kernel only grows, once per device (calls from many threads
    // then skip the attribute call)
    static std::mutex lock;
    static size_t granted[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> g(lock);
        const int slot = dev & 63;
        if (smem > granted[slot]) {
            e = cudaFuncSetAttribute(posteriorKernel<C, L, K, MAXW, ADJ, V, SW>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            if (e == cudaSuccess) granted[slot] = smem;
        }
    }
    if (e != cudaSuccess) return e;
    posteriorKernel<C, L, K, MAXW, ADJ, V, SW><<<blocks, warps * 32, smem, s>>>(a);
    return cudaGetLastError();
}

// The FP32 posterior variants come in two builds: with the switch transitions, and without them
// for models whose switch transitions are zero (the shipped model's); the FP64 variants and the
// adjoint always carry them.
template <int C, int L, int K, int MAXW, bool ADJ = false, class V = float>
static cudaError_t launchT(const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    if (warps > MAXW || warps < 1) return cudaErrorInvalidValue;
    if constexpr (!ADJ && std::is_same<V, float>::value) {
        if (a.noSwitch) return launchSW<C, L, K, MAXW, ADJ, V, false>(a, blocks, warps, s);
    }
    return launchSW<C, L, K, MAXW, ADJ, V, true>(a, blocks, warps, s);
}

// Kernel variants: (index, C slots per lane, L lanes per task, K checkpoint stride,
// maximum warps per block = launch bound, arithmetic type). The window is S = L*C slots,
// a warp carries 32/L tasks and a task fits when its band hull spans at most S - 2C slots.
// Variants 0-6 and 12 compute in FP32, 7-11 in FP64 (same schedule; for the sub-problems whose
// range FP32 cannot hold, and for the likelihood-only mode). Variant 12 trades a shorter
// checkpoint stride for more resident warps (an autotuner candidate).
#define MP_VARIANTS(X)            \
    X(0, 2, 32, 8, 12, float)     \
    X(1, 4, 16, 4, 8, float)      \
    X(2, 8, 8, 4, 5, float)       \
    X(3, 3, 32, 8, 8, float)      \
    X(4, 4, 32, 4, 8, float)      \
    X(5, 6, 32, 4, 8, float)      \
    X(6, 8, 32, 4, 5, float)      \
    X(7, 2, 32, 8, 6, double)     \
    X(8, 3, 32, 8, 4, double)     \
    X(9, 4, 32, 4, 6, double)     \
    X(10, 6, 32, 4, 4, double)    \
    X(11, 8, 32, 4, 3, double)    \
    X(12, 2, 32, 4, 16, float)

// Adjoint variants (one task per warp; the block also holds the expected-count histograms).
#define MP_ADJ_VARIANTS(X) \
    X(0, 2, 32, 8, 8)      \
    X(1, 3, 32, 8, 4)      \
    X(2, 4, 32, 4, 6)

int variantCount() {
    return 13;
}

bool variantIsF64(int v) {
    switch (v) {
#define MP_F64(i, c_, l_, k_, w_, t_) \
    case i: return sizeof(t_) == 8;
        MP_VARIANTS(MP_F64)
#undef MP_F64
        default: return false;
    }
}

bool variantShape(int v, int *C, int *L, int *K) {
    switch (v) {
#define MP_SHAPE(i, c_, l_, k_, w_, t_) \
    case i: *C = c_; *L = l_; *K = k_; return true;
        MP_VARIANTS(MP_SHAPE)
#undef MP_SHAPE
        default: return false;
    }
}

// As many warps as the kernel's bound and 227 KB of shared memory per block allow (0: none).
int variantMaxWarps(int v, int nTables) {
    const size_t limit = 227 * 1024;
    switch (v) {
#define MP_MAXW(i, c_, l_, k_, w_, t_)                                             \
    case i: {                                                                      \
        int w = w_;                                                                \
        while (w > 1 && smemFor<c_, l_, k_, false, t_>(w, nTables) > limit) w--;   \
        return smemFor<c_, l_, k_, false, t_>(w, nTables) > limit ? 0 : w;         \
    }
        MP_VARIANTS(MP_MAXW)
#undef MP_MAXW
        default: return 0;
    }
}

cudaError_t launchVariant(int v, const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    switch (v) {
#define MP_LAUNCH(i, c_, l_, k_, w_, t_) \
    case i: return launchT<c_, l_, k_, w_, false, t_>(a, blocks, warps, s);
        MP_VARIANTS(MP_LAUNCH)
#undef MP_LAUNCH
        default: return cudaErrorInvalidValue;
    }
}

int adjointVariantCount() {
    return 3;
}

bool adjointVariantShape(int v, int *C, int *L, int *K) {
    switch (v) {
#define MP_SHAPE(i, c_, l_, k_, w_) \
    case i: *C = c_; *L = l_; *K = k_; return true;
        MP_ADJ_VARIANTS(MP_SHAPE)
#undef MP_SHAPE
        default: return false;
    }
}

int adjointVariantMaxWarps(int v, int nTables) {
    const size_t limit = 227 * 1024;
    switch (v) {
#define MP_MAXW(i, c_, l_, k_, w_)                                                \
    case i: {                                                                     \
        int w = w_;                                                               \
        while (w > 1 && smemFor<c_, l_, k_, true>(w, nTables) > limit) w--;       \
        return smemFor<c_, l_, k_, true>(w, nTables) > limit ? 0 : w;             \
    }
        MP_ADJ_VARIANTS(MP_MAXW)
#undef MP_MAXW
        default: return 0;
    }
}

cudaError_t launchAdjointVariant(int v, const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    switch (v) {
#define MP_LAUNCH(i, c_, l_, k_, w_) \
    case i: return launchT<c_, l_, k_, w_, true, float>(a, blocks, warps, s);
        MP_ADJ_VARIANTS(MP_LAUNCH)
#undef MP_LAUNCH
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mp
