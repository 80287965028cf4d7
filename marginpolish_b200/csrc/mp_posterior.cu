// Posterior kernel of the realignment engine (sm_100a).
//
// Hot path: the anchored, banded 3-state pair-HMM forward / backward /
// posterior pass of MarginPolish (getPosteriorProbsWithBanding,
// impl/pairwiseAligner.c:687-808, over the split rectangles of :942-991; cell
// recurrence impl/stateMachine.c:559-581; posterior rules
// impl/pairwiseAligner.c:586-664), re-designed for one warp per banded
// sub-problem ("task"), persistent, fed from a length-sorted queue:
//
//  * The cells of anti-diagonal d live in a window of S = 32*C slots, C
//    consecutive slots per lane; slot i holds x-y = 2(Q+i) + (d&1). The
//    window origin Q moves only by whole lanes, when the 5-diagonal band hull
//    leaves it, so the exchange between diagonals is one shuffle per lane.
//  * FP32 probabilities (not logs), in push form: each cell sends its three
//    outgoing sums (to gap-x, gap-y and match successors); the receiving
//    cell multiplies by its emission. Emissions are zeroed outside the band,
//    which also masks every product built on them. Values are rescaled by
//    exact powers of two every K diagonals and the integer exponents are
//    tracked per block, so no log / exp is evaluated per cell; the FP64
//    log-likelihood is ln(mantissa) + exponent*ln2 once per segment.
//  * The forward sweep stores one float4 per slot every K diagonals (the
//    checkpoint: outgoing gap sums of d-1 and match sums of d-1, d-2). A
//    traceback walk (at the end, or at the reference's intermediate traceback
//    points) recomputes each block of K diagonals into shared memory and runs
//    the backward recurrence and the posteriors over it, top block first,
//    prefetching the next block's checkpoint and band records into registers.
//  * Posterior tuples are ranked in the warp (packed prefix sum) and written
//    from the top of the task's output region downwards: the region then
//    reads in the reference's order (ascending anti-diagonal, descending x-y,
//    later traceback segments first).
#include "mp_internal.h"

#include <algorithm>
#include <cstdint>

namespace mp {

#define FULL_MASK 0xffffffffu

template <int C>
struct Geo {
    static constexpr int S = 32 * C;
    static constexpr int R = (S + 64 <= 128) ? 128 : ((S + 64 <= 256) ? 256 : 512);
};

__device__ __forceinline__ float pow2f(int k) {  // 2^k, k in [-126, 127]
    return __int_as_float((127 + k) << 23);
}

__device__ __forceinline__ int exponentOf(float m) {  // floor(log2 m) for normal m
    return ((__float_as_int(m) >> 23) & 0xff) - 127;
}

__device__ __forceinline__ float warpMax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

__device__ __forceinline__ float warpSum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ void cpAsync16(void *smem, const void *gmem) {
    unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cpAsyncCommit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void cpAsyncWaitAllButOne() {
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Task context (uniform over the warp)
// ---------------------------------------------------------------------------

struct Ctx {
    int lane;
    int lx, ly, N;
    const uint16_t *xs;
    const uint16_t *ys;
    const int4 *band;       // (xmyL, xmyR, hullL, hullR) of d = 0..N
    float t[9];
    const char *rp;         // shared repeat-probability table of the task's model
    const float *sm;        // shared match table [25] of the model
    const float *gx;        // shared gap-x [5]
    const float *gy;        // shared gap-y [5]
    int rle;
    int strandFwd;
};

// Decoded symbols: packed (repeat-table byte offset | match-table byte offset << 17) and gap emission.
__device__ __forceinline__ uint2 decodeX(const Ctx &c, int pos, int &bad) {
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
    uint32_t pk = (uint32_t) ((row * (kMaxRepeat * kMaxRepeat) + rc * kMaxRepeat) * 4) | ((uint32_t) (b * 20) << 17);
    return make_uint2(pk, __float_as_uint(c.gx[b]));
}

__device__ __forceinline__ uint2 decodeY(const Ctx &c, int pos, int &bad) {
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
    return make_uint2(pk, __float_as_uint(c.gy[b]));
}

__device__ __forceinline__ float matchEmission(const Ctx &c, uint32_t xpk, uint32_t ypk) {
    uint32_t s = xpk + ypk;
    float r = *reinterpret_cast<const float *>(c.rp + (s & 0x1ffffu));
    float m = *reinterpret_cast<const float *>(reinterpret_cast<const char *>(c.sm) + (s >> 17));
    return r * m;
}

// Decoded symbols of a span of positions in shared memory (one ring per sequence).
template <int R>
struct Ring {
    uint2 *buf;
    int lo;
    int bad;
};

// Decodes positions [newLo, newLo+R) into the ring; returns 1 if a symbol was out of range.
template <int R, bool IS_X>
__device__ __noinline__ int ringFillRaw(Ctx c, uint2 *buf, int newLo) {
    int bad = 0;
#pragma unroll 4
    for (int k = 0; k < R / 32; k++) {
        int p = newLo + k * 32 + c.lane;
        buf[p & (R - 1)] = IS_X ? decodeX(c, p, bad) : decodeY(c, p, bad);
    }
    bad = __any_sync(FULL_MASK, bad) ? 1 : 0;
    __syncwarp();
    return bad;
}

template <int R, bool IS_X>
__device__ __forceinline__ void ringFill(const Ctx &c, Ring<R> &r, int newLo) {
    r.lo = newLo;
    r.bad |= ringFillRaw<R, IS_X>(c, r.buf, newLo);
}

template <int R, bool IS_X>
__device__ __forceinline__ void ringEnsure(const Ctx &c, Ring<R> &r, int needLo, int needHi, bool up) {
    if (needLo < r.lo || needHi >= r.lo + R) {
        int slack = R - (needHi - needLo + 1);
        ringFill<R, IS_X>(c, r, up ? needLo - slack / 8 : needLo - (slack - slack / 8));
    }
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
__device__ __forceinline__ void loadSlots(const Ctx &c, const Ring<R> &rx, const Ring<R> &ry, int d, int Q,
                                          Slots<C> &s) {
    int x0 = slotX0(d, Q), y0 = d - x0;
#pragma unroll
    for (int j = 0; j < C; j++) {
        int i = c.lane * C + j;
        uint2 vx = rx.buf[(x0 + i - 1) & (R - 1)];
        uint2 vy = ry.buf[(y0 - i - 1) & (R - 1)];
        s.xpk[j] = vx.x;
        s.ex[j] = __uint_as_float(vx.y);
        s.ypk[j] = vy.x;
        s.ey[j] = __uint_as_float(vy.y);
    }
}

// Slot symbols from diagonal d-1 to d (window unchanged): entering odd d the x of
// every slot grows by one, entering even d the y of every slot grows by one.
template <int C, int R, int PAR>
__device__ __forceinline__ void stepSlots(const Ctx &c, const Ring<R> &rx, const Ring<R> &ry, int d, int Q,
                                          Slots<C> &s) {
    constexpr int S = 32 * C;
    if (PAR) {
        uint2 fresh = rx.buf[(slotX0(d, Q) + S - 2) & (R - 1)];
        uint32_t npk = __shfl_down_sync(FULL_MASK, s.xpk[0], 1);
        float ne = __shfl_down_sync(FULL_MASK, s.ex[0], 1);
        if (c.lane == 31) {
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
        uint2 fresh = ry.buf[(d - slotX0(d, Q) - 1) & (R - 1)];
        uint32_t npk = __shfl_up_sync(FULL_MASK, s.ypk[C - 1], 1);
        float ne = __shfl_up_sync(FULL_MASK, s.ey[C - 1], 1);
        if (c.lane == 0) {
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

// Forward state between diagonals: outgoing gap-x / gap-y sums of d-1 and
// outgoing match sums of d-1 and d-2 (even diagonals own mA, odd own mB).
template <int C>
struct Fwd {
    float ox[C], oy[C], mA[C], mB[C];
};

// New lane l takes old lane l+dl (values leaving the warp become zero).
template <int C>
__device__ __forceinline__ void laneShift(float (&v)[C], int dl, int lane) {
    int src = lane + dl;
    bool ok = src >= 0 && src < 32;
#pragma unroll
    for (int j = 0; j < C; j++) {
        float w = __shfl_sync(FULL_MASK, v[j], src & 31);
        v[j] = ok ? w : 0.0f;
    }
}

template <int C>
__device__ __forceinline__ void shiftFwd(Fwd<C> &f, int dl, int lane) {
    laneShift<C>(f.ox, dl, lane);
    laneShift<C>(f.oy, dl, lane);
    laneShift<C>(f.mA, dl, lane);
    laneShift<C>(f.mB, dl, lane);
}

// The window must contain the hull of the bands of d-2..d+2; returns the lane
// shift (new Q = Q + C*shift). Shared by the sweep and the recompute, so both
// take the same decisions. Sets *bad when the hull does not fit the class.
template <int C>
__device__ __forceinline__ int windowShift(int Q, int hullLo, int hullHi, bool &bad) {
    constexpr int S = 32 * C;
    int needLo = hullLo >> 1, needHi = hullHi >> 1;
    if (needLo >= Q && needHi <= Q + S - 1) return 0;
    int span = needHi - needLo + 1;
    if (span > S - 2 * C) {
        bad = true;
        return 0;
    }
    int diff = needLo - (S - span) / 2 - Q;
    int dl = diff >= 0 ? diff / C : -((-diff + C - 1) / C);
    if (Q + C * dl + S - 1 < needHi) dl++;
    if (Q + C * dl > needLo) bad = true;
    return dl;
}

template <int C>
__device__ __forceinline__ int initialWindow(int hullLo, int hullHi) {
    constexpr int S = 32 * C;
    int needLo = hullLo >> 1, needHi = hullHi >> 1;
    return needLo - (S - (needHi - needLo + 1)) / 2;
}

// One forward anti-diagonal (PAR = d & 1). Emissions are zeroed outside the band
// [sLo, sHi], which zeroes the cell. With CACHE, the cell values and the masked
// emissions are written to the block cache (slot-major, lane-minor).
template <int C, int PAR, bool CACHE>
__device__ __forceinline__ void forwardDiagonal(const Ctx &c, Fwd<C> &st, const Slots<C> &sy, int sLo, int sHi,
                                                float4 *cacheA, float2 *cacheB) {
    float inX[C], inY[C];
    if (PAR) {  // odd d: gap-x source slot i, gap-y source slot i+1
        float nb = __shfl_down_sync(FULL_MASK, st.oy[0], 1);
        if (c.lane == 31) nb = 0.0f;
#pragma unroll
        for (int j = 0; j < C; j++) {
            inX[j] = st.ox[j];
            inY[j] = (j < C - 1) ? st.oy[j + 1] : nb;
        }
    } else {  // even d: gap-x source slot i-1, gap-y source slot i
        float nb = __shfl_up_sync(FULL_MASK, st.ox[C - 1], 1);
        if (c.lane == 0) nb = 0.0f;
#pragma unroll
        for (int j = 0; j < C; j++) {
            inX[j] = (j > 0) ? st.ox[j - 1] : nb;
            inY[j] = st.oy[j];
        }
    }
    const int base = c.lane * C - sLo;
    const unsigned span = (unsigned) (sHi - sLo);
#pragma unroll
    for (int j = 0; j < C; j++) {
        const bool in = (unsigned) (base + j) <= span;
        const float eM = in ? matchEmission(c, sy.xpk[j], sy.ypk[j]) : 0.0f;
        const float eX = in ? sy.ex[j] : 0.0f;
        const float eY = in ? sy.ey[j] : 0.0f;
        const float fM = eM * (PAR ? st.mB[j] : st.mA[j]);
        const float fX = eX * inX[j];
        const float fY = eY * inY[j];
        const float nm = __fmaf_rn(c.t[2 * 3 + 0], fY, __fmaf_rn(c.t[1 * 3 + 0], fX, c.t[0 * 3 + 0] * fM));
        const float nx = __fmaf_rn(c.t[2 * 3 + 1], fY, __fmaf_rn(c.t[1 * 3 + 1], fX, c.t[0 * 3 + 1] * fM));
        const float ny = __fmaf_rn(c.t[1 * 3 + 2], fX, __fmaf_rn(c.t[2 * 3 + 2], fY, c.t[0 * 3 + 2] * fM));
        if (PAR) st.mB[j] = nm; else st.mA[j] = nm;
        st.ox[j] = nx;
        st.oy[j] = ny;
        if (CACHE) {
            cacheA[j * 32 + c.lane] = make_float4(fM, fX, fY, eM);
            cacheB[j * 32 + c.lane] = make_float2(eX, eY);
        }
    }
}

// Diagonal 0: the start cell (x-y = 0) holds the start (or ragged-start) probabilities.
template <int C, bool CACHE>
__device__ __forceinline__ void forwardOrigin(const Ctx &c, const float *startP, int Q, Fwd<C> &st, float4 *cacheA,
                                              float2 *cacheB) {
#pragma unroll
    for (int j = 0; j < C; j++) {
        const bool here = c.lane * C + j == -Q;
        const float fM = here ? startP[0] : 0.0f;
        const float fX = here ? startP[1] : 0.0f;
        const float fY = here ? startP[2] : 0.0f;
        st.mA[j] = __fmaf_rn(c.t[2 * 3 + 0], fY, __fmaf_rn(c.t[1 * 3 + 0], fX, c.t[0 * 3 + 0] * fM));
        st.ox[j] = __fmaf_rn(c.t[2 * 3 + 1], fY, __fmaf_rn(c.t[1 * 3 + 1], fX, c.t[0 * 3 + 1] * fM));
        st.oy[j] = __fmaf_rn(c.t[1 * 3 + 2], fX, __fmaf_rn(c.t[2 * 3 + 2], fY, c.t[0 * 3 + 2] * fM));
        st.mB[j] = 0.0f;
        if (CACHE) {
            cacheA[j * 32 + c.lane] = make_float4(fM, fX, fY, 0.0f);
            cacheB[j * 32 + c.lane] = make_float2(0.0f, 0.0f);
        }
    }
}

template <int C>
__device__ __forceinline__ int rescaleFwd(Fwd<C> &st) {
    float m = 0.0f;
#pragma unroll
    for (int j = 0; j < C; j++) m = fmaxf(m, fmaxf(fmaxf(st.ox[j], st.oy[j]), fmaxf(st.mA[j], st.mB[j])));
    m = warpMax(m);
    if (!(m > 0.0f)) return 0;
    const int k = exponentOf(m);
    const float sc = pow2f(-k);
#pragma unroll
    for (int j = 0; j < C; j++) {
        st.ox[j] *= sc;
        st.oy[j] *= sc;
        st.mA[j] *= sc;
        st.mB[j] *= sc;
    }
    return k;
}

// ---------------------------------------------------------------------------
// Output: ordered warp compaction of one diagonal's tuples.
// ---------------------------------------------------------------------------

struct Out {
    int32_t *w[3];
    int32_t *x[3];
    int32_t *y[3];
    int top[3];
    int written[3];
    int xShift, yShift;
};

template <int C>
__device__ __forceinline__ void emitDiagonal(int lane, Out &o, const float (&p)[3][C], float thr, int x0, int d) {
    uint32_t mask = 0;  // bit k*C+j: list k, slot j
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int j = 0; j < C; j++) mask |= (p[k][j] >= thr ? 1u : 0u) << (k * C + j);
    }
    if (__ballot_sync(FULL_MASK, mask != 0) == 0) return;
    constexpr uint32_t listBits = (1u << C) - 1u;
    const uint32_t cnt = (uint32_t) __popc(mask & listBits) | ((uint32_t) __popc(mask & (listBits << C)) << 10) |
                         ((uint32_t) __popc(mask & (listBits << (2 * C))) << 20);
    uint32_t incl = cnt;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t v = __shfl_up_sync(FULL_MASK, incl, off);
        if (lane >= off) incl += v;
    }
    const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    uint32_t rank = incl - cnt;  // packed exclusive ranks, advanced as this lane writes
    while (mask) {
        const int bit = __ffs(mask) - 1;
        mask &= mask - 1;
        const int k = bit / C, j = bit - k * C;
        const int r = o.written[k] + (int) ((rank >> (10 * k)) & 1023u);
        rank += 1u << (10 * k);
        const int pos = o.top[k] - 1 - r;
        if (pos >= 0) {
            const int x = x0 + lane * C + j;
            float v = 0.0f;
#pragma unroll
            for (int kk = 0; kk < 3; kk++) {
#pragma unroll
                for (int jj = 0; jj < C; jj++) v = bit == kk * C + jj ? p[kk][jj] : v;
            }
            v = fminf(v, 1.0f);
            o.w[k][pos] = (int32_t) floorf(v * (float) kProbOne);
            o.x[k][pos] = x - 1 + o.xShift;
            o.y[k][pos] = d - x - 1 + o.yShift;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) o.written[k] += (int) ((total >> (10 * k)) & 1023u);
}

// ---------------------------------------------------------------------------
// Per-warp shared workspace
// ---------------------------------------------------------------------------

template <int C, int K>
struct WarpSmem {
    static constexpr int R = Geo<C>::R;
    static constexpr size_t ringBytes = 2 * R * sizeof(uint2);
    static constexpr size_t bandRingBytes = 64 * sizeof(int4);
    static constexpr size_t walkBandBytes = K * sizeof(int4);
    static constexpr size_t cacheABytes = (size_t) K * C * 32 * sizeof(float4);
    static constexpr size_t cacheBBytes = (size_t) K * C * 32 * sizeof(float2);
    static constexpr size_t infoBytes = K * sizeof(int2);
    static constexpr size_t bytes = ringBytes + bandRingBytes + walkBandBytes + cacheABytes + cacheBBytes + infoBytes;
};

struct Scratch {
    float4 *chk;      // checkpoints of this warp: [block][C][32]
    int2 *scal;       // (exponent, window) per checkpoint
    float4 *resume;   // sweep state across an intermediate walk
    int blocks;
};

template <int C, int K>
struct WarpMem {
    Ring<Geo<C>::R> rx, ry;
    int4 *bandRing;
    int4 *walkBand;
    float4 *cacheA;
    float2 *cacheB;
    int2 *info;
};

template <int C>
__device__ __forceinline__ void storeFwd(float4 *p, int lane, const Fwd<C> &st) {
#pragma unroll
    for (int j = 0; j < C; j++) p[j * 32 + lane] = make_float4(st.ox[j], st.oy[j], st.mA[j], st.mB[j]);
}

template <int C>
__device__ __forceinline__ void loadFwd(const float4 (&v)[C], Fwd<C> &st) {
#pragma unroll
    for (int j = 0; j < C; j++) {
        st.ox[j] = v[j].x;
        st.oy[j] = v[j].y;
        st.mA[j] = v[j].z;
        st.mB[j] = v[j].w;
    }
}

// ---------------------------------------------------------------------------
// Traceback walk over (tbTo, D]: recompute each block of K diagonals into the
// shared cache, then the backward recurrence and posteriors over it.
// ---------------------------------------------------------------------------

struct WalkArgs {
    int D, tbTo, tbFrom, atEnd;
    const float *startP;
    const float *endP;
    float thr;
};

template <int C, int K>
__device__ __forceinline__ void walkSegment(const Ctx &c, WarpMem<C, K> &wm, const Scratch &sc, const WalkArgs &wa,
                                            Out &o, double &logLik, bool &bad) {
    constexpr int S = 32 * C;
    constexpr int R = Geo<C>::R;
    const int lane = c.lane;
    int untilRefresh = 0;
    float gX[C], gY[C], gA[C], gB[C];  // backward u-values: gap-x / gap-y of d+1, match (even d in A, odd in B)
#pragma unroll
    for (int j = 0; j < C; j++) gX[j] = gY[j] = gA[j] = gB[j] = 0.0f;
    int Eb = 0, posts = 0, ET = 0;
    float Tm = 0.0f;
    const int D = wa.D;
    const int bTop = D / K, bBot = (wa.tbTo + 1) / K;

    // register prefetch of a block's checkpoint and band records
    float4 pchk[C];
    int2 pscal = make_int2(0, 0);
    int4 pband = make_int4(0, 0, 0, 0);
    auto prefetch = [&](int b) {
        if (b > 0) {
#pragma unroll
            for (int j = 0; j < C; j++) pchk[j] = sc.chk[((size_t) b * C + j) * 32 + lane];
            pscal = sc.scal[b];
        }
        const int dd = b * K + lane;
        if (lane < K && dd <= c.N) pband = c.band[dd];
    };
    prefetch(bTop);

    for (int b = bTop; b >= bBot; b--) {
        const int dStart = b * K;
        const int dEnd = min(dStart + K - 1, D);
        Fwd<C> rs;
        float4 cchk[C];
#pragma unroll
        for (int j = 0; j < C; j++) cchk[j] = pchk[j];
        const int2 cscal = pscal;
        if (lane < K) wm.walkBand[lane] = pband;
        __syncwarp();
        if (b > bBot) prefetch(b - 1);

        // ---------------- recompute the block ----------------
        int Q, Ef;
        float chkSM[C];
        if (b == 0) {
            const int4 b0 = wm.walkBand[0];
            Q = initialWindow<C>(b0.z, b0.w);
            Ef = 0;
#pragma unroll
            for (int j = 0; j < C; j++) chkSM[j] = 0.0f;
        } else {
            loadFwd<C>(cchk, rs);
            Ef = cscal.x;
            Q = cscal.y;
#pragma unroll
            for (int j = 0; j < C; j++) chkSM[j] = rs.mB[j];
        }
        Slots<C> sy;
        bool have = false;
        for (int k = 0; k <= dEnd - dStart; k++) {
            const int d = dStart + k;
            const int4 bd = wm.walkBand[k];
            int dl = 0;
            if (d == 0) {
                int x0 = slotX0(0, Q);
                ringEnsure<R, true>(c, wm.rx, x0 - 1, x0 + S - 2, false);
                ringEnsure<R, false>(c, wm.ry, -x0 - S, -x0 - 1, false);
                loadSlots<C, R>(c, wm.rx, wm.ry, 0, Q, sy);
                have = true;
                forwardOrigin<C, true>(c, wa.startP, Q, rs, wm.cacheA, wm.cacheB);
            } else {
                dl = windowShift<C>(Q, bd.z, bd.w, bad);
                if (dl != 0) {
                    shiftFwd<C>(rs, dl, lane);
                    Q += C * dl;
                    have = false;
                }
                const int x0 = slotX0(d, Q), y0 = d - x0;
                ringEnsure<R, true>(c, wm.rx, x0 - 1, x0 + S - 2, false);
                ringEnsure<R, false>(c, wm.ry, y0 - S, y0 - 1, false);
                const int sLo = (bd.x >> 1) - Q, sHi = (bd.y >> 1) - Q;
                float4 *ca = wm.cacheA + (size_t) k * C * 32;
                float2 *cb = wm.cacheB + (size_t) k * C * 32;
                if (d & 1) {
                    if (have) stepSlots<C, R, 1>(c, wm.rx, wm.ry, d, Q, sy); else loadSlots<C, R>(c, wm.rx, wm.ry, d, Q, sy);
                    forwardDiagonal<C, 1, true>(c, rs, sy, sLo, sHi, ca, cb);
                } else {
                    if (have) stepSlots<C, R, 0>(c, wm.rx, wm.ry, d, Q, sy); else loadSlots<C, R>(c, wm.rx, wm.ry, d, Q, sy);
                    forwardDiagonal<C, 0, true>(c, rs, sy, sLo, sHi, ca, cb);
                }
                have = true;
            }
            if (lane == 0) wm.info[k] = make_int2(Q, dl);
        }
        __syncwarp();
        if (bad) break;

        // ---------------- backward over the block ----------------
        const int kLow = max(dStart, wa.tbTo + 1) - dStart;
        for (int k = dEnd - dStart; k >= kLow; k--) {
            const int d = dStart + k;
            const int2 inf = wm.info[k];
            const float4 *ca = wm.cacheA + (size_t) k * C * 32;
            const float2 *cb = wm.cacheB + (size_t) k * C * 32;
            float4 f[C];
            float2 e[C];
#pragma unroll
            for (int j = 0; j < C; j++) {
                f[j] = ca[j * 32 + lane];
                e[j] = cb[j * 32 + lane];
            }
            float bM[C], bX[C], bY[C];
            if (d == D) {
#pragma unroll
                for (int j = 0; j < C; j++) {
                    bM[j] = wa.endP[0];
                    bX[j] = wa.endP[1];
                    bY[j] = wa.endP[2];
                }
            } else {
                float sX[C], sY[C];
                if (d & 1) {
                    float nb = __shfl_down_sync(FULL_MASK, gX[0], 1);
                    if (lane == 31) nb = 0.0f;
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        sX[j] = (j < C - 1) ? gX[j + 1] : nb;
                        sY[j] = gY[j];
                    }
                } else {
                    float nb = __shfl_up_sync(FULL_MASK, gY[C - 1], 1);
                    if (lane == 0) nb = 0.0f;
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        sX[j] = gX[j];
                        sY[j] = (j > 0) ? gY[j - 1] : nb;
                    }
                }
#pragma unroll
                for (int j = 0; j < C; j++) {
                    const float s2 = (d & 1) ? gB[j] : gA[j];
                    bM[j] = __fmaf_rn(c.t[0 * 3 + 0], s2, __fmaf_rn(c.t[0 * 3 + 2], sY[j], c.t[0 * 3 + 1] * sX[j]));
                    bX[j] = __fmaf_rn(c.t[1 * 3 + 0], s2, __fmaf_rn(c.t[1 * 3 + 2], sY[j], c.t[1 * 3 + 1] * sX[j]));
                    bY[j] = __fmaf_rn(c.t[2 * 3 + 0], s2, __fmaf_rn(c.t[2 * 3 + 2], sY[j], c.t[2 * 3 + 1] * sX[j]));
                }
            }
            if (d <= wa.tbFrom) {
                if (untilRefresh == 0) {
                    untilRefresh = 10;
                    // total: cells of d plus the match transitions crossing d (impl/pairwiseAligner.c:567-584)
                    float sM1[C];
                    if (k > 0) {
                        const float4 *cp = wm.cacheA + (size_t) (k - 1) * C * 32;
#pragma unroll
                        for (int j = 0; j < C; j++) {
                            const float4 q = cp[j * 32 + lane];
                            sM1[j] = __fmaf_rn(c.t[2 * 3 + 0], q.z, __fmaf_rn(c.t[1 * 3 + 0], q.y, c.t[0 * 3 + 0] * q.x));
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < C; j++) sM1[j] = chkSM[j];
                    }
                    if (inf.y != 0) laneShift<C>(sM1, inf.y, lane);
                    float part = 0.0f;
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        const float uMn = (d & 1) ? gA[j] : gB[j];  // match u of d+1
                        part = __fmaf_rn(f[j].x, bM[j], part);
                        part = __fmaf_rn(f[j].y, bX[j], part);
                        part = __fmaf_rn(f[j].z, bY[j], part);
                        part = __fmaf_rn(uMn, sM1[j], part);
                    }
                    const float T = warpSum(part);
                    if (T > 0.0f) {
                        const int ex = exponentOf(T);
                        Tm = T * pow2f(-ex);
                        ET = Ef + Eb + ex;
                    } else {
                        Tm = 0.0f;
                        ET = 0;
                    }
                    if (wa.atEnd && posts == 0) {
                        logLik += Tm > 0.0f ? log((double) Tm) + (double) ET * 0.69314718055994530942 : -INFINITY;
                    }
                }
                posts++;
                untilRefresh--;
                if (Tm > 0.0f) {
                    const int ex = max(-126, min(127, Ef + Eb - ET));
                    const float scale = __fdividef(pow2f(ex), Tm);
                    float p[3][C];
#pragma unroll
                    for (int j = 0; j < C; j++) {
                        p[0][j] = (f[j].x * bM[j]) * scale;
                        p[1][j] = (f[j].y * bX[j]) * scale;
                        p[2][j] = (f[j].z * bY[j]) * scale;
                    }
                    emitDiagonal<C>(lane, o, p, wa.thr, slotX0(d, inf.x), d);
                }
            }
            // u-values of d (emissions are zero outside the band)
#pragma unroll
            for (int j = 0; j < C; j++) {
                gX[j] = e[j].x * bX[j];
                gY[j] = e[j].y * bY[j];
                const float uM = f[j].w * bM[j];
                if (d & 1) gB[j] = uM; else gA[j] = uM;
            }
            // moving below d crosses the window shift met when entering d
            if (inf.y != 0) {
                laneShift<C>(gX, -inf.y, lane);
                laneShift<C>(gY, -inf.y, lane);
                laneShift<C>(gA, -inf.y, lane);
                laneShift<C>(gB, -inf.y, lane);
            }
        }
        // rescale the carried backward state at the block boundary
        {
            float m = 0.0f;
#pragma unroll
            for (int j = 0; j < C; j++) m = fmaxf(m, fmaxf(fmaxf(gX[j], gY[j]), fmaxf(gA[j], gB[j])));
            m = warpMax(m);
            if (m > 0.0f) {
                const int kx = exponentOf(m);
                const float s = pow2f(-kx);
#pragma unroll
                for (int j = 0; j < C; j++) {
                    gX[j] *= s;
                    gY[j] *= s;
                    gA[j] *= s;
                    gB[j] *= s;
                }
                Eb += kx;
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// One task: forward sweep with checkpoints, walks at traceback points and end.
// ---------------------------------------------------------------------------

template <int C, int K>
__device__ __forceinline__ void runTask(const DpArgs &a, const float *rpAll, const float *smAll, const float *gxAll,
                                        const float *gyAll, int taskIndex, WarpMem<C, K> &wm, const Scratch &sc) {
    constexpr int S = 32 * C;
    constexpr int R = Geo<C>::R;
    const int lane = threadIdx.x & 31;
    const Task &tk = a.tasks[taskIndex];
    TaskOut *to = a.out + taskIndex;
    Ctx c;
    c.lane = lane;
    c.lx = tk.lx;
    c.ly = tk.ly;
    c.N = tk.lx + tk.ly;
    c.xs = a.xs + tk.xOff;
    c.ys = a.ys + tk.yOff;
    c.band = reinterpret_cast<const int4 *>(a.band) + tk.bandOff;
    const int model = (tk.flags & 4) ? 0 : 1;
    const DevModel &dm = a.models[model];
#pragma unroll
    for (int k = 0; k < 9; k++) c.t[k] = dm.t[k];
    c.rp = reinterpret_cast<const char *>(rpAll + (a.sharedRepeat ? 0 : model * kRepTable));
    c.sm = smAll + model * 25;
    c.gx = gxAll + model * 5;
    c.gy = gyAll + model * 5;
    c.rle = dm.runLength;
    c.strandFwd = dm.strand;
    const int status0 = to->status;
    if (c.N == 0 || (status0 & kTaskBand)) {
        if (lane == 0) {
            to->count[0] = to->count[1] = to->count[2] = 0;
            to->logLik = 0.0;
        }
        return;
    }
    if (c.N / K + 1 > sc.blocks) {
        if (lane == 0) {
            to->status = status0 | kTaskScratch;
            to->count[0] = to->count[1] = to->count[2] = 0;
        }
        return;
    }
    Out o;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        o.w[k] = a.outW[k] + tk.outOff[k];
        o.x[k] = a.outX[k] + tk.outOff[k];
        o.y[k] = a.outY[k] + tk.outOff[k];
        o.top[k] = tk.cap[k];
        o.written[k] = 0;
    }
    o.xShift = tk.x1 + tk.xShift;
    o.yShift = tk.y1;
    WalkArgs wa;
    wa.startP = (tk.flags & 1) ? dm.raggedStart : dm.start;
    wa.thr = a.threshold;
    double logLik = 0.0;
    bool bad = false;
    wm.rx.bad = 0;
    wm.ry.bad = 0;

    // band records: 32-diagonal chunks through cp.async into the warp's ring of 64
    auto issueChunk = [&](int chunk) {
        const int dd = chunk * 32 + lane;
        if (dd <= c.N) cpAsync16(&wm.bandRing[dd & 63], &c.band[dd]);
        cpAsyncCommit();
    };
    issueChunk(0);
    issueChunk(1);
    cpAsyncWaitAllButOne();
    __syncwarp();

    Fwd<C> st;
    Slots<C> sy;
    const int4 b0 = wm.bandRing[0];
    int Q = initialWindow<C>(b0.z, b0.w);
    int Ef = 0;
    {
        const int x0 = slotX0(0, Q);
        ringFill<R, true>(c, wm.rx, x0 - 1 - 8);
        ringFill<R, false>(c, wm.ry, -x0 - S - 8);
        forwardOrigin<C, false>(c, wa.startP, Q, st, nullptr, nullptr);
    }
    bool have = false;
    int tracedBackTo = 0;
    for (int d = 1; d <= c.N; d++) {
        if ((d & 31) == 0) {
            issueChunk((d >> 5) + 1);
            cpAsyncWaitAllButOne();
            __syncwarp();
        }
        if ((d & (K - 1)) == 0) {
            Ef += rescaleFwd<C>(st);
            const int b = d / K;
            storeFwd<C>(sc.chk + (size_t) b * C * 32, lane, st);
            if (lane == 0) sc.scal[b] = make_int2(Ef, Q);
        }
        const int4 bd = wm.bandRing[d & 63];
        const int dl = windowShift<C>(Q, bd.z, bd.w, bad);
        if (bad) break;
        if (dl != 0) {
            shiftFwd<C>(st, dl, lane);
            Q += C * dl;
            have = false;
        }
        const int x0 = slotX0(d, Q), y0 = d - x0;
        ringEnsure<R, true>(c, wm.rx, x0 - 1, x0 + S - 2, true);
        ringEnsure<R, false>(c, wm.ry, y0 - S, y0 - 1, true);
        const int sLo = (bd.x >> 1) - Q, sHi = (bd.y >> 1) - Q;
        if (d & 1) {
            if (have) stepSlots<C, R, 1>(c, wm.rx, wm.ry, d, Q, sy); else loadSlots<C, R>(c, wm.rx, wm.ry, d, Q, sy);
            forwardDiagonal<C, 1, false>(c, st, sy, sLo, sHi, nullptr, nullptr);
        } else {
            if (have) stepSlots<C, R, 0>(c, wm.rx, wm.ry, d, Q, sy); else loadSlots<C, R>(c, wm.rx, wm.ry, d, Q, sy);
            forwardDiagonal<C, 0, false>(c, st, sy, sLo, sHi, nullptr, nullptr);
        }
        have = true;
        const bool atEnd = d == c.N;
        const int width = ((bd.y - bd.x) >> 1) + 1;
        if (atEnd || (d >= tracedBackTo + a.minDiagsBetweenTraceBack && width <= 2 * a.diagonalExpansion + 1)) {
            if (!atEnd) storeFwd<C>(sc.resume, lane, st);
            wa.D = d;
            wa.tbTo = tracedBackTo;
            wa.tbFrom = atEnd ? d : d - (a.traceBackDiagonals + 1);
            wa.atEnd = atEnd ? 1 : 0;
            wa.endP = (atEnd && (tk.flags & 2)) ? dm.raggedEnd : dm.end;
            walkSegment<C, K>(c, wm, sc, wa, o, logLik, bad);
            tracedBackTo = wa.tbFrom;
            if (bad || atEnd) break;
            float4 v[C];
#pragma unroll
            for (int j = 0; j < C; j++) v[j] = sc.resume[j * 32 + lane];
            loadFwd<C>(v, st);
            have = false;
        }
    }
    // drain the band prefetch group before the ring is reused
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    if (lane == 0) {
        int s = status0;
        if (bad) s |= kTaskWindow;
        if (wm.rx.bad | wm.ry.bad) s |= kTaskSymbol;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            to->count[k] = bad ? 0 : o.written[k];
            if (!bad && o.written[k] > o.top[k]) s |= kTaskCapacity;
        }
        to->status = s;
        to->logLik = logLik;
    }
}

template <int C, int K, int MAXW>
__global__ void __launch_bounds__(MAXW * 32, 1) posteriorKernel(DpArgs a) {
    using WS = WarpSmem<C, K>;
    constexpr int R = Geo<C>::R;
    extern __shared__ __align__(16) unsigned char smemRaw[];
    const int nTables = a.sharedRepeat ? 1 : 2;
    float *rp = reinterpret_cast<float *>(smemRaw);
    float *sm = rp + nTables * kRepTable;
    float *gx = sm + 2 * 25;
    float *gy = gx + 2 * 5;
    unsigned char *warpBase =
        smemRaw + (((size_t) (nTables * kRepTable + 2 * 25 + 2 * 5 + 2 * 5) * sizeof(float) + 15) & ~(size_t) 15);
    for (int i = threadIdx.x; i < nTables * kRepTable; i += blockDim.x) rp[i] = a.repeatProb[i];
    for (int i = threadIdx.x; i < 2 * 25; i += blockDim.x) sm[i] = a.models[i / 25].match[i % 25];
    for (int i = threadIdx.x; i < 2 * 5; i += blockDim.x) {
        gx[i] = a.models[i / 5].gapX[i % 5];
        gy[i] = a.models[i / 5].gapY[i % 5];
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * (blockDim.x >> 5) + warp;
    unsigned char *mine = warpBase + (size_t) warp * WS::bytes;
    WarpMem<C, K> wm;
    wm.rx = Ring<R>{reinterpret_cast<uint2 *>(mine), 0, 0};
    wm.ry = Ring<R>{reinterpret_cast<uint2 *>(mine) + R, 0, 0};
    wm.bandRing = reinterpret_cast<int4 *>(mine + WS::ringBytes);
    wm.walkBand = reinterpret_cast<int4 *>(mine + WS::ringBytes + WS::bandRingBytes);
    wm.cacheA = reinterpret_cast<float4 *>(mine + WS::ringBytes + WS::bandRingBytes + WS::walkBandBytes);
    wm.cacheB = reinterpret_cast<float2 *>(mine + WS::ringBytes + WS::bandRingBytes + WS::walkBandBytes +
                                           WS::cacheABytes);
    wm.info = reinterpret_cast<int2 *>(mine + WS::ringBytes + WS::bandRingBytes + WS::walkBandBytes +
                                       WS::cacheABytes + WS::cacheBBytes);
    Scratch sc;
    sc.blocks = a.scratchBlocks;
    sc.chk = a.scratch + (size_t) gwarp * a.scratchBlocks * (C * 32);
    sc.scal = a.scratchScalars + (size_t) gwarp * a.scratchBlocks;
    sc.resume = a.resume + (size_t) gwarp * (C * 32);

    while (true) {
        int t = 0;
        if (lane == 0) t = atomicAdd(a.queue, 1);
        t = __shfl_sync(FULL_MASK, t, 0);
        if (t >= a.nTasks) break;
        runTask<C, K>(a, rp, sm, gx, gy, a.order[t], wm, sc);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------

size_t tableBytes(int nTables) {
    return (((size_t) (nTables * kRepTable + 2 * 25 + 2 * 5 + 2 * 5) * sizeof(float) + 15) & ~(size_t) 15);
}

template <int C, int K>
static size_t smemFor(int warps, int nTables) {
    return tableBytes(nTables) + (size_t) warps * WarpSmem<C, K>::bytes;
}

template <int C, int K, int MAXW>
static cudaError_t launchT(const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    if (warps > MAXW || warps < 1) return cudaErrorInvalidValue;
    const size_t smem = smemFor<C, K>(warps, a.sharedRepeat ? 1 : 2);
    cudaError_t e = cudaFuncSetAttribute(posteriorKernel<C, K, MAXW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) smem);
    if (e != cudaSuccess) return e;
    posteriorKernel<C, K, MAXW><<<blocks, warps * 32, smem, s>>>(a);
    return cudaGetLastError();
}

// Slot classes: C slots per lane (window S = 32*C), checkpoint stride K.
int classStride(int C) {
    return C <= 3 ? 8 : 4;
}

static int maxWarpsFor(int C, int nTables) {
    // as many warps as the 227 KB of shared memory per block allows, at most 16
    const size_t limit = 227 * 1024;
    int w = 16;
    while (w > 1) {
        size_t need = 0;
        switch (C) {
            case 2: need = smemFor<2, 8>(w, nTables); break;
            case 3: need = smemFor<3, 8>(w, nTables); break;
            case 4: need = smemFor<4, 4>(w, nTables); break;
            case 6: need = smemFor<6, 4>(w, nTables); break;
            case 8: need = smemFor<8, 4>(w, nTables); break;
            default: need = limit + 1;
        }
        if (need <= limit) break;
        w--;
    }
    return w;
}

// Upper bounds on warps per block per class (shared-memory limited with one table);
// they are the kernels' launch bounds, so the compiler may use 65536/(32*MAXW) registers.
constexpr int kMaxW2 = 12, kMaxW3 = 8, kMaxW4 = 10, kMaxW6 = 8, kMaxW8 = 5;

int classMaxWarps(int C, int nTables) {
    int cap = C == 2 ? kMaxW2 : C == 3 ? kMaxW3 : C == 4 ? kMaxW4 : C == 6 ? kMaxW6 : kMaxW8;
    return std::min(cap, maxWarpsFor(C, nTables));
}

cudaError_t launchPosterior(int C, const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    switch (C) {
        case 2: return launchT<2, 8, kMaxW2>(a, blocks, warps, s);
        case 3: return launchT<3, 8, kMaxW3>(a, blocks, warps, s);
        case 4: return launchT<4, 4, kMaxW4>(a, blocks, warps, s);
        case 6: return launchT<6, 4, kMaxW6>(a, blocks, warps, s);
        case 8: return launchT<8, 4, kMaxW8>(a, blocks, warps, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mp
