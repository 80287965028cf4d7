// Device kernels of the realignment engine (sm_100a).
//
// Hot path: the anchored, banded 3-state pair-HMM forward / backward /
// posterior pass of MarginPolish (impl/pairwiseAligner.c:687-808 driven by
// :942-991, cell recurrence impl/stateMachine.c:559-581, posterior rules
// impl/pairwiseAligner.c:586-664), re-designed for one warp per banded
// sub-problem:
//
//  * Cells of one anti-diagonal d live in a window of S = 32*C slots, C
//    consecutive slots per lane; slot i holds xmy = 2(Q+i) + (d&1). The window
//    origin Q only moves (by whole lanes) when the band leaves it, so the
//    neighbour exchange between diagonals is one __shfl per lane per diagonal.
//  * Values are FP32 probabilities (not logs), rescaled by exact powers of two
//    every K diagonals; the integer exponents are tracked per block of K
//    diagonals, so no log/exp is evaluated per cell and the FP64 likelihood is
//    ln(mantissa) + exponent*ln2 once per segment.
//  * The forward sweep writes a checkpoint (4 floats per slot) every K
//    diagonals. Each traceback walk recomputes the forward values of one block
//    of K diagonals into registers and runs the backward recurrence and the
//    posteriors over that block, from the top block down.
//  * Posterior tuples are compacted in the warp (ballot + prefix) and written
//    from the top of the task's output region downwards, which yields the
//    reference's output order (ascending anti-diagonal, descending x-y within
//    one, later traceback segments first) without a separate reversal.
#include "mp_internal.h"

#include <cstdio>

namespace mp {

#define FULL_MASK 0xffffffffu

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

template <int C>
struct Geometry {
    static constexpr int S = 32 * C;
    // symbol ring: covers the window plus enough room to move
    static constexpr int R = (S + 64 <= 128) ? 128 : ((S + 64 <= 256) ? 256 : 512);
};

__device__ __forceinline__ float pow2f(int k) {
    // 2^k for k in [-126, 127]
    return __int_as_float((127 + k) << 23);
}

__device__ __forceinline__ int exponentOf(float m) {
    // floor(log2(m)) for normal m; -127 for denormals
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

// Uniform task constants held by every lane.
struct TaskCtx {
    const Task *task;
    int lane;
    int lx, ly, N;
    const uint16_t *xs;
    const uint16_t *ys;
    const int4 *band;       // (xmyL, xmyR, hullL, hullR) per diagonal of this task
    float t[9];
    const float *rpS;       // shared: this model's repeat table
    const float *smS;       // shared: this model's match table [25]
    const float *gxS;       // shared: gap-x [5]
    const float *gyS;       // shared: gap-y [5]
    const float *bStart;    // global model boundary vectors
    const float *bEnd;
    int rle;
    int strandFwd;          // model's strand flag
    int rpByteBase;         // byte offset of this model's table in the shared repeat region
};

// Decoded X symbol: packed (repeat-table byte offset | match-row byte offset << 17), gap-x emission.
__device__ __forceinline__ uint2 decodeX(const TaskCtx &c, int pos, int &bad) {
    int b = 4, rc = 0;
    if (pos >= 0 && pos < c.lx) {
        uint32_t s = c.xs[pos];
        if (c.rle) {
            b = s & 255;
            rc = s >> 8;
        } else {
            b = (int) s;
        }
        b = b > 4 ? 4 : b;
        if (rc >= kMaxRepeat) {  // keeps the table lookup in bounds; reported as an argument error
            rc = kMaxRepeat - 1;
            bad = 1;
        }
    }
    int bb = b == 4 ? 0 : b;  // 'N' reads the A row of the repeat table
    int row = c.strandFwd ? bb : 3 - bb;
    uint32_t pk = (uint32_t) (c.rpByteBase + (row * (kMaxRepeat * kMaxRepeat) + rc * kMaxRepeat) * 4) |
                  ((uint32_t) (b * 20) << 17);
    return make_uint2(pk, __float_as_uint(c.gxS[b]));
}

// Decoded Y symbol: packed (repeat column byte offset | match-column byte offset << 17), gap-y emission.
__device__ __forceinline__ uint2 decodeY(const TaskCtx &c, int pos, int &bad) {
    int b = 4, rc = 0;
    if (pos >= 0 && pos < c.ly) {
        uint32_t s = c.ys[pos];
        if (c.rle) {
            b = s & 255;
            rc = s >> 8;
        } else {
            b = (int) s;
        }
        b = b > 4 ? 4 : b;
        if (rc >= kMaxRepeat) {
            rc = kMaxRepeat - 1;
            bad = 1;
        }
    }
    uint32_t pk = (uint32_t) (rc * 4) | ((uint32_t) (b * 4) << 17);
    return make_uint2(pk, __float_as_uint(c.gyS[b]));
}

// Match emission of a cell from the two packed symbols.
__device__ __forceinline__ float matchEmission(const TaskCtx &c, const char *rpBase, uint32_t xpk, uint32_t ypk) {
    uint32_t s = xpk + ypk;
    float r = *reinterpret_cast<const float *>(rpBase + (s & 0x1ffffu));
    float m = *reinterpret_cast<const float *>(reinterpret_cast<const char *>(c.smS) + (s >> 17));
    return r * m;
}

// ---------------------------------------------------------------------------
// Symbol rings: decoded symbols of a span of positions, in shared memory.
// ---------------------------------------------------------------------------

template <int R>
struct Ring {
    uint2 *buf;
    int lo;   // first cached position (uniform)
    int bad;  // sticky: a decoded symbol had a repeat count >= kMaxRepeat (clamped)
};

template <int R, bool IS_X>
__device__ __forceinline__ void ringFill(const TaskCtx &c, Ring<R> &r, int newLo) {
    r.lo = newLo;
    int bad = 0;
#pragma unroll
    for (int k = 0; k < R / 32; k++) {
        int p = newLo + k * 32 + c.lane;
        r.buf[p & (R - 1)] = IS_X ? decodeX(c, p, bad) : decodeY(c, p, bad);
    }
    if (__any_sync(FULL_MASK, bad)) r.bad = 1;
    __syncwarp();
}

// Make positions [needLo, needHi] resident; on a miss the ring is re-centred
// so that `up` movement (forward sweep) or downward movement (walk) has room.
template <int R, bool IS_X>
__device__ __forceinline__ void ringEnsure(const TaskCtx &c, Ring<R> &r, int needLo, int needHi, bool up) {
    if (needLo < r.lo || needHi >= r.lo + R) {
        int slack = R - (needHi - needLo + 1);
        int newLo = up ? needLo - slack / 8 : needLo - (slack - slack / 8);
        ringFill<R, IS_X>(c, r, newLo);
    }
}

template <int R>
__device__ __forceinline__ uint2 ringGet(const Ring<R> &r, int p) {
    return r.buf[p & (R - 1)];
}

// ---------------------------------------------------------------------------
// Per-lane slot state
// ---------------------------------------------------------------------------

template <int C>
struct Slots {
    uint32_t xpk[C];
    float ex[C];
    uint32_t ypk[C];
    float ey[C];
};

// Load slot symbols for diagonal d, window Q, from the rings.
template <int C, int R>
__device__ __forceinline__ void loadSlots(const TaskCtx &c, const Ring<R> &rx, const Ring<R> &ry, int d, int Q,
                                          Slots<C> &s) {
    int x0 = Q + ((d + 1) >> 1);  // x of slot 0
    int y0 = d - x0;               // y of slot 0
#pragma unroll
    for (int j = 0; j < C; j++) {
        int i = c.lane * C + j;
        uint2 vx = ringGet(rx, x0 + i - 1);
        uint2 vy = ringGet(ry, y0 - i - 1);
        s.xpk[j] = vx.x;
        s.ex[j] = __uint_as_float(vx.y);
        s.ypk[j] = vy.x;
        s.ey[j] = __uint_as_float(vy.y);
    }
}

// Advance slot symbols from diagonal d-1 to d (window unchanged).
// Entering odd d: x of every slot grows by one (shift X down a slot).
// Entering even d: y of every slot grows by one (shift Y up a slot).
template <int C, int R>
__device__ __forceinline__ void stepSlots(const TaskCtx &c, const Ring<R> &rx, const Ring<R> &ry, int d, int Q,
                                          Slots<C> &s) {
    constexpr int S = 32 * C;
    if (d & 1) {
        uint2 fresh = ringGet(rx, Q + ((d + 1) >> 1) + S - 2);
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
        int y0 = d - (Q + ((d + 1) >> 1));
        uint2 fresh = ringGet(ry, y0 - 1);
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

// Forward state carried between diagonals: outgoing gap-x / gap-y sums of d-1
// and outgoing match sums of d-1 and d-2 (even diagonals own mA, odd own mB).
template <int C>
struct FwdState {
    float ox[C], oy[C], mA[C], mB[C];
};

// Shift a per-slot array by `dl` whole lanes: new lane l takes old lane l+dl.
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

// Window rule, shared by the sweep and the recompute so that both take the same
// decisions: the window must contain the hull of bands d-2..d+2. Returns the lane
// shift (new Q = Q + C*shift); sets *bad if the hull does not fit.
template <int C>
__device__ __forceinline__ int windowShift(int Q, int hullLo, int hullHi, bool *bad) {
    constexpr int S = 32 * C;
    int needLo = hullLo >> 1, needHi = hullHi >> 1;
    if (needLo >= Q && needHi <= Q + S - 1) return 0;
    int span = needHi - needLo + 1;
    if (span > S - 2 * C) {
        *bad = true;
        return 0;
    }
    int target = needLo - (S - span) / 2;
    int diff = target - Q;
    int dl = diff >= 0 ? diff / C : -((-diff + C - 1) / C);
    int q2 = Q + C * dl;
    if (q2 + S - 1 < needHi) dl++;
    if (Q + C * dl > needLo) *bad = true;
    return dl;
}

template <int C>
__device__ __forceinline__ int initialWindow(int hullLo, int hullHi) {
    constexpr int S = 32 * C;
    int needLo = hullLo >> 1, needHi = hullHi >> 1;
    int span = needHi - needLo + 1;
    return needLo - (S - span) / 2;
}

// ---------------------------------------------------------------------------
// One forward anti-diagonal (push form). PAR = d & 1.
// ---------------------------------------------------------------------------

struct FwdCell {
    float fM, fX, fY;
};

template <int C, int PAR>
__device__ __forceinline__ void forwardDiagonal(const TaskCtx &c, const char *rpBase, FwdState<C> &st,
                                                const Slots<C> &sy, int sLo, int sHi, FwdCell (&out)[C],
                                                float (&eMOut)[C], uint32_t &inbBits, int inbShift) {
    float inX[C], inY[C];
    if (PAR) {  // odd d: gap-x source is slot i, gap-y source is slot i+1
        float nb = __shfl_down_sync(FULL_MASK, st.oy[0], 1);
        if (c.lane == 31) nb = 0.0f;
#pragma unroll
        for (int j = 0; j < C; j++) {
            inX[j] = st.ox[j];
            inY[j] = (j < C - 1) ? st.oy[j + 1] : nb;
        }
    } else {  // even d: gap-x source is slot i-1, gap-y source is slot i
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
        float mid = PAR ? st.mB[j] : st.mA[j];
        float eM = matchEmission(c, rpBase, sy.xpk[j], sy.ypk[j]);
        float fM = eM * mid;
        float fX = sy.ex[j] * inX[j];
        float fY = sy.ey[j] * inY[j];
        bool in = (unsigned) (base + j) <= span;
        fM = in ? fM : 0.0f;
        fX = in ? fX : 0.0f;
        fY = in ? fY : 0.0f;
        inbBits |= (in ? 1u : 0u) << (inbShift + j);
        float nm = __fmaf_rn(c.t[2 * 3 + 0], fY, __fmaf_rn(c.t[1 * 3 + 0], fX, c.t[0 * 3 + 0] * fM));
        float nx = __fmaf_rn(c.t[2 * 3 + 1], fY, __fmaf_rn(c.t[1 * 3 + 1], fX, c.t[0 * 3 + 1] * fM));
        float ny = __fmaf_rn(c.t[1 * 3 + 2], fX, __fmaf_rn(c.t[2 * 3 + 2], fY, c.t[0 * 3 + 2] * fM));
        if (PAR) st.mB[j] = nm; else st.mA[j] = nm;
        st.ox[j] = nx;
        st.oy[j] = ny;
        out[j].fM = fM;
        out[j].fX = fX;
        out[j].fY = fY;
        eMOut[j] = eM;
    }
}

// Diagonal 0: the start cell (xmy = 0) holds the start (or ragged-start) probabilities.
template <int C>
__device__ __forceinline__ void forwardOrigin(const TaskCtx &c, const float *startP, int Q, FwdState<C> &st,
                                              FwdCell (&out)[C]) {
    int i0 = -Q;  // slot of xmy = 0 at d = 0
#pragma unroll
    for (int j = 0; j < C; j++) {
        bool here = c.lane * C + j == i0;
        float fM = here ? startP[0] : 0.0f;
        float fX = here ? startP[1] : 0.0f;
        float fY = here ? startP[2] : 0.0f;
        st.mA[j] = __fmaf_rn(c.t[2 * 3 + 0], fY, __fmaf_rn(c.t[1 * 3 + 0], fX, c.t[0 * 3 + 0] * fM));
        st.ox[j] = __fmaf_rn(c.t[2 * 3 + 1], fY, __fmaf_rn(c.t[1 * 3 + 1], fX, c.t[0 * 3 + 1] * fM));
        st.oy[j] = __fmaf_rn(c.t[1 * 3 + 2], fX, __fmaf_rn(c.t[2 * 3 + 2], fY, c.t[0 * 3 + 2] * fM));
        st.mB[j] = 0.0f;
        out[j].fM = fM;
        out[j].fX = fX;
        out[j].fY = fY;
    }
}

// Rescale the carried forward state by a power of two; returns the exponent removed.
template <int C>
__device__ __forceinline__ int rescaleForward(FwdState<C> &st) {
    float m = 0.0f;
#pragma unroll
    for (int j = 0; j < C; j++) m = fmaxf(m, fmaxf(fmaxf(st.ox[j], st.oy[j]), fmaxf(st.mA[j], st.mB[j])));
    m = warpMax(m);
    if (!(m > 0.0f)) return 0;
    int k = exponentOf(m);
    float sc = pow2f(-k);
#pragma unroll
    for (int j = 0; j < C; j++) {
        st.ox[j] *= sc;
        st.oy[j] *= sc;
        st.mA[j] *= sc;
        st.mB[j] *= sc;
    }
    return k;
}

template <int C>
__device__ __forceinline__ void shiftForward(FwdState<C> &st, int dl, int lane) {
    laneShift<C>(st.ox, dl, lane);
    laneShift<C>(st.oy, dl, lane);
    laneShift<C>(st.mA, dl, lane);
    laneShift<C>(st.mB, dl, lane);
}

// Checkpoint store / load: one float4 per slot, coalesced over the warp.
template <int C>
__device__ __forceinline__ void storeCheckpoint(float4 *chk, int lane, const FwdState<C> &st) {
#pragma unroll
    for (int j = 0; j < C; j++) chk[j * 32 + lane] = make_float4(st.ox[j], st.oy[j], st.mA[j], st.mB[j]);
}

template <int C>
__device__ __forceinline__ void loadCheckpoint(const float4 *chk, int lane, FwdState<C> &st) {
#pragma unroll
    for (int j = 0; j < C; j++) {
        float4 v = chk[j * 32 + lane];
        st.ox[j] = v.x;
        st.oy[j] = v.y;
        st.mA[j] = v.z;
        st.mB[j] = v.w;
    }
}

// ---------------------------------------------------------------------------
// Output: ordered warp compaction of the tuples of one diagonal.
// ---------------------------------------------------------------------------

struct OutCursor {
    int32_t *w[3];
    int32_t *x[3];
    int32_t *y[3];
    int top[3];       // capacity
    int written[3];   // tuples emitted so far (also counted past capacity)
};

// Emits, for each list, the tuples of this diagonal in ascending slot order at
// positions top-1-(written+rank), i.e. the final list reads them in descending x-y.
template <int C>
__device__ __forceinline__ void emitDiagonal(int lane, OutCursor &oc, const float (&p)[3][C], float thr,
                                             int x0, int d, int xOutShift, int yOutShift) {
    // per-lane packed counts: 10 bits per list
    uint32_t cnt = 0;
#pragma unroll
    for (int j = 0; j < C; j++) {
        cnt += (p[0][j] >= thr ? 1u : 0u) + (p[1][j] >= thr ? 1024u : 0u) + (p[2][j] >= thr ? 1048576u : 0u);
    }
    if (__ballot_sync(FULL_MASK, cnt != 0) == 0) return;
    // exclusive warp prefix of the packed counts
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(FULL_MASK, incl, o);
        if (lane >= o) incl += v;
    }
    uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    uint32_t excl = incl - cnt;
    if (cnt != 0) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            int r = oc.written[k] + (int) ((excl >> (10 * k)) & 1023u);
#pragma unroll
            for (int j = 0; j < C; j++) {
                float v = p[k][j];
                if (v >= thr) {
                    int pos = oc.top[k] - 1 - r;
                    if (pos >= 0) {
                        int x = x0 + lane * C + j;
                        int y = d - x;
                        float q = fminf(v, 1.0f);
                        oc.w[k][pos] = (int32_t) floorf(q * (float) kProbOne);
                        oc.x[k][pos] = x - 1 + xOutShift;
                        oc.y[k][pos] = y - 1 + yOutShift;
                    }
                    r++;
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) oc.written[k] += (int) ((total >> (10 * k)) & 1023u);
}

// ---------------------------------------------------------------------------
// The posterior kernel: persistent, one warp per task, length-sorted queue.
// ---------------------------------------------------------------------------

template <int C, int K>
struct WarpWork {
    static constexpr int S = 32 * C;
    static constexpr int R = Geometry<C>::R;
};

struct SharedTables {
    float *rp;      // [2][kRepTable]
    float *sm;      // [2][25]
    float *gx;      // [2][5]
    float *gy;      // [2][5]
};

template <int C, int K>
__device__ void runTask(const DpArgs &a, const SharedTables &tab, int taskIndex, Ring<Geometry<C>::R> &rx,
                        Ring<Geometry<C>::R> &ry, float4 *chkBase, int2 *chkScal, float4 *resumeBase) {
    constexpr int S = 32 * C;
    constexpr int R = Geometry<C>::R;
    const int lane = threadIdx.x & 31;
    const Task &tk = a.tasks[taskIndex];
    TaskOut *to = a.out + taskIndex;

    TaskCtx c;
    c.task = &tk;
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
    c.rpS = tab.rp + model * kRepTable;
    c.smS = tab.sm + model * 25;
    c.gxS = tab.gx + model * 5;
    c.gyS = tab.gy + model * 5;
    c.rle = dm.runLength;
    c.strandFwd = dm.strand;
    c.rpByteBase = 0;
    const char *rpBase = reinterpret_cast<const char *>(c.rpS);
    const bool raggedL = tk.flags & 1, raggedR = tk.flags & 2;
    const float *startP = raggedL ? dm.raggedStart : dm.start;

    int status = to->status;  // band kernel may already have flagged the task
    if (c.N == 0 || (status & kTaskBand)) {
        if (lane == 0) {
            to->count[0] = to->count[1] = to->count[2] = 0;
            to->logLik = 0.0;
        }
        return;
    }
    const int nBlocks = c.N / K + 1;
    if (nBlocks > a.scratchBlocks) {
        if (lane == 0) {
            to->status = status | kTaskScratch;
            to->count[0] = to->count[1] = to->count[2] = 0;
        }
        return;
    }

    OutCursor oc;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        oc.w[k] = a.outW[k] + tk.outOff[k];
        oc.x[k] = a.outX[k] + tk.outOff[k];
        oc.y[k] = a.outY[k] + tk.outOff[k];
        oc.top[k] = tk.cap[k];
        oc.written[k] = 0;
    }
    const int xOutShift = tk.x1 + tk.xShift;
    const int yOutShift = tk.y1;
    const float thr = a.threshold;
    double logLik = 0.0;
    bool bad = false;

    rx.bad = 0;
    ry.bad = 0;

    // ------------------------------------------------------------------
    // Forward sweep
    // ------------------------------------------------------------------
    FwdState<C> st;
    Slots<C> sy;
    int4 b0 = c.band[0];
    int Q = initialWindow<C>(b0.z, b0.w);
    int Ef = 0;
    {
        ringFill<R, true>(c, rx, Q + 0 - 1 - 8);
        ringFill<R, false>(c, ry, 0 - Q - S - 8);
        FwdCell dummy[C];
        forwardOrigin<C>(c, startP, Q, st, dummy);
    }
    int tracedBackTo = 0;
    int d = 1;
    // window and symbols for diagonal 1 are set at the top of the loop
    bool haveSlots = false;
    while (d <= c.N && !bad) {
        if ((d % K) == 0) {
            Ef += rescaleForward<C>(st);
            int b = d / K;
            storeCheckpoint<C>(chkBase + (size_t) b * (C * 32), lane, st);
            if (lane == 0) chkScal[b] = make_int2(Ef, Q);
        }
        int4 bd = c.band[d];
        int dl = windowShift<C>(Q, bd.z, bd.w, &bad);
        if (bad) break;
        if (dl != 0) {
            shiftForward<C>(st, dl, lane);
            Q += C * dl;
            haveSlots = false;
        }
        {
            int x0 = Q + ((d + 1) >> 1);
            int y0 = d - x0;
            ringEnsure<R, true>(c, rx, x0 - 1, x0 + S - 2, true);
            ringEnsure<R, false>(c, ry, y0 - S, y0 - 1, true);
            if (!haveSlots) {
                loadSlots<C, R>(c, rx, ry, d, Q, sy);
                haveSlots = true;
            } else {
                stepSlots<C, R>(c, rx, ry, d, Q, sy);
            }
        }
        int sLo = (bd.x >> 1) - Q, sHi = (bd.y >> 1) - Q;
        FwdCell fc[C];
        float eMv[C];
        uint32_t inb = 0;
        if (d & 1) forwardDiagonal<C, 1>(c, rpBase, st, sy, sLo, sHi, fc, eMv, inb, 0);
        else forwardDiagonal<C, 0>(c, rpBase, st, sy, sLo, sHi, fc, eMv, inb, 0);

        const bool atEnd = d == c.N;
        const int width = ((bd.y - bd.x) >> 1) + 1;
        const bool tbPoint = d >= tracedBackTo + a.minDiagsBetweenTraceBack && width <= 2 * a.diagonalExpansion + 1;
        if (atEnd || tbPoint) {
            // ---- save the sweep state (resumed after the walk) ----
            if (!atEnd) {
                storeCheckpoint<C>(resumeBase, lane, st);
            }
            const int D = d;
            const int tbFrom = atEnd ? D : D - (a.traceBackDiagonals + 1);
            // ---- traceback walk over (tracedBackTo, D] ----
            float gX[C], gY[C], gA[C], gB[C];  // backward u-values: gap-x, gap-y of d+1; match of d (A even, B odd)
#pragma unroll
            for (int j = 0; j < C; j++) gX[j] = gY[j] = gA[j] = gB[j] = 0.0f;
            int Eb = 0;
            int posts = 0;
            float Tm = 0.0f;
            int ET = 0;
            int carryShift = 0;  // window shift met when entering the block above (from its first diagonal)
            const int bTop = D / K, bBot = (tracedBackTo + 1) / K;
            for (int b = bTop; b >= bBot && !bad; b--) {
                const int dStart = b * K;
                const int dEnd = min(dStart + K - 1, D);
                // -------- recompute forward values of this block --------
                FwdState<C> rs;
                Slots<C> rsy;
                int rQ, rEf;
                float chkSM[C];  // outgoing match sum of dStart-1 (crossing term)
                FwdCell F[K][C];
                float EM[K][C], EXc[K][C], EYc[K][C];
                uint32_t inbK = 0;
                int shiftAt[K];
                int sLoK[K], sHiK[K];
                bool rHave = false;
                if (b == 0) {
                    rQ = initialWindow<C>(b0.z, b0.w);
                    rEf = 0;
                } else {
                    loadCheckpoint<C>(chkBase + (size_t) b * (C * 32), lane, rs);
                    int2 sc = chkScal[b];
                    rEf = sc.x;
                    rQ = sc.y;
                }
#pragma unroll
                for (int j = 0; j < C; j++) chkSM[j] = rs.mB[j];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    shiftAt[k] = 0;
                    const int dd = dStart + k;
                    if (dd <= dEnd) {
                        if (dd == 0) {
                            int4 bz = c.band[0];
                            int x0 = rQ;
                            ringEnsure<R, true>(c, rx, x0 - 1, x0 + S - 2, false);
                            ringEnsure<R, false>(c, ry, -rQ - S, -rQ - 1, false);
                            loadSlots<C, R>(c, rx, ry, 0, rQ, rsy);
                            rHave = true;
                            forwardOrigin<C>(c, startP, rQ, rs, F[k]);
#pragma unroll
                            for (int j = 0; j < C; j++) {
                                EM[k][j] = 0.0f;
                                EXc[k][j] = rsy.ex[j];
                                EYc[k][j] = rsy.ey[j];
                            }
                            sLoK[k] = (bz.x >> 1) - rQ;
                            sHiK[k] = (bz.y >> 1) - rQ;
                            const unsigned span0 = (unsigned) (sHiK[k] - sLoK[k]);
#pragma unroll
                            for (int j = 0; j < C; j++)
                                inbK |= (((unsigned) (lane * C + j - sLoK[k]) <= span0) ? 1u : 0u) << (k * C + j);
                            continue;
                        }
                        int4 bd2 = c.band[dd];
                        int dl2 = windowShift<C>(rQ, bd2.z, bd2.w, &bad);
                        if (dl2 != 0) {
                            shiftForward<C>(rs, dl2, lane);
                            rQ += C * dl2;
                            rHave = false;
                        }
                        shiftAt[k] = dl2;
                        int x0 = rQ + ((dd + 1) >> 1);
                        int y0 = dd - x0;
                        ringEnsure<R, true>(c, rx, x0 - 1, x0 + S - 2, false);
                        ringEnsure<R, false>(c, ry, y0 - S, y0 - 1, false);
                        if (!rHave) {
                            loadSlots<C, R>(c, rx, ry, dd, rQ, rsy);
                            rHave = true;
                        } else {
                            stepSlots<C, R>(c, rx, ry, dd, rQ, rsy);
                        }
                        sLoK[k] = (bd2.x >> 1) - rQ;
                        sHiK[k] = (bd2.y >> 1) - rQ;
                        if (dd & 1)
                            forwardDiagonal<C, 1>(c, rpBase, rs, rsy, sLoK[k], sHiK[k], F[k], EM[k], inbK, k * C);
                        else
                            forwardDiagonal<C, 0>(c, rpBase, rs, rsy, sLoK[k], sHiK[k], F[k], EM[k], inbK, k * C);
#pragma unroll
                        for (int j = 0; j < C; j++) {
                            EXc[k][j] = rsy.ex[j];
                            EYc[k][j] = rsy.ey[j];
                        }
                    }
                }
                if (bad) break;
                // -------- backward over this block, top to bottom --------
                // bring the carried backward state from the window of dStart+K to that of dEnd
                if (carryShift != 0) {
                    laneShift<C>(gX, -carryShift, lane);
                    laneShift<C>(gY, -carryShift, lane);
                    laneShift<C>(gA, -carryShift, lane);
                    laneShift<C>(gB, -carryShift, lane);
                }
#pragma unroll
                for (int k = K - 1; k >= 0; k--) {
                    const int dd = dStart + k;
                    if (dd <= dEnd && dd > tracedBackTo) {
                        if (k < K - 1 && dStart + k + 1 <= dEnd && shiftAt[k + 1] != 0) {
                            laneShift<C>(gX, -shiftAt[k + 1], lane);
                            laneShift<C>(gY, -shiftAt[k + 1], lane);
                            laneShift<C>(gA, -shiftAt[k + 1], lane);
                            laneShift<C>(gB, -shiftAt[k + 1], lane);
                        }
                        float bM[C], bX[C], bY[C];
                        if (dd == D) {
                            const float *endP = (atEnd && raggedR) ? dm.raggedEnd : dm.end;
#pragma unroll
                            for (int j = 0; j < C; j++) {
                                bool in = (inbK >> (k * C + j)) & 1u;
                                bM[j] = in ? endP[0] : 0.0f;
                                bX[j] = in ? endP[1] : 0.0f;
                                bY[j] = in ? endP[2] : 0.0f;
                            }
                        } else {
                            float sX[C], sY[C];
                            if (dd & 1) {  // odd: gap-x successor slot i+1, gap-y successor slot i
                                float nb = __shfl_down_sync(FULL_MASK, gX[0], 1);
                                if (lane == 31) nb = 0.0f;
#pragma unroll
                                for (int j = 0; j < C; j++) {
                                    sX[j] = (j < C - 1) ? gX[j + 1] : nb;
                                    sY[j] = gY[j];
                                }
                            } else {  // even: gap-x successor slot i, gap-y successor slot i-1
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
                                float sm = (dd & 1) ? gB[j] : gA[j];
                                bool in = (inbK >> (k * C + j)) & 1u;
                                float m_ = __fmaf_rn(c.t[0 * 3 + 0], sm, __fmaf_rn(c.t[0 * 3 + 2], sY[j], c.t[0 * 3 + 1] * sX[j]));
                                float x_ = __fmaf_rn(c.t[1 * 3 + 0], sm, __fmaf_rn(c.t[1 * 3 + 2], sY[j], c.t[1 * 3 + 1] * sX[j]));
                                float y_ = __fmaf_rn(c.t[2 * 3 + 0], sm, __fmaf_rn(c.t[2 * 3 + 2], sY[j], c.t[2 * 3 + 1] * sX[j]));
                                bM[j] = in ? m_ : 0.0f;
                                bX[j] = in ? x_ : 0.0f;
                                bY[j] = in ? y_ : 0.0f;
                            }
                        }
                        // posteriors of this diagonal
                        if (dd <= tbFrom) {
                            if (posts % 10 == 0) {
                                // total: sum over cells of f.b plus match transitions crossing dd
                                float sMd1[C];
#pragma unroll
                                for (int j = 0; j < C; j++) {
                                    if (k > 0) {
                                        sMd1[j] = __fmaf_rn(c.t[2 * 3 + 0], F[k > 0 ? k - 1 : 0][j].fY,
                                                            __fmaf_rn(c.t[1 * 3 + 0], F[k > 0 ? k - 1 : 0][j].fX,
                                                                      c.t[0 * 3 + 0] * F[k > 0 ? k - 1 : 0][j].fM));
                                    } else {
                                        sMd1[j] = chkSM[j];
                                    }
                                }
                                if (shiftAt[k] != 0) laneShift<C>(sMd1, shiftAt[k], lane);
                                float part = 0.0f;
#pragma unroll
                                for (int j = 0; j < C; j++) {
                                    float uMn = (dd & 1) ? gA[j] : gB[j];  // match u of dd+1
                                    part = __fmaf_rn(F[k][j].fM, bM[j], part);
                                    part = __fmaf_rn(F[k][j].fX, bX[j], part);
                                    part = __fmaf_rn(F[k][j].fY, bY[j], part);
                                    part = __fmaf_rn(uMn, sMd1[j], part);
                                }
                                float T = warpSum(part);
                                if (T > 0.0f) {
                                    int e = exponentOf(T);
                                    Tm = T * pow2f(-e);
                                    ET = rEf + Eb + e;
                                } else {
                                    Tm = 0.0f;
                                    ET = 0;
                                }
                                if (atEnd && posts == 0) {
                                    logLik += (Tm > 0.0f) ? (log((double) Tm) + (double) ET * 0.69314718055994530942)
                                                          : -INFINITY;
                                }
                            }
                            posts++;
                            if (Tm > 0.0f) {
                                int ex = rEf + Eb - ET;
                                ex = max(-126, min(127, ex));
                                float scale = pow2f(ex) / Tm;
                                float p[3][C];
#pragma unroll
                                for (int j = 0; j < C; j++) {
                                    p[0][j] = (F[k][j].fM * bM[j]) * scale;
                                    p[1][j] = (F[k][j].fX * bX[j]) * scale;
                                    p[2][j] = (F[k][j].fY * bY[j]) * scale;
                                }
                                int x0 = rQ + ((dd + 1) >> 1);
                                // rQ is the window of the block's last diagonal; slots of dd use its own window
                                int qd = rQ;
#pragma unroll
                                for (int kk = K - 1; kk > 0; kk--) {
                                    if (kk > k && dStart + kk <= dEnd) qd -= C * shiftAt[kk];
                                }
                                x0 = qd + ((dd + 1) >> 1);
                                emitDiagonal<C>(lane, oc, p, thr, x0, dd, xOutShift, yOutShift);
                            }
                        }
                        // u-values of dd for the diagonals below
#pragma unroll
                        for (int j = 0; j < C; j++) {
                            gX[j] = EXc[k][j] * bX[j];
                            gY[j] = EYc[k][j] * bY[j];
                            float uM = EM[k][j] * bM[j];
                            if (dd & 1) gB[j] = uM; else gA[j] = uM;
                        }
                    }
                }
                carryShift = shiftAt[0];
                // rescale the carried backward state at the block boundary
                {
                    float m = 0.0f;
#pragma unroll
                    for (int j = 0; j < C; j++) m = fmaxf(m, fmaxf(fmaxf(gX[j], gY[j]), fmaxf(gA[j], gB[j])));
                    m = warpMax(m);
                    if (m > 0.0f) {
                        int kx = exponentOf(m);
                        float sc = pow2f(-kx);
#pragma unroll
                        for (int j = 0; j < C; j++) {
                            gX[j] *= sc;
                            gY[j] *= sc;
                            gA[j] *= sc;
                            gB[j] *= sc;
                        }
                        Eb += kx;
                    }
                }
            }
            tracedBackTo = tbFrom;
            if (!atEnd && !bad) {
                // resume the sweep after D
                loadCheckpoint<C>(resumeBase, lane, st);
                haveSlots = false;
            }
        }
        d++;
    }

    if (lane == 0) {
        int s = status;
        if (bad) s |= kTaskWindow;
        if (rx.bad | ry.bad) s |= kTaskSymbol;
        for (int k = 0; k < 3; k++) {
            to->count[k] = bad ? 0 : oc.written[k];
            if (!bad && oc.written[k] > oc.top[k]) s |= kTaskCapacity;
        }
        to->status = s;
        to->logLik = logLik;
    }
}

template <int C, int K, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) posteriorKernel(DpArgs a, int warpsPerBlock) {
    constexpr int R = Geometry<C>::R;
    extern __shared__ __align__(16) unsigned char smemRaw[];
    float *rp = reinterpret_cast<float *>(smemRaw);
    float *sm = rp + 2 * kRepTable;
    float *gx = sm + 2 * 25;
    float *gy = gx + 2 * 5;
    uint2 *rings = reinterpret_cast<uint2 *>(gy + 2 * 5 + 2);  // 8-byte aligned (offset is even in floats)
    // stage tables
    for (int i = threadIdx.x; i < 2 * kRepTable; i += blockDim.x) rp[i] = a.repeatProb[i];
    for (int i = threadIdx.x; i < 2 * 25; i += blockDim.x) sm[i] = a.models[i / 25].match[i % 25];
    for (int i = threadIdx.x; i < 2 * 5; i += blockDim.x) {
        gx[i] = a.models[i / 5].gapX[i % 5];
        gy[i] = a.models[i / 5].gapY[i % 5];
    }
    __syncthreads();
    SharedTables tab{rp, sm, gx, gy};

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * warpsPerBlock + warp;
    Ring<R> rx{rings + (size_t) warp * 2 * R, 0, 0};
    Ring<R> ry{rings + (size_t) warp * 2 * R + R, 0, 0};
    float4 *chkBase = a.scratch + (size_t) gwarp * a.scratchBlocks * (C * 32);
    int2 *chkScal = a.scratchScalars + (size_t) gwarp * a.scratchBlocks;
    float4 *resumeBase = a.resume + (size_t) gwarp * (C * 32);

    while (true) {
        int t = 0;
        if (lane == 0) t = atomicAdd(a.queue, 1);
        t = __shfl_sync(FULL_MASK, t, 0);
        if (t >= a.nTasks) break;
        runTask<C, K>(a, tab, a.order[t], rx, ry, chkBase, chkScal, resumeBase);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Band kernel: per task, (xmyL, xmyR) of every anti-diagonal from the anchor
// boxes (impl/pairwiseAligner.c:96-173), then the hull of d-2..d+2.
// One warp per task; each lane walks one anchor box at a time.
// ---------------------------------------------------------------------------

__device__ __forceinline__ bool boxDiagonal(int d, int xL, int yL, int xU, int yU, int &lo, int &hi) {
    int l = xL - yL, h = xU - yU;
    if ((d + l) & 1) l++;
    if ((d + h) & 1) h++;
    int x = (d + l) / 2;
    if (x < xL) l += 2 * (xL - x);
    int y = (d - l) / 2;
    if (yL < y) l += 2 * (y - yL);
    x = (d + h) / 2;
    if (xU < x) h -= 2 * (x - xU);
    y = (d - h) / 2;
    if (y < yU) h -= 2 * (yU - y);
    lo = l;
    hi = h;
    return l <= h;
}

__device__ __forceinline__ int clampCoord(int z, int lz) {
    return z < 0 ? 0 : (z > lz ? lz : z);
}

__global__ void bandKernel(BandArgs a) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= a.nTasks) return;
    const Task &tk = a.tasks[t];
    const int lx = tk.lx, ly = tk.ly, N = lx + ly;
    const int nA = tk.nAnchors;
    const int32_t *an = a.anchors + 3 * tk.anchorOff;
    int2 *band = a.band + 2 * tk.bandOff;  // int4 records viewed as pairs: [2d] = (lo, hi)
    const bool dynamic = tk.flags & 8;
    long long cells = 0;
    bool ok = true;
    if (lane == 0) {
        band[0] = make_int2(0, 0);
        cells += N > 0 ? 1 : 0;  // an empty sub-problem computes nothing (impl/pairwiseAligner.c:698-701)
    }
    for (int k0 = 0; k0 <= nA; k0 += 32) {
        int k = k0 + lane;
        if (k <= nA && N > 0) {
            int px = 0, py = 0, nx, ny, e;
            if (k > 0) {
                px = an[3 * (k - 1)] - tk.x1 + 1;
                py = an[3 * (k - 1) + 1] - tk.y1 + 1;
            }
            if (k < nA) {
                nx = an[3 * k] - tk.x1 + 1;
                ny = an[3 * k + 1] - tk.y1 + 1;
                e = dynamic ? an[3 * k + 2] : tk.expansion;
            } else {
                nx = lx;
                ny = ly;
                e = dynamic ? (nA > 0 ? an[3 * (nA - 1) + 2] : 0) : tk.expansion;
            }
            int pxay = px + py, pxmy = px - py, nxay = nx + ny, nxmy = nx - ny;
            int xL = clampCoord((pxay + (pxmy - e)) / 2, lx);
            int yL = clampCoord((nxay - (nxmy - e)) / 2, ly);
            int xU = clampCoord((nxay + (nxmy + e)) / 2, lx);
            int yU = clampCoord((pxay - (pxmy + e)) / 2, ly);
            int dEnd = min(nxay, N);
            for (int dd = pxay + 1; dd <= dEnd; dd++) {
                int lo, hi;
                if (!boxDiagonal(dd, xL, yL, xU, yU, lo, hi)) {
                    ok = false;
                    lo = 0;
                    hi = 0;
                }
                band[2 * dd] = make_int2(lo, hi);
                cells += ((hi - lo) >> 1) + 1;
            }
        }
    }
    // reduce cells and validity
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cells += __shfl_xor_sync(FULL_MASK, cells, o);
    bool allOk = __all_sync(FULL_MASK, ok);
    if (lane == 0) {
        a.out[t].cells = cells;
        a.out[t].status = allOk ? 0 : kTaskBand;
    }
}

// Hull of the bands of d-2..d+2 (clamped to the task), written into the second
// pair of each diagonal record. One warp per task, lanes stride over diagonals.
__global__ void hullKernel(BandArgs a) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= a.nTasks) return;
    const Task &tk = a.tasks[t];
    const int N = tk.lx + tk.ly;
    int2 *band = a.band + 2 * tk.bandOff;
    for (int d = lane; d <= N; d += 32) {
        int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
        for (int k = -2; k <= 2; k++) {
            int e = d + k;
            if (e < 0 || e > N) continue;
            int2 v = band[2 * e];
            lo = min(lo, v.x);
            hi = max(hi, v.y);
        }
        band[2 * d + 1] = make_int2(lo, hi);
    }
}

// ---------------------------------------------------------------------------
// Compaction: gathers each task's tuples (top of its region) into the final
// per-job layout (tasks of a job are consecutive, in split order).
// ---------------------------------------------------------------------------

__global__ void compactKernel(const Task *tasks, const TaskOut *out, int nTasks, const int64_t *dst0,
                              const int64_t *dst1, const int64_t *dst2, int32_t *const *srcW, int32_t *const *srcX,
                              int32_t *const *srcY, int32_t *const *dstW, int32_t *const *dstX,
                              int32_t *const *dstY) {
    const int k = blockIdx.y;
    const int t = blockIdx.x;
    if (t >= nTasks) return;
    const Task &tk = tasks[t];
    const int n = out[t].count[k];
    const int64_t *dst = k == 0 ? dst0 : (k == 1 ? dst1 : dst2);
    const int64_t from = tk.outOff[k] + tk.cap[k] - n;
    const int64_t to = dst[t];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        dstW[k][to + i] = srcW[k][from + i];
        dstX[k][to + i] = srcX[k][from + i];
        dstY[k][to + i] = srcY[k][from + i];
    }
}

// ---------------------------------------------------------------------------
// FP32 FMA throughput probe: 16 independent FMA chains per thread.
// ---------------------------------------------------------------------------

__global__ void fmaProbeKernel(float *out, int iters) {
    float a[16];
    const float m = 1.0000001f, c = 1e-7f;
#pragma unroll
    for (int k = 0; k < 16; k++) a[k] = (float) (threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) a[k] = __fmaf_rn(a[k], m, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; k++) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t launchFmaProbe(float *out, int blocks, int threads, int iters, cudaStream_t s) {
    fmaProbeKernel<<<blocks, threads, 0, s>>>(out, iters);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host-side launch wrappers
// ---------------------------------------------------------------------------

template <int C>
static size_t posteriorSmem(int warps) {
    constexpr int R = Geometry<C>::R;
    size_t tables = sizeof(float) * (2 * kRepTable + 2 * 25 + 2 * 5 + 2 * 5 + 2);
    return tables + (size_t) warps * 2 * R * sizeof(uint2);
}

template <int C, int K, int MAXT>
static cudaError_t launchPosteriorT(const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    if (warps * 32 > MAXT) return cudaErrorInvalidValue;
    size_t smem = posteriorSmem<C>(warps);
    cudaError_t e = cudaFuncSetAttribute(posteriorKernel<C, K, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) smem);
    if (e != cudaSuccess) return e;
    posteriorKernel<C, K, MAXT><<<blocks, warps * 32, smem, s>>>(a, warps);
    return cudaGetLastError();
}

// Slot classes: C slots per lane (window S = 32*C), checkpoint stride K, threads per block bound.
int classStride(int C) {
    return C <= 4 ? 4 : 2;
}

int classMaxWarps(int C) {
    return C <= 2 ? 16 : 8;
}

size_t posteriorSmemBytes(int C, int warps) {
    switch (C) {
        case 2: return posteriorSmem<2>(warps);
        case 3: return posteriorSmem<3>(warps);
        case 4: return posteriorSmem<4>(warps);
        case 6: return posteriorSmem<6>(warps);
        case 8: return posteriorSmem<8>(warps);
        default: return 0;
    }
}

cudaError_t launchPosterior(int C, const DpArgs &a, int blocks, int warps, cudaStream_t s) {
    switch (C) {
        case 2: return launchPosteriorT<2, 4, 512>(a, blocks, warps, s);
        case 3: return launchPosteriorT<3, 4, 256>(a, blocks, warps, s);
        case 4: return launchPosteriorT<4, 4, 256>(a, blocks, warps, s);
        case 6: return launchPosteriorT<6, 2, 256>(a, blocks, warps, s);
        case 8: return launchPosteriorT<8, 2, 256>(a, blocks, warps, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchBand(const BandArgs &a, cudaStream_t s) {
    if (a.nTasks == 0) return cudaSuccess;
    int threads = 256;
    int blocks = (a.nTasks * 32 + threads - 1) / threads;
    bandKernel<<<blocks, threads, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    hullKernel<<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launchCompact(const Task *tasks, const TaskOut *out, int nTasks, const int64_t *dst0,
                          const int64_t *dst1, const int64_t *dst2, int32_t *const *srcW, int32_t *const *srcX,
                          int32_t *const *srcY, int32_t *const *dstW, int32_t *const *dstX, int32_t *const *dstY,
                          cudaStream_t s) {
    if (nTasks == 0) return cudaSuccess;
    dim3 grid(nTasks, 3);
    compactKernel<<<grid, 128, 0, s>>>(tasks, out, nTasks, dst0, dst1, dst2, srcW, srcX, srcY, dstW, dstX, dstY);
    return cudaGetLastError();
}

}  // namespace mp
