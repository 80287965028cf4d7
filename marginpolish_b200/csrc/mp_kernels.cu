// Auxiliary device kernels of the realignment engine (sm_100a): anchor band
// construction (impl/pairwiseAligner.c:96-173) with its 5-diagonal hull in one pass, the
// per-job compaction of posterior tuples, and an FP32 FMA throughput probe.
// The posterior kernel itself is in mp_posterior.cu.
#include "mp_internal.h"

#include <algorithm>
#include <cstdio>

namespace mp {

#define FULL_MASK 0xffffffffu

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

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

// Band and hull in one pass. One warp per task; lane l computes the raw band of anti-diagonal
// d = base + l of each step of 32 (impl/pairwiseAligner.c:96-173). The anchor boxes follow
// each other along x+y: box k covers the diagonals (e_{k-1}, e_k] with e_k = (x_k + 1) +
// (y_k + 1) in sub-problem coordinates (e_nA = N). The 32 boxes from the one holding `base`
// (each covers at least 2 diagonals) hold every diagonal of the step: lane i holds box kb+i,
// the step's box ends are gathered into one bit mask (one warp OR), and the box of d is the
// count of ends before it. The hull of d-2..d+2 needs the next two diagonals, so each step
// writes the records of base-2 .. base+29 (a last step writes the remainder), one 16-byte
// store per diagonal, in window-slot units: x-y = 2*slot + (d&1), slot = (x-y) >> 1.
__global__ void bandHullKernel(BandArgs a) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= a.nTasks) return;
    const Task &tk = a.tasks[t];
    const int lx = tk.lx, ly = tk.ly, N = lx + ly;
    const int nA = tk.nAnchors;
    const int32_t *an = a.anchors + 3 * tk.anchorOff;
    int4 *rec = reinterpret_cast<int4 *>(a.band) + tk.bandOff;
    const bool dynamic = tk.flags & 8;
    const int2 none = make_int2(INT_MAX, INT_MIN);
    long long cells = 0;
    bool ok = true;
    int kb = 0;             // box holding the step's first diagonal (diagonal 0: box 0)
    int2 prev = none;       // this lane's raw band in the previous step
    for (int base = 0; base <= N + 2; base += 32) {
        // lane i: box kb + i
        const int k = kb + lane;
        int end = INT_MAX, xL = 0, yL = 0, xU = 0, yU = 0;
        if (k <= nA && base <= N) {
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
            const int pxay = px + py, pxmy = px - py, nxay = nx + ny, nxmy = nx - ny;
            xL = clampCoord((pxay + (pxmy - e)) / 2, lx);
            yL = clampCoord((nxay - (nxmy - e)) / 2, ly);
            xU = clampCoord((nxay + (nxmy + e)) / 2, lx);
            yU = clampCoord((pxay - (pxmy + e)) / 2, ly);
            end = k < nA ? nxay : N;
        }
        // ends within the step (box kb ends at or after base, so none is before it)
        const int m = end - base;
        const unsigned ends = __reduce_or_sync(FULL_MASK, (m >= 0 && m < 32) ? 1u << m : 0u);
        const int box = __popc(ends & ((1u << lane) - 1u));  // boxes ending before d
        const int bxL = __shfl_sync(FULL_MASK, xL, box), byL = __shfl_sync(FULL_MASK, yL, box);
        const int bxU = __shfl_sync(FULL_MASK, xU, box), byU = __shfl_sync(FULL_MASK, yU, box);
        const int d = base + lane;
        int2 v = none;
        if (d == 0) {
            v = make_int2(0, 0);
        } else if (d <= N) {
            int lo, hi;
            if (!boxDiagonal(d, bxL, byL, bxU, byU, lo, hi)) {
                ok = false;
                lo = hi = 0;
            }
            v = make_int2(lo, hi);
        }
        if (d <= N && N > 0) cells += ((v.y - v.x) >> 1) + 1;  // an empty sub-problem computes nothing
        // record of diagonal f = base - 2 + lane: raw bands of f-2 .. f+2 = base-4+lane .. base+lane
        const int f = d - 2;
        int2 w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const int src = lane + q - 4;
            const int2 cur = make_int2(__shfl_sync(FULL_MASK, v.x, src & 31), __shfl_sync(FULL_MASK, v.y, src & 31));
            const int2 old = make_int2(__shfl_sync(FULL_MASK, prev.x, src & 31), __shfl_sync(FULL_MASK, prev.y, src & 31));
            w[q] = src >= 0 ? cur : old;
        }
        if (f >= 0 && f <= N) {
            int lo = w[2].x, hi = w[2].y;
#pragma unroll
            for (int q = 0; q < 5; q++) {  // diagonals outside 0..N hold `none`
                lo = min(lo, w[q].x);
                hi = max(hi, w[q].y);
            }
            rec[f] = make_int4(w[2].x >> 1, w[2].y >> 1, lo >> 1, hi >> 1);
        }
        prev = v;
        // the next step starts at the box of diagonal base + 32
        kb += __popc(__ballot_sync(FULL_MASK, m < 32));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cells += __shfl_xor_sync(FULL_MASK, cells, o);
    const bool allOk = __all_sync(FULL_MASK, ok);
    if (lane == 0) {
        a.out[t].cells = cells;
        a.out[t].status = allOk ? 0 : kTaskBand;
    }
}

// ---------------------------------------------------------------------------
// Compaction: gathers each task's tuples (top of its region) into the final
// per-job layout (tasks of a job are consecutive, in split order). A small grid of warps
// walks the (task, list) items: the compaction often shares the SMs with posterior blocks of
// other batches, so it asks for few blocks and no shared memory.
// ---------------------------------------------------------------------------

__global__ void compactKernel(CompactArgs a) {
    // one warp per (task, list) item, items strided over the grid's warps
    const int lane = threadIdx.x & 31;
    const int nItems = 3 * a.nTasks;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < nItems; item += warps) {
        const int t = item / 3, k = item - 3 * t;
        const Task &tk = a.tasks[t];
        const int n = a.out[t].count[k];
        const int64_t from = tk.outOff[k] + tk.cap[k] - n;
        const int64_t to = a.dst[k] ? a.dst[k][t] : 0;
        const int4 *src = a.src[k] + from;
        int32_t *w = a.w[k] + to, *x = a.x[k] + to, *y = a.y[k] + to;
        for (int i = lane; i < n; i += 32) {
            const int4 v = src[i];
            w[i] = v.x;
            x[i] = v.y;
            y[i] = v.z;
        }
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

// FP64 issue rate: 16 independent chains of separately rounded adds and products per thread
// (the operations the bubble scorer is made of).
__global__ void dpProbeKernel(double *out, int iters) {
    double a[16];
    const double m = 1.0000001, c = 1e-7;
#pragma unroll
    for (int k = 0; k < 16; k++) a[k] = (double) (threadIdx.x + k) * 1e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) a[k] = (k & 1) ? __dmul_rn(a[k], m) : __dadd_rn(a[k], c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 16; k++) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t launchDpProbe(double *out, int blocks, int threads, int iters, cudaStream_t s) {
    dpProbeKernel<<<blocks, threads, 0, s>>>(out, iters);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host-side launch wrappers
// ---------------------------------------------------------------------------

cudaError_t launchBand(const BandArgs &a, cudaStream_t s) {
    if (a.nTasks == 0) return cudaSuccess;
    int threads = 256;
    int blocks = (a.nTasks * 32 + threads - 1) / threads;
    bandHullKernel<<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

// Task statuses into mapped page-locked host memory (16-byte words; a TaskOut is two).
__global__ void statusCopyKernel(const int4 *src, int4 *dst, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

cudaError_t launchStatusCopy(const TaskOut *src, TaskOut *dst, int nTasks, cudaStream_t s) {
    static_assert(sizeof(TaskOut) == 32, "a task status is two 16-byte words");
    const int n = 2 * nTasks;
    const int blocks = std::min(148, (n + 255) / 256);
    statusCopyKernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const int4 *>(src), reinterpret_cast<int4 *>(dst), n);
    return cudaGetLastError();
}

cudaError_t launchCompact(const CompactArgs &a, cudaStream_t s) {
    if (a.nTasks == 0) return cudaSuccess;
    const int items = 3 * a.nTasks;                      // warps of work
    const int blocks = std::min(4 * 148, (items + 7) / 8);  // 8 warps a block
    compactKernel<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mp
