// Auxiliary device kernels of the realignment engine (sm_100a): anchor band
// construction (impl/pairwiseAligner.c:96-173) with its 5-diagonal hull in one pass, the
// per-job compaction of posterior tuples, and an FP32 FMA throughput probe.
// The posterior kernel itself is in mp_posterior.cu.
#include "mp_internal.h"

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

// Band and hull in one pass. One warp per task; lane l takes anti-diagonal d = base + l of
// each step of 32. The anchor boxes follow each other along x+y: box k covers the diagonals
// (e_{k-1}, e_k] with e_k = (x_k + 1) + (y_k + 1) in sub-problem coordinates (e_nA = N), so the
// 32 boxes from the one holding `base` (each covers at least 2 diagonals) hold every diagonal
// of the step: a lane finds its box by a binary search over the boxes' ends held across the
// warp. The raw band of d (impl/pairwiseAligner.c:96-173) and the hull of d-2..d+2 are then
// written as one 16-byte record, in window-slot units: x-y = 2*slot + (d&1), slot = (x-y) >> 1.
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
    int kb = 0;                        // box holding the step's first diagonal (diagonal 0: box 0)
    int2 below1 = none, below2 = none; // raw bands of base-1 and base-2
    for (int base = 0; base <= N; base += 32) {
        // lane i: box kb + i
        const int k = kb + lane;
        int end = INT_MAX, xL = 0, yL = 0, xU = 0, yU = 0;
        if (k <= nA) {
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
        // raw band of diagonal dd (0 <= dd <= N); `box` receives its box offset from kb
        auto rawBand = [&](int dd, int &box) -> int2 {
            int pos = 0;  // first loaded box whose end >= dd
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int v = __shfl_sync(FULL_MASK, end, pos + step - 1);
                if (v < dd) pos += step;
            }
            box = pos;
            const int bxL = __shfl_sync(FULL_MASK, xL, pos), byL = __shfl_sync(FULL_MASK, yL, pos);
            const int bxU = __shfl_sync(FULL_MASK, xU, pos), byU = __shfl_sync(FULL_MASK, yU, pos);
            if (dd == 0) return make_int2(0, 0);
            int lo, hi;
            if (!boxDiagonal(dd, bxL, byL, bxU, byU, lo, hi)) {
                ok = false;
                return make_int2(0, 0);
            }
            return make_int2(lo, hi);
        };
        const int d = base + lane;
        int box0 = 0, boxUp = 0;
        const int2 v = d <= N ? rawBand(d, box0) : (rawBand(N, box0), none);
        // diagonals base+32 and base+33 (the hull of the step's last two lanes needs them)
        const int du = base + 32 + (lane & 1);
        const int2 up = du <= N ? rawBand(du, boxUp) : (rawBand(N, boxUp), none);
        if (d <= N && N > 0) cells += ((v.y - v.x) >> 1) + 1;  // an empty sub-problem computes nothing
        int2 n[4];  // raw bands of d-2, d-1, d+1, d+2
        const int offs[4] = {-2, -1, 1, 2};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int src = lane + offs[q];
            int2 w;
            w.x = __shfl_sync(FULL_MASK, v.x, src & 31);
            w.y = __shfl_sync(FULL_MASK, v.y, src & 31);
            const int2 ab = make_int2(__shfl_sync(FULL_MASK, up.x, src & 1), __shfl_sync(FULL_MASK, up.y, src & 1));
            if (src < 0) w = src == -1 ? below1 : below2;
            if (src > 31) w = ab;
            const int e = d + offs[q];
            n[q] = (e < 0 || e > N) ? none : w;
        }
        int lo = v.x, hi = v.y;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            lo = min(lo, n[q].x);
            hi = max(hi, n[q].y);
        }
        if (d <= N) rec[d] = make_int4(v.x >> 1, v.y >> 1, lo >> 1, hi >> 1);
        below1 = make_int2(__shfl_sync(FULL_MASK, v.x, 31), __shfl_sync(FULL_MASK, v.y, 31));
        below2 = make_int2(__shfl_sync(FULL_MASK, v.x, 30), __shfl_sync(FULL_MASK, v.y, 30));
        // the next step starts at the box of diagonal base + 32
        kb += __shfl_sync(FULL_MASK, boxUp, 0);
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
// per-job layout (tasks of a job are consecutive, in split order).
// ---------------------------------------------------------------------------

__global__ void compactKernel(CompactArgs a) {
    const int k = blockIdx.y;
    const int t = blockIdx.x;
    if (t >= a.nTasks) return;
    const Task &tk = a.tasks[t];
    const int n = a.out[t].count[k];
    const int64_t from = tk.outOff[k] + tk.cap[k] - n;
    const int64_t to = a.dst[k] ? a.dst[k][t] : 0;
    const int4 *src = a.src[k] + from;
    int32_t *w = a.w[k] + to, *x = a.x[k] + to, *y = a.y[k] + to;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int4 v = src[i];
        w[i] = v.x;
        x[i] = v.y;
        y[i] = v.z;
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

cudaError_t launchBand(const BandArgs &a, cudaStream_t s) {
    if (a.nTasks == 0) return cudaSuccess;
    int threads = 256;
    int blocks = (a.nTasks * 32 + threads - 1) / threads;
    bandHullKernel<<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launchCompact(const CompactArgs &a, cudaStream_t s) {
    if (a.nTasks == 0) return cudaSuccess;
    dim3 grid(a.nTasks, 3);
    compactKernel<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mp
