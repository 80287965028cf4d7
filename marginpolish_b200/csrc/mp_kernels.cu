// Auxiliary device kernels of the realignment engine (sm_100a): anchor band
// construction (impl/pairwiseAligner.c:96-173) and its 5-diagonal hull, the
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

// Hull of the bands of d-2..d+2 (clamped to the task), then every record is
// converted to window-slot units: x-y = 2*slot + (d&1), so slot = (x-y) >> 1 (floor)
// for both the band and the hull of the diagonal. One warp per task, lanes stride
// over diagonals; the raw bands of the two diagonals below each 32-diagonal chunk
// are carried in registers because the chunk before has already been converted.
__global__ void hullKernel(BandArgs a) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= a.nTasks) return;
    const Task &tk = a.tasks[t];
    const int N = tk.lx + tk.ly;
    int2 *band = a.band + 2 * tk.bandOff;
    const int2 none = make_int2(INT_MAX, INT_MIN);
    int2 below1 = none, below2 = none;  // raw bands of base-1 and base-2
    for (int base = 0; base <= N; base += 32) {
        const int d = base + lane;
        const int2 v = d <= N ? band[2 * d] : none;
        // the two diagonals above the chunk are not converted yet
        const int2 above = (lane < 2 && base + 32 + lane <= N) ? band[2 * (base + 32 + lane)] : none;
        int2 n[4];  // bands of d-2, d-1, d+1, d+2
        const int offs[4] = {-2, -1, 1, 2};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int src = lane + offs[q];
            int2 w;
            w.x = __shfl_sync(FULL_MASK, v.x, src & 31);
            w.y = __shfl_sync(FULL_MASK, v.y, src & 31);
            const int2 ab = make_int2(__shfl_sync(FULL_MASK, above.x, src & 1),
                                      __shfl_sync(FULL_MASK, above.y, src & 1));
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
        below1 = make_int2(__shfl_sync(FULL_MASK, v.x, 31), __shfl_sync(FULL_MASK, v.y, 31));
        below2 = make_int2(__shfl_sync(FULL_MASK, v.x, 30), __shfl_sync(FULL_MASK, v.y, 30));
        __syncwarp();
        if (d <= N) {
            band[2 * d] = make_int2(v.x >> 1, v.y >> 1);
            band[2 * d + 1] = make_int2(lo >> 1, hi >> 1);
        }
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
    bandKernel<<<blocks, threads, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    hullKernel<<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launchCompact(const CompactArgs &a, cudaStream_t s) {
    if (a.nTasks == 0) return cudaSuccess;
    dim3 grid(a.nTasks, 3);
    compactKernel<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mp
