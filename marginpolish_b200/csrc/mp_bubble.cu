// Bubble scoring: the forward likelihood of many small (allele, read substring) pairs in the
// reference's own arithmetic.
//
// The polish step's bubble graph (MarginPolish impl/bubbleGraph.c:905-955) scores every allele
// of a bubble against every distinct read substring with computeForwardProbability
// (impl/pairwiseAligner.c:813-865): no anchors, so the band is the whole matrix, and no ragged
// ends. The reference keeps its cells as FP64 natural logs and sums them with an approximate
// log-sum (impl/pairwiseAligner.c:279-299, a four-piece cubic of the difference); the allele
// choice compares sums of these values. To make the same choices this kernel computes the same
// numbers: FP64 log cells, the same cubic with the coefficients as the reference writes them
// (single-precision literals widened to double), the same grouping f + (e + t) and the same
// order of the three incoming terms of every state (the reference's stateMachine3_cellCalculate,
// impl/stateMachine.c:559-581). Every addition and product is rounded on its own
// (__dadd_rn / __dmul_rn) so that no fused multiply-add changes a bit. The cells are visited row
// by row instead of by anti-diagonal; each cell reads only its three neighbours, so the values
// are the same.
//
// Layout: one thread per pair. A thread keeps one row of the matrix (3 states per column) and
// sweeps the read: column x of row y needs (x-1, y) (the value it just wrote, in registers),
// (x, y-1) and (x-1, y-1) (the row before, in the row array, the latter saved in a register
// before it is overwritten). For alleles of at most 16, 32 or 64 runs the row lives in shared
// memory, thread-minor ([column][state][thread]) so that a warp's accesses fall in distinct
// banks; longer alleles use a row in global memory (L1-cached). Pairs of one bubble are adjacent
// and share their read substring and alleles of similar length, so a warp's threads run loops of
// similar length and read the same allele symbols.
//
// Roofline: FP64 issue. A cell is 4 approximate log-sums with a switch-free model (the first
// term of each state needs none; the two switch transitions are log 0) plus 19 additions: about
// 70 FP64 instructions, against B200's 2 FP64 warp instructions per clock per SM.
#include "../../include/mpgpu.h"
#include "mp_host.h"
#include "mp_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "mp_refmath.cuh"

using mp::DevLogModel;
using mp::PairArgs;

#define PAIR_TRY(expr)                 \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

namespace {

// One cell of stateMachine3_cellCalculate (impl/stateMachine.c:559-581) with doTransitionForward:
// lower (gap-x from (x-1, y)), middle (match from (x-1, y-1)), upper (gap-y from (x, y-1)); a
// missing neighbour leaves its state at LOG_ZERO. The first term of a state needs no log-sum
// (logAdd(LOG_ZERO, v) = v); without switch transitions (SW false) their terms are log 0 and
// leave the sum unchanged, so they are skipped.
template <bool SW>
__device__ __forceinline__ void cellForward(const Tables &T, const DevLogModel &m, bool lower, bool middle, bool upper,
                                            double eX, double eM, double eY, const double *l, const double *d,
                                            const double *u, double *c) {
    c[0] = c[1] = c[2] = kLogZero;
    if (lower) {
        double v = term(l[0], eX, m.t[1]);
        v = logAdd(T, v, term(l[1], eX, m.t[4]));
        if (SW) v = logAdd(T, v, term(l[2], eX, m.t[7]));
        c[1] = v;
    }
    if (middle) {
        double v = term(d[0], eM, m.t[0]);
        v = logAdd(T, v, term(d[1], eM, m.t[3]));
        v = logAdd(T, v, term(d[2], eM, m.t[6]));
        c[0] = v;
    }
    if (upper) {
        double v = term(u[0], eY, m.t[2]);
        v = logAdd(T, v, term(u[2], eY, m.t[8]));
        if (SW) v = logAdd(T, v, term(u[1], eY, m.t[5]));
        c[2] = v;
    }
}

// The match emission of the run-length model (impl/stateMachine.c:718-722): the base pair's
// log probability plus 2.3025 * log10 R[row][x run][y run] (the product precomputed on the host).
__device__ __forceinline__ double matchEmission(const DevLogModel &m, const double *rep, int xb, int repRow, int yb,
                                                int ry) {
    double e = m.match[xb * 5 + yb];
    if (m.runLength) e = __dadd_rn(e, rep[repRow + ry]);
    return e;
}

__device__ __forceinline__ int repRowOf(const DevLogModel &m, uint16_t cx, int xb) {
    if (!m.runLength) return 0;
    const int r = xb == 4 ? 0 : xb;
    const int tableRow = m.strand ? r : 3 - r;
    return (tableRow * mp::kMaxRepeat + (cx >> 8)) * mp::kMaxRepeat;
}

// The total of diagonalCalculationTotalProbability at the last diagonal
// (impl/pairwiseAligner.c:567-584), where only the cell (lx, ly) is in the band: cellDot with the
// end probabilities, then logAdd(LOG_ZERO, .).
__device__ __forceinline__ double totalAtEnd(const Tables &T, const DevLogModel &m, const double *c) {
    double v = __dadd_rn(c[0], m.end[0]);
    v = logAdd(T, v, __dadd_rn(c[1], m.end[1]));
    v = logAdd(T, v, __dadd_rn(c[2], m.end[2]));
    return logAdd(T, kLogZero, v);
}

// The row of one thread: column x, state k.
struct SharedRow {
    double *base;
    __device__ __forceinline__ double &at(int x, int k) const { return base[(x * 3 + k) * blockDim.x]; }
};

struct GlobalRow {
    double *base;
    __device__ __forceinline__ double &at(int x, int k) const { return base[x * 3 + k]; }
};

// One pair on one thread: the matrix row by row (row y = 0: the start cell, then gap-x cells;
// then per row the gap-y cell of column 0 and the full cells).
template <bool SW, class Row>
__device__ double forwardPairThread(const Tables &T, const PairArgs &a, int p, const Row &row) {
    const int lx = a.xLen[p], ly = a.yLen[p];
    if (lx + ly == 0) return 0.0;  // LOG_ONE (impl/pairwiseAligner.c:822-824)
    const DevLogModel &m = T.models[a.strand[p] ? 0 : 1];
    const double *rep = a.repeatLog + (a.strand[p] ? 0 : mp::kRepTable);
    const uint16_t *sx = a.xs + a.xOff[p];
    const uint16_t *sy = a.ys + a.yOff[p];
    const int rl = m.runLength;
    double l[3] = {m.start[0], m.start[1], m.start[2]}, c[3];
    row.at(0, 0) = l[0];
    row.at(0, 1) = l[1];
    row.at(0, 2) = l[2];
    for (int x = 1; x <= lx; x++) {
        cellForward<SW>(T, m, true, false, false, m.gapX[baseOf(sx[x - 1], rl)], 0.0, 0.0, l, l, l, c);
        l[0] = c[0], l[1] = c[1], l[2] = c[2];
        row.at(x, 0) = c[0];
        row.at(x, 1) = c[1];
        row.at(x, 2) = c[2];
    }
    for (int y = 1; y <= ly; y++) {
        const uint16_t cy = sy[y - 1];
        const int yb = baseOf(cy, rl);
        const int ry = rl ? (cy >> 8) : 0;
        const double eY = m.gapY[yb];
        double d[3] = {row.at(0, 0), row.at(0, 1), row.at(0, 2)};  // (x-1, y-1) for column 1
        cellForward<SW>(T, m, false, false, true, 0.0, 0.0, eY, d, d, d, l);
        row.at(0, 0) = l[0];
        row.at(0, 1) = l[1];
        row.at(0, 2) = l[2];
        for (int x = 1; x <= lx; x++) {
            const uint16_t cx = sx[x - 1];
            const int xb = baseOf(cx, rl);
            const double u[3] = {row.at(x, 0), row.at(x, 1), row.at(x, 2)};  // (x, y-1)
            const double eM = matchEmission(m, rep, xb, repRowOf(m, cx, xb), yb, ry);
            cellForward<SW>(T, m, true, true, true, m.gapX[xb], eM, eY, l, d, u, c);
            d[0] = u[0], d[1] = u[1], d[2] = u[2];
            l[0] = c[0], l[1] = c[1], l[2] = c[2];
            row.at(x, 0) = c[0];
            row.at(x, 1) = c[1];
            row.at(x, 2) = c[2];
        }
    }
    return totalAtEnd(T, m, l);
}

// Short alleles (at most LXMAX = 16 or 31 runs): one thread per pair, its row in shared memory;
// LXMAX = 0: any length, rows in global memory.
template <int LXMAX, bool SW>
__global__ void __launch_bounds__(128) pairThreadKernel(PairArgs a) {
    extern __shared__ double smemRows[];
    __shared__ Tables T;
    loadTables(T, a.models);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nPairs) return;
    const int p = a.pairs[i];
    double r;
    if (LXMAX > 0) {
        r = forwardPairThread<SW>(T, a, p, SharedRow{smemRows + threadIdx.x});
    } else {
        r = forwardPairThread<SW>(T, a, p, GlobalRow{a.rows + a.rowOff[i]});
    }
    a.out[p] = r;
}

// Longer alleles (32 to 32 S - 1 runs): one warp per pair, sweeping anti-diagonals. Lane l owns
// the columns x = l + 32 k (k < S) and keeps, per column, the cell it computed on the previous
// anti-diagonal; the left column's cells of the two previous anti-diagonals come by shuffles.
// Every cell is cellForward of the same neighbours as in the row sweep, so the values agree.
template <int S, bool SW>
__global__ void __launch_bounds__(128) pairWarpKernel(PairArgs a) {
    __shared__ Tables T;
    loadTables(T, a.models);
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= a.nPairs) return;  // warp-uniform
    const int p = a.pairs[i];
    const int lx = a.xLen[p], ly = a.yLen[p];
    if (lx + ly == 0) {
        if (lane == 0) a.out[p] = 0.0;
        return;
    }
    const DevLogModel &m = T.models[a.strand[p] ? 0 : 1];
    const double *rep = a.repeatLog + (a.strand[p] ? 0 : mp::kRepTable);
    const uint16_t *sx = a.xs + a.xOff[p];
    const uint16_t *sy = a.ys + a.yOff[p];
    const int rl = m.runLength;
    int xb[S], repRow[S];
    double eX[S], own[S][3], left2[S][3];
#pragma unroll
    for (int k = 0; k < S; k++) {
        const int x = lane + 32 * k;
        xb[k] = 4;
        repRow[k] = 0;
        eX[k] = 0.0;
        if (x >= 1 && x <= lx) {
            const uint16_t cx = sx[x - 1];
            xb[k] = baseOf(cx, rl);
            repRow[k] = repRowOf(m, cx, xb[k]);
            eX[k] = m.gapX[xb[k]];
        }
        own[k][0] = own[k][1] = own[k][2] = kLogZero;
        left2[k][0] = left2[k][1] = left2[k][2] = kLogZero;
    }
    if (lane == 0) {  // anti-diagonal 0: the start cell (0, 0)
        own[0][0] = m.start[0];
        own[0][1] = m.start[1];
        own[0][2] = m.start[2];
    }
    const int N = lx + ly;
    for (int dg = 1; dg <= N; dg++) {
        double left1[S][3];
#pragma unroll
        for (int k = 0; k < S; k++) {
#pragma unroll
            for (int s = 0; s < 3; s++) {
                const double up = __shfl_up_sync(0xffffffffu, own[k][s], 1);
                const double wrap = k > 0 ? __shfl_sync(0xffffffffu, own[k > 0 ? k - 1 : 0][s], 31) : kLogZero;
                left1[k][s] = lane == 0 ? wrap : up;
            }
        }
#pragma unroll
        for (int k = 0; k < S; k++) {
            const int x = lane + 32 * k, y = dg - x;
            if (x <= lx && y >= 0 && y <= ly) {
                double eY = 0.0, eM = 0.0;
                if (y >= 1) {
                    const uint16_t cy = sy[y - 1];
                    const int yb = baseOf(cy, rl);
                    eY = m.gapY[yb];
                    if (x >= 1) eM = matchEmission(m, rep, xb[k], repRow[k], yb, rl ? (cy >> 8) : 0);
                }
                double c[3];
                cellForward<SW>(T, m, x >= 1, x >= 1 && y >= 1, y >= 1, eX[k], eM, eY, left1[k], left2[k], own[k],
                                c);
                own[k][0] = c[0], own[k][1] = c[1], own[k][2] = c[2];
                if (x == lx && y == ly) a.out[p] = totalAtEnd(T, m, c);  // the last anti-diagonal's one cell
            }
            left2[k][0] = left1[k][0], left2[k][1] = left1[k][1], left2[k][2] = left1[k][2];
        }
    }
}

constexpr int kThreads = 128;
constexpr int kShortMax = 16;     // thread-per-pair class with shared-memory rows of 17 columns
constexpr int kMidMax = 31;       // the same with rows of 32 columns
constexpr int kWarpStrips = 4;    // warp-per-pair classes: alleles of up to 32 * 4 - 1 runs

// Launch classes: 0 short and 1 mid (thread, shared rows), 2..4 warp with S = 2..4 strips,
// 5 long (thread, global rows).
constexpr int kClasses = 6;

int classOf(int32_t lx) {
    if (lx <= kShortMax) return 0;
    if (lx <= kMidMax) return 1;
    if (lx < 32 * kWarpStrips) return (lx + 1 + 31) / 32;  // S = strips for columns 0..lx
    return kClasses - 1;
}

template <int LXMAX>
constexpr size_t rowBytes() {
    return sizeof(double) * 3 * (LXMAX + 1) * kThreads;
}

// Callers hold the engine's one-shot lock; the shared-memory attributes are set once per device.
template <bool SW>
cudaError_t setAttributes(int device) {
    static std::mutex lock;
    static bool granted[128] = {};
    std::lock_guard<std::mutex> g(lock);
    if (granted[device & 127]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(pairThreadKernel<kShortMax, SW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) rowBytes<kShortMax>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pairThreadKernel<kMidMax, SW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int) rowBytes<kMidMax>());
    if (e == cudaSuccess) granted[device & 127] = true;
    return e;
}

template <bool SW>
cudaError_t launchAll(PairArgs a, const int32_t *const cls[kClasses], const int32_t nCls[kClasses], int device,
                      cudaStream_t st) {
    cudaError_t e = setAttributes<SW>(device);
    if (e != cudaSuccess) return e;
    auto blocksFor = [](int32_t threads) { return (threads + kThreads - 1) / kThreads; };
    // the warp classes first (longest first): their pairs are the longest
    for (int c = kWarpStrips; c >= 2; c--) {
        if (nCls[c] == 0) continue;
        a.pairs = cls[c];
        a.nPairs = nCls[c];
        const int blocks = blocksFor(32 * nCls[c]);
        switch (c) {
            case 2: pairWarpKernel<2, SW><<<blocks, kThreads, 0, st>>>(a); break;
            case 3: pairWarpKernel<3, SW><<<blocks, kThreads, 0, st>>>(a); break;
            default: pairWarpKernel<4, SW><<<blocks, kThreads, 0, st>>>(a); break;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (nCls[kClasses - 1] > 0) {
        a.pairs = cls[kClasses - 1];
        a.nPairs = nCls[kClasses - 1];
        pairThreadKernel<0, SW><<<blocksFor(a.nPairs), kThreads, 0, st>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (nCls[1] > 0) {
        a.pairs = cls[1];
        a.nPairs = nCls[1];
        pairThreadKernel<kMidMax, SW><<<blocksFor(a.nPairs), kThreads, rowBytes<kMidMax>(), st>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (nCls[0] > 0) {
        a.pairs = cls[0];
        a.nPairs = nCls[0];
        pairThreadKernel<kShortMax, SW><<<blocksFor(a.nPairs), kThreads, rowBytes<kShortMax>(), st>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

// Per-model FP64 log-space tables for the bubble scorer (called by mp_model_create).
mp_status mp_model_lower_log(const mp_model_desc *d, DevLogModel &m, double *rep) {
    for (int k = 0; k < 9; k++) m.t[k] = d->log_transitions[k];
    for (int k = 0; k < 3; k++) {
        m.start[k] = d->log_start[k];
        m.raggedStart[k] = d->log_ragged_start[k];
        m.end[k] = d->log_end[k];
        m.raggedEnd[k] = d->log_ragged_end[k];
    }
    for (int k = 0; k < 25; k++) m.match[k] = d->log_match[k];
    for (int k = 0; k < 5; k++) {
        m.gapX[k] = d->log_gap_x[k];
        m.gapY[k] = d->log_gap_y[k];
    }
    m.runLength = d->run_length ? 1 : 0;
    m.strand = d->strand ? 1 : 0;
    m.noSwitch = (std::isinf(m.t[1 * 3 + 2]) && m.t[1 * 3 + 2] < 0 && std::isinf(m.t[2 * 3 + 1]) && m.t[2 * 3 + 1] < 0)
                     ? 1 : 0;
    m.pad = 0;
    // 2.3025 * log10 R as the reference's RLE match emission forms it (impl/stateMachine.c:718-722)
    for (int i = 0; i < mp::kRepTable; i++) rep[i] = m.runLength && d->repeat_log10 ? d->repeat_scale * d->repeat_log10[i] : 0.0;
    return MP_OK;
}

extern "C" mp_status mp_forward_pairs(mp_engine *e, const mp_model *m, const mp_pair_batch *b, double *log_prob) {
    if (!e || !m || !b || (b->n_pairs > 0 && !log_prob)) return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs: NULL argument");
    const int64_t n = b->n_pairs;
    if (n < 0 || n > INT32_MAX) return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs: n_pairs out of range");
    if (n == 0) return MP_OK;
    if (!b->x_offset || !b->x_length || !b->y_offset || !b->y_length || !b->strand || !b->x_symbols || !b->y_symbols)
        return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs: pair arrays missing");
    // every pair inside its symbol buffers; every symbol's run length inside the repeat table
    for (int64_t j = 0; j < n; j++) {
        if (b->x_length[j] < 0 || b->y_length[j] < 0 || b->x_offset[j] < 0 || b->y_offset[j] < 0 ||
            b->x_offset[j] + b->x_length[j] > b->x_symbols_length || b->y_offset[j] + b->y_length[j] > b->y_symbols_length)
            return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs: pair %lld outside the symbol buffers", (long long) j);
    }
    const bool rle = m->logHost[0].runLength || m->logHost[1].runLength;
    if (rle) {
        for (int64_t i = 0; i < b->x_symbols_length; i++)
            if ((b->x_symbols[i] >> 8) >= mp::kMaxRepeat)
                return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs: x symbol %lld has run length >= %d", (long long) i,
                               mp::kMaxRepeat);
        for (int64_t i = 0; i < b->y_symbols_length; i++)
            if ((b->y_symbols[i] >> 8) >= mp::kMaxRepeat)
                return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs: y symbol %lld has run length >= %d", (long long) i,
                               mp::kMaxRepeat);
    }
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    cudaSetDevice(e->device);
    mp_pair_scratch &s = e->pairScratch;
    // pairs ordered by allele length (a counting sort, stable: pairs of a bubble stay together),
    // which makes the classes contiguous and gives the threads of a warp equal row lengths
    const int kSortMax = 32 * kWarpStrips;
    std::vector<int32_t> idx((size_t) n);
    {
        std::vector<int64_t> at((size_t) kSortMax + 2, 0);
        for (int64_t j = 0; j < n; j++) at[(size_t) std::min<int32_t>(b->x_length[j], kSortMax) + 1]++;
        for (int k = 1; k <= kSortMax + 1; k++) at[k] += at[k - 1];
        for (int64_t j = 0; j < n; j++) idx[(size_t) at[(size_t) std::min<int32_t>(b->x_length[j], kSortMax)]++] = (int32_t) j;
    }
    int32_t nCls[kClasses] = {}, start[kClasses] = {};
    for (int64_t j = 0; j < n; j++) nCls[classOf(b->x_length[j])]++;
    for (int c = 1; c < kClasses; c++) start[c] = start[c - 1] + nCls[c - 1];
    // warp classes longest first
    for (int c = 2; c <= kWarpStrips; c++) std::reverse(idx.begin() + start[c], idx.begin() + start[c] + nCls[c]);
    const int cl = kClasses - 1;
    std::vector<int64_t> rowOff((size_t) nCls[cl] + 1, 0);
    for (int32_t k = 0; k < nCls[cl]; k++)
        rowOff[(size_t) k + 1] = rowOff[(size_t) k] + 3 * ((int64_t) b->x_length[idx[(size_t) (start[cl] + k)]] + 1);
    const size_t nx = (size_t) std::max<int64_t>(b->x_symbols_length, 1), ny = (size_t) std::max<int64_t>(b->y_symbols_length, 1);
    PAIR_TRY(s.idx.reserve(sizeof(int32_t) * (size_t) n));
    PAIR_TRY(s.xOff.reserve(sizeof(int64_t) * (size_t) n));
    PAIR_TRY(s.yOff.reserve(sizeof(int64_t) * (size_t) n));
    PAIR_TRY(s.xLen.reserve(sizeof(int32_t) * (size_t) n));
    PAIR_TRY(s.yLen.reserve(sizeof(int32_t) * (size_t) n));
    PAIR_TRY(s.strand.reserve((size_t) n));
    PAIR_TRY(s.xs.reserve(sizeof(uint16_t) * nx));
    PAIR_TRY(s.ys.reserve(sizeof(uint16_t) * ny));
    PAIR_TRY(s.out.reserve(sizeof(double) * (size_t) n));
    PAIR_TRY(s.rowOff.reserve(sizeof(int64_t) * rowOff.size()));
    PAIR_TRY(s.rows.reserve(sizeof(double) * (size_t) std::max<int64_t>(rowOff.back(), 1)));
    cudaStream_t st = e->stream;
    struct Up {
        void *dst;
        const void *src;
        size_t bytes;
    } ups[] = {
        {s.idx.p, idx.data(), sizeof(int32_t) * (size_t) n},
        {s.xOff.p, b->x_offset, sizeof(int64_t) * (size_t) n},
        {s.yOff.p, b->y_offset, sizeof(int64_t) * (size_t) n},
        {s.xLen.p, b->x_length, sizeof(int32_t) * (size_t) n},
        {s.yLen.p, b->y_length, sizeof(int32_t) * (size_t) n},
        {s.strand.p, b->strand, (size_t) n},
        {s.xs.p, b->x_symbols, sizeof(uint16_t) * (size_t) b->x_symbols_length},
        {s.ys.p, b->y_symbols, sizeof(uint16_t) * (size_t) b->y_symbols_length},
        {s.rowOff.p, rowOff.data(), sizeof(int64_t) * rowOff.size()},
    };
    for (const Up &u : ups) {
        if (u.bytes == 0) continue;
        cudaError_t ce = cudaMemcpyAsync(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice, st);
        if (ce != cudaSuccess) return mp_fail(MP_ERR_CUDA, "mp_forward_pairs: upload failed: %s", cudaGetErrorString(ce));
    }
    PairArgs a;
    memset(&a, 0, sizeof(a));
    a.xOff = s.xOff.as<int64_t>();
    a.yOff = s.yOff.as<int64_t>();
    a.xLen = s.xLen.as<int32_t>();
    a.yLen = s.yLen.as<int32_t>();
    a.strand = s.strand.as<uint8_t>();
    a.xs = s.xs.as<uint16_t>();
    a.ys = s.ys.as<uint16_t>();
    a.models = m->logModels.as<DevLogModel>();
    a.repeatLog = m->logRepeat.as<double>();
    a.rows = s.rows.as<double>();
    a.rowOff = s.rowOff.as<int64_t>();
    a.out = s.out.as<double>();
    const int32_t *cls[kClasses];
    for (int c = 0; c < kClasses; c++) cls[c] = s.idx.as<int32_t>() + start[c];
    const bool sw = !(m->logHost[0].noSwitch && m->logHost[1].noSwitch);
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < 2 && ce == cudaSuccess; k++)
        if (!s.ev[k]) ce = cudaEventCreate(&s.ev[k]);
    if (ce == cudaSuccess) ce = cudaEventRecord(s.ev[0], st);
    if (ce == cudaSuccess)
        ce = sw ? launchAll<true>(a, cls, nCls, e->device, st) : launchAll<false>(a, cls, nCls, e->device, st);
    if (ce == cudaSuccess) ce = cudaEventRecord(s.ev[1], st);
    if (ce != cudaSuccess) return mp_fail(MP_ERR_CUDA, "mp_forward_pairs: launch failed: %s", cudaGetErrorString(ce));
    ce = cudaMemcpyAsync(log_prob, s.out.p, sizeof(double) * (size_t) n, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&s.kernelMs, s.ev[0], s.ev[1]);
    if (ce != cudaSuccess) return mp_fail(MP_ERR_CUDA, "mp_forward_pairs: %s", cudaGetErrorString(ce));
    int64_t cells = 0;
    for (int64_t j = 0; j < n; j++) cells += ((int64_t) b->x_length[j] + 1) * ((int64_t) b->y_length[j] + 1);
    s.cells = cells;
    s.pairs = n;
    return MP_OK;
}

extern "C" mp_status mp_forward_pairs_timing(mp_engine *e, float *kernel_ms, int64_t *cells, int64_t *pairs) {
    if (!e) return mp_fail(MP_ERR_ARGUMENT, "mp_forward_pairs_timing: NULL engine");
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    if (kernel_ms) *kernel_ms = e->pairScratch.kernelMs;
    if (cells) *cells = e->pairScratch.cells;
    if (pairs) *pairs = e->pairScratch.pairs;
    return MP_OK;
}
