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

#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

using mp::DevLogModel;
using mp::PairArgs;

#define PAIR_TRY(expr)                 \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

namespace {

constexpr double kLogZero = -INFINITY;

// lookup() of impl/pairwiseAligner.c:282-293 for 0 <= d < 7.5, each operation rounded alone.
__device__ __forceinline__ double lookupCubic(double d) {
    double c3, c2, c1, c0;
    if (d <= (double) 1.00f) {
        c3 = (double) -0.009350833524763f;
        c2 = (double) 0.130659527668286f;
        c1 = (double) 0.498799810682272f;
        c0 = (double) 0.693203116424741f;
    } else if (d <= (double) 2.50f) {
        c3 = (double) -0.014532321752540f;
        c2 = (double) 0.139942324101744f;
        c1 = (double) 0.495635523139337f;
        c0 = (double) 0.692140569840976f;
    } else if (d <= (double) 4.50f) {
        c3 = (double) -0.004605031767994f;
        c2 = (double) 0.063427417320019f;
        c1 = (double) 0.695956496475118f;
        c0 = (double) 0.514272634594009f;
    } else {
        c3 = (double) -0.000458661602210f;
        c2 = (double) 0.009695946122598f;
        c1 = (double) 0.930734667215156f;
        c0 = (double) 0.168037164329057f;
    }
    double v = __dmul_rn(c3, d);
    v = __dadd_rn(v, c2);
    v = __dmul_rn(v, d);
    v = __dadd_rn(v, c1);
    v = __dmul_rn(v, d);
    return __dadd_rn(v, c0);
}

// logAdd of impl/pairwiseAligner.c:295-299.
__device__ __forceinline__ double logAdd(double x, double y) {
    if (x < y) {
        const double d = __dsub_rn(y, x);
        return (x == kLogZero || d >= 7.5) ? y : __dadd_rn(lookupCubic(d), x);
    }
    const double d = __dsub_rn(x, y);
    return (y == kLogZero || d >= 7.5) ? x : __dadd_rn(lookupCubic(d), y);
}

// f + (e + t): the term doTransitionForward adds (impl/pairwiseAligner.c:311-314).
__device__ __forceinline__ double term(double f, double e, double t) {
    return __dadd_rn(f, __dadd_rn(e, t));
}

__device__ __forceinline__ int baseOf(uint16_t s, int runLength) {
    const int b = runLength ? (s & 255) : s;
    return b >= 4 ? 4 : b;
}

// The row of one thread: column x, state k.
template <int LXMAX>
struct SharedRow {
    double *base;
    __device__ __forceinline__ double &at(int x, int k) const { return base[(x * 3 + k) * blockDim.x]; }
};

struct GlobalRow {
    double *base;
    __device__ __forceinline__ double &at(int x, int k) const { return base[x * 3 + k]; }
};

// One pair: the forward recursion over the whole (lx+1) x (ly+1) matrix and the total at the
// last cell with the end probabilities (diagonalCalculationTotalProbability at the last
// diagonal, impl/pairwiseAligner.c:567-584, where only that cell is in the band).
template <bool SW, class Row>
__device__ double forwardPair(const PairArgs &a, int p, const Row &row) {
    const int lx = a.xLen[p], ly = a.yLen[p];
    if (lx + ly == 0) return 0.0;  // LOG_ONE (impl/pairwiseAligner.c:822-824)
    const DevLogModel &m = a.models[a.strand[p] ? 0 : 1];
    const double *rep = a.repeatLog + (a.strand[p] ? 0 : mp::kRepTable);
    const uint16_t *sx = a.xs + a.xOff[p];
    const uint16_t *sy = a.ys + a.yOff[p];
    const int rl = m.runLength;
    const double t00 = m.t[0], t01 = m.t[1], t02 = m.t[2];
    const double t10 = m.t[3], t11 = m.t[4], t12 = m.t[5];
    const double t20 = m.t[6], t21 = m.t[7], t22 = m.t[8];
    // row y = 0: the start cell, then gap-x cells fed from the left
    double l0 = m.start[0], l1 = m.start[1], l2 = m.start[2];
    row.at(0, 0) = l0;
    row.at(0, 1) = l1;
    row.at(0, 2) = l2;
    for (int x = 1; x <= lx; x++) {
        const double e = m.gapX[baseOf(sx[x - 1], rl)];
        double c1 = term(l0, e, t01);
        c1 = logAdd(c1, term(l1, e, t11));
        if (SW) c1 = logAdd(c1, term(l2, e, t21));
        l0 = kLogZero;
        l1 = c1;
        l2 = kLogZero;
        row.at(x, 0) = l0;
        row.at(x, 1) = l1;
        row.at(x, 2) = l2;
    }
    for (int y = 1; y <= ly; y++) {
        const uint16_t cy = sy[y - 1];
        const int yb = baseOf(cy, rl);
        const int ry = rl ? (cy >> 8) : 0;
        const double eY = m.gapY[yb];
        // column 0: a gap-y cell fed from above
        double d0 = row.at(0, 0), d1 = row.at(0, 1), d2 = row.at(0, 2);  // (x-1, y-1) for column 1
        {
            double c2 = term(d0, eY, t02);
            c2 = logAdd(c2, term(d2, eY, t22));
            if (SW) c2 = logAdd(c2, term(d1, eY, t12));
            l0 = kLogZero;
            l1 = kLogZero;
            l2 = c2;
            row.at(0, 0) = l0;
            row.at(0, 1) = l1;
            row.at(0, 2) = l2;
        }
        for (int x = 1; x <= lx; x++) {
            const uint16_t cx = sx[x - 1];
            const int xb = baseOf(cx, rl);
            const double u0 = row.at(x, 0), u1 = row.at(x, 1), u2 = row.at(x, 2);  // (x, y-1)
            // lower: gap-x from (x-1, y)
            const double eX = m.gapX[xb];
            double c1 = term(l0, eX, t01);
            c1 = logAdd(c1, term(l1, eX, t11));
            if (SW) c1 = logAdd(c1, term(l2, eX, t21));
            // middle: match from (x-1, y-1)
            double eM = m.match[xb * 5 + yb];
            if (rl) {
                const int rx = cx >> 8;
                const int r = xb == 4 ? 0 : xb;
                const int tableRow = m.strand ? r : 3 - r;
                eM = __dadd_rn(eM, rep[(tableRow * mp::kMaxRepeat + rx) * mp::kMaxRepeat + ry]);
            }
            double c0 = term(d0, eM, t00);
            c0 = logAdd(c0, term(d1, eM, t10));
            c0 = logAdd(c0, term(d2, eM, t20));
            // upper: gap-y from (x, y-1)
            double c2 = term(u0, eY, t02);
            c2 = logAdd(c2, term(u2, eY, t22));
            if (SW) c2 = logAdd(c2, term(u1, eY, t12));
            d0 = u0;
            d1 = u1;
            d2 = u2;
            l0 = c0;
            l1 = c1;
            l2 = c2;
            row.at(x, 0) = c0;
            row.at(x, 1) = c1;
            row.at(x, 2) = c2;
        }
    }
    // the last cell (lx, ly) with the end probabilities: cellDot, then logAdd(LOG_ZERO, .)
    double v = __dadd_rn(l0, m.end[0]);
    v = logAdd(v, __dadd_rn(l1, m.end[1]));
    v = logAdd(v, __dadd_rn(l2, m.end[2]));
    return logAdd(kLogZero, v);
}

// LXMAX > 0: alleles of at most LXMAX runs, rows in shared memory; LXMAX = 0: any length, rows
// in global memory.
template <int LXMAX, bool SW>
__global__ void __launch_bounds__(128) pairForwardKernel(PairArgs a) {
    extern __shared__ double smemRows[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nPairs) return;
    const int p = a.pairs[i];
    double r;
    if (LXMAX > 0) {
        SharedRow<LXMAX> row{smemRows + threadIdx.x};
        r = forwardPair<SW>(a, p, row);
    } else {
        GlobalRow row{a.rows + a.rowOff[i]};
        r = forwardPair<SW>(a, p, row);
    }
    a.out[p] = r;
}

constexpr int kThreads = 128;

template <int LXMAX>
size_t sharedBytes() {
    return LXMAX > 0 ? sizeof(double) * 3 * (LXMAX + 1) * kThreads : 0;
}

// Callers hold the engine's one-shot lock; the attribute is set once per device and kernel.
template <int LXMAX, bool SW>
cudaError_t launchClass(const PairArgs &a, int device, cudaStream_t st) {
    if (a.nPairs == 0) return cudaSuccess;
    const size_t smem = sharedBytes<LXMAX>();
    static std::mutex lock;
    static bool granted[128] = {};
    if (smem > 48 * 1024) {
        std::lock_guard<std::mutex> g(lock);
        if (!granted[device & 127]) {
            cudaError_t e = cudaFuncSetAttribute(pairForwardKernel<LXMAX, SW>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            if (e != cudaSuccess) return e;
            granted[device & 127] = true;
        }
    }
    const int blocks = (a.nPairs + kThreads - 1) / kThreads;
    pairForwardKernel<LXMAX, SW><<<blocks, kThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool SW>
cudaError_t launchAll(PairArgs a, const int32_t *const cls[4], const int32_t nCls[4], int device, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    a.pairs = cls[0];
    a.nPairs = nCls[0];
    if ((e = launchClass<16, SW>(a, device, st)) != cudaSuccess) return e;
    a.pairs = cls[1];
    a.nPairs = nCls[1];
    if ((e = launchClass<32, SW>(a, device, st)) != cudaSuccess) return e;
    a.pairs = cls[2];
    a.nPairs = nCls[2];
    if ((e = launchClass<64, SW>(a, device, st)) != cudaSuccess) return e;
    a.pairs = cls[3];
    a.nPairs = nCls[3];
    return launchClass<0, SW>(a, device, st);
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
    // length classes by allele length (stable: pairs of a bubble stay together)
    std::vector<int32_t> idx((size_t) n);
    int32_t nCls[4] = {0, 0, 0, 0};
    auto classOf = [](int32_t lx) { return lx <= 16 ? 0 : lx <= 32 ? 1 : lx <= 64 ? 2 : 3; };
    for (int64_t j = 0; j < n; j++) nCls[classOf(b->x_length[j])]++;
    int32_t start[4] = {0, nCls[0], nCls[0] + nCls[1], nCls[0] + nCls[1] + nCls[2]};
    int32_t at[4] = {start[0], start[1], start[2], start[3]};
    std::vector<int64_t> rowOff((size_t) nCls[3] + 1, 0);
    for (int64_t j = 0; j < n; j++) {
        const int c = classOf(b->x_length[j]);
        if (c == 3) rowOff[(size_t) (at[3] - start[3]) + 1] = 3 * ((int64_t) b->x_length[j] + 1);
        idx[(size_t) at[c]++] = (int32_t) j;
    }
    for (size_t k = 1; k < rowOff.size(); k++) rowOff[k] += rowOff[k - 1];
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
    const int32_t *cls[4];
    for (int c = 0; c < 4; c++) cls[c] = s.idx.as<int32_t>() + start[c];
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
