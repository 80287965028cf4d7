// Match posteriors of small anchor-free alignments in the reference's own arithmetic.
//
// Chunk stitching (removeOverlap, impl/polisher.c:1937-2006) cuts two chunks at the first match
// pair of the largest integer weight. Over an overlap of identical sequence the weights form a
// plateau near 10^7 whose maximum is decided by the last bits of the reference's approximate
// log-sum, so the cut agrees with the reference only if the weights are the reference's. This
// kernel computes getAlignedPairs (impl/pairwiseAligner.c:1132-1139) as the reference does:
// FP64 log cells over the whole matrix, the forward recursion, the backward walk from the end
// (and from every traceback point, impl/pairwiseAligner.c:722-737), the total probability
// refreshed every 10 posterior diagonals (:567-584, with the crossing term of the next
// diagonal), and the match posterior exp(f + b - total) floored to the integer scale (:586-620).
// One thread walks one alignment with its forward and backward matrices in global memory; the
// stitching windows are a hundred characters, so the work is small and its cost is the launch.
// exp() is CUDA's double-precision exp: within one unit in the last place of the host library's,
// it moves an integer weight only when the scaled posterior falls within that of an integer.
#include "../../include/mpgpu.h"
#include "mp_host.h"
#include "mp_internal.h"
#include "mp_refmath.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

#define PAIRS_TRY(expr)                \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

namespace {

// One alignment: symbols, lengths and where its matrices and tuples live.
struct RefJob {
    int64_t xOff, yOff;       // symbols
    int64_t cellOff;          // first cell of its matrices (3 doubles a cell)
    int64_t outOff;           // first tuple slot (lx * ly slots)
    int64_t liveOff;          // first byte of its live-diagonal flags (lx + ly + 2)
    int32_t lx, ly;
    int32_t flags;            // bit0 ragged left, bit1 ragged right, bit2 forward-strand model
    int32_t pad;
};

struct RefArgs {
    const RefJob *jobs;
    int32_t nJobs;
    const uint16_t *xs, *ys;
    const DevLogModel *models;
    double *F, *B;            // cells, 3 doubles each
    uint8_t *live;
    int4 *out;                // (weight, x, y, 0) in emission order
    int32_t *count;           // tuples per job
    double threshold;
    int64_t minDiagsBetweenTraceBack, traceBackDiagonals, diagonalExpansion;
};

// The full matrix as the reference's band of an anchor-free alignment: diagonal d holds the
// cells x - y = xmy for xmy in [lo(d), hi(d)] step 2.
struct Matrix {
    int lx, ly;
    const uint16_t *sx, *sy;
    double *F, *B;
    uint8_t *live;
    __device__ int lo(int d) const { return 2 * max(0, d - ly) - d; }
    __device__ int hi(int d) const { return 2 * min(lx, d) - d; }
    // cell (d, xmy) when it is in the band (0 <= d <= lx + ly), else null
    __device__ double *cell(double *base, int d, int xmy) const {
        if (d < 0 || d > lx + ly || xmy < lo(d) || xmy > hi(d)) return nullptr;
        const int x = (d + xmy) >> 1, y = (d - xmy) >> 1;
        return base + 3 * ((int64_t) y * (lx + 1) + x);
    }
    __device__ uint16_t xSym(int d, int xmy) const {
        const int x = (d + xmy) >> 1;
        return x > 0 ? sx[x - 1] : 4;
    }
    __device__ uint16_t ySym(int d, int xmy) const {
        const int y = (d - xmy) >> 1;
        return y > 0 ? sy[y - 1] : 4;
    }
};

__device__ __forceinline__ double emitMatch(const DevLogModel &m, uint16_t cx, uint16_t cy) {
    return m.match[baseOf(cx, m.runLength) * 5 + baseOf(cy, m.runLength)];
}

// Forward cells of diagonal d (stateMachine3_cellCalculate with doTransitionForward).
__device__ void forwardDiag(const Tables &T, const DevLogModel &m, const Matrix &M, int d) {
    const double *t = m.t;
    for (int xmy = M.lo(d); xmy <= M.hi(d); xmy += 2) {
        double *cur = M.cell(M.F, d, xmy);
        const double *lower = M.cell(M.F, d - 1, xmy - 1);
        const double *middle = d >= 2 ? M.cell(M.F, d - 2, xmy) : nullptr;
        const double *upper = M.cell(M.F, d - 1, xmy + 1);
        const uint16_t cx = M.xSym(d, xmy), cy = M.ySym(d, xmy);
        if (lower) {
            const double e = m.gapX[baseOf(cx, m.runLength)];
            cur[1] = logAdd(T, cur[1], term(lower[0], e, t[0 * 3 + 1]));
            cur[1] = logAdd(T, cur[1], term(lower[1], e, t[1 * 3 + 1]));
            cur[1] = logAdd(T, cur[1], term(lower[2], e, t[2 * 3 + 1]));
        }
        if (middle) {
            const double e = emitMatch(m, cx, cy);
            cur[0] = logAdd(T, cur[0], term(middle[0], e, t[0 * 3 + 0]));
            cur[0] = logAdd(T, cur[0], term(middle[1], e, t[1 * 3 + 0]));
            cur[0] = logAdd(T, cur[0], term(middle[2], e, t[2 * 3 + 0]));
        }
        if (upper) {
            const double e = m.gapY[baseOf(cy, m.runLength)];
            cur[2] = logAdd(T, cur[2], term(upper[0], e, t[0 * 3 + 2]));
            cur[2] = logAdd(T, cur[2], term(upper[2], e, t[2 * 3 + 2]));
            cur[2] = logAdd(T, cur[2], term(upper[1], e, t[1 * 3 + 2]));
        }
    }
}

// Backward push from diagonal d into d-1 and d-2 (doTransitionBackward), into live diagonals.
__device__ void backwardDiag(const Tables &T, const DevLogModel &m, const Matrix &M, int d) {
    const double *t = m.t;
    const bool live1 = d - 1 >= 0 && M.live[d - 1];
    const bool live2 = d - 2 >= 0 && M.live[d - 2];
    for (int xmy = M.lo(d); xmy <= M.hi(d); xmy += 2) {
        const double *cur = M.cell(M.B, d, xmy);
        double *lower = live1 ? M.cell(M.B, d - 1, xmy - 1) : nullptr;
        double *middle = live2 ? M.cell(M.B, d - 2, xmy) : nullptr;
        double *upper = live1 ? M.cell(M.B, d - 1, xmy + 1) : nullptr;
        const uint16_t cx = M.xSym(d, xmy), cy = M.ySym(d, xmy);
        if (lower) {
            const double e = m.gapX[baseOf(cx, m.runLength)];
            lower[0] = logAdd(T, lower[0], term(cur[1], e, t[0 * 3 + 1]));
            lower[1] = logAdd(T, lower[1], term(cur[1], e, t[1 * 3 + 1]));
            lower[2] = logAdd(T, lower[2], term(cur[1], e, t[2 * 3 + 1]));
        }
        if (middle) {
            const double e = emitMatch(m, cx, cy);
            middle[0] = logAdd(T, middle[0], term(cur[0], e, t[0 * 3 + 0]));
            middle[1] = logAdd(T, middle[1], term(cur[0], e, t[1 * 3 + 0]));
            middle[2] = logAdd(T, middle[2], term(cur[0], e, t[2 * 3 + 0]));
        }
        if (upper) {
            const double e = m.gapY[baseOf(cy, m.runLength)];
            upper[0] = logAdd(T, upper[0], term(cur[2], e, t[0 * 3 + 2]));
            upper[2] = logAdd(T, upper[2], term(cur[2], e, t[2 * 3 + 2]));
            upper[1] = logAdd(T, upper[1], term(cur[2], e, t[1 * 3 + 2]));
        }
    }
}

__device__ __forceinline__ double cellDot(const Tables &T, const double *a, const double *b) {
    double v = __dadd_rn(a[0], b[0]);
    v = logAdd(T, v, __dadd_rn(a[1], b[1]));
    return logAdd(T, v, __dadd_rn(a[2], b[2]));
}

// diagonalCalculationTotalProbability (impl/pairwiseAligner.c:567-584): the cells of d, plus the
// match transitions that cross from d-1 into a live diagonal d+1.
__device__ double totalProb(const Tables &T, const DevLogModel &m, const Matrix &M, int d) {
    double total = kLogZero;
    for (int xmy = M.lo(d); xmy <= M.hi(d); xmy += 2)
        total = logAdd(T, total, cellDot(T, M.cell(M.F, d, xmy), M.cell(M.B, d, xmy)));
    if (d + 1 <= M.lx + M.ly && M.live[d + 1] && d - 1 >= 0) {
        const double *t = m.t;
        double crossing = kLogZero;
        for (int xmy = M.lo(d + 1); xmy <= M.hi(d + 1); xmy += 2) {
            double mc[3] = {kLogZero, kLogZero, kLogZero};
            const double *middle = M.cell(M.F, d - 1, xmy);
            if (middle) {
                const double e = emitMatch(m, M.xSym(d + 1, xmy), M.ySym(d + 1, xmy));
                mc[0] = logAdd(T, mc[0], term(middle[0], e, t[0 * 3 + 0]));
                mc[0] = logAdd(T, mc[0], term(middle[1], e, t[1 * 3 + 0]));
                mc[0] = logAdd(T, mc[0], term(middle[2], e, t[2 * 3 + 0]));
            }
            crossing = logAdd(T, crossing, cellDot(T, mc, M.cell(M.B, d + 1, xmy)));
        }
        total = logAdd(T, total, crossing);
    }
    return total;
}

__device__ __forceinline__ void fill(double *c, int n, double v) {
    for (int i = 0; i < n; i++) c[i] = v;
}

// One alignment: getPosteriorProbsWithBanding (impl/pairwiseAligner.c:687-808) with the match
// posterior callback, the walk schedule of traceback points included.
__global__ void __launch_bounds__(32) refMatchKernel(RefArgs a) {
    __shared__ Tables T;
    loadTables(T, a.models);
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.nJobs) return;
    const RefJob &job = a.jobs[j];
    const DevLogModel &m = T.models[(job.flags & 4) ? 0 : 1];
    Matrix M{job.lx, job.ly, a.xs + job.xOff, a.ys + job.yOff, a.F + 3 * job.cellOff, a.B + 3 * job.cellOff,
             a.live + job.liveOff};
    const int N = job.lx + job.ly;
    int n = 0;
    int4 *out = a.out + job.outOff;
    if (N > 0) {
        const int64_t cells = (int64_t) (job.lx + 1) * (job.ly + 1);
        fill(M.F, (int) (3 * cells), kLogZero);
        fill(M.B, (int) (3 * cells), kLogZero);
        for (int d = 0; d <= N + 1; d++) M.live[d] = 0;
        double *origin = M.cell(M.F, 0, 0);
        const double *start = (job.flags & 1) ? m.raggedStart : m.start;
        origin[0] = start[0], origin[1] = start[1], origin[2] = start[2];
        int tracedBackTo = 0;
        for (int d = 1; d <= N; d++) {
            forwardDiag(T, m, M, d);
            const bool atEnd = d == N;
            const int width = (M.hi(d) - M.lo(d)) / 2 + 1;
            const bool tracebackPoint = d >= tracedBackTo + a.minDiagsBetweenTraceBack &&
                                        width <= a.diagonalExpansion * 2 + 1;
            if (!(atEnd || tracebackPoint)) continue;
            const double *end = (atEnd && (job.flags & 2)) ? m.raggedEnd : m.end;
            for (int xmy = M.lo(d); xmy <= M.hi(d); xmy += 2) {
                double *c = M.cell(M.B, d, xmy);
                c[0] = end[0], c[1] = end[1], c[2] = end[2];
            }
            M.live[d] = 1;
            auto reset = [&](int dd) {
                for (int xmy = M.lo(dd); xmy <= M.hi(dd); xmy += 2) fill(M.cell(M.B, dd, xmy), 3, kLogZero);
            };
            if (d > tracedBackTo + 1) {
                reset(d - 1);
                M.live[d - 1] = 1;
            }
            const int tracedBackFrom = d - (atEnd ? 0 : (int) a.traceBackDiagonals + 1);
            double totalLog = kLogZero;
            int posteriorsThisWalk = 0;
            for (int d2 = d; d2 > tracedBackTo; d2--) {
                if (d2 > tracedBackTo + 2) {
                    reset(d2 - 2);
                    M.live[d2 - 2] = 1;
                }
                if (d2 > tracedBackTo + 1) backwardDiag(T, m, M, d2);
                if (d2 <= tracedBackFrom) {
                    if (posteriorsThisWalk++ % 10 == 0) totalLog = totalProb(T, m, M, d2);
                    // diagonalCalculationPosteriorMatchProbs / addPosteriorProb (:586-620)
                    for (int xmy = M.lo(d2); xmy <= M.hi(d2); xmy += 2) {
                        const int x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
                        if (x <= 0 || y <= 0) continue;
                        const double *f = M.cell(M.F, d2, xmy), *b = M.cell(M.B, d2, xmy);
                        double pm = exp(__dsub_rn(__dadd_rn(f[0], b[0]), totalLog));
                        if (pm >= a.threshold) {
                            if (pm > 1.0) pm = 1.0;
                            out[n++] = make_int4((int) floor(__dmul_rn(pm, (double) mp::kProbOne)), x - 1, y - 1, 0);
                        }
                    }
                }
                if (d2 + 1 <= N) M.live[d2 + 1] = 0;
            }
            for (int k = tracedBackTo; k <= d; k++) M.live[k] = 0;
            tracedBackTo = tracedBackFrom;
        }
    }
    a.count[j] = n;
}

}  // namespace

mp_status refMatchPairs(mp_engine *e, const mp_model *m, const mp_params *p, const std::vector<RefPair> &pairs,
                        const std::vector<uint16_t> &xs, const std::vector<uint16_t> &ys,
                        std::vector<std::vector<RefTuple>> &out) {
    out.assign(pairs.size(), {});
    if (pairs.empty()) return MP_OK;
    if (m->logHost[0].runLength || m->logHost[1].runLength)
        return mp_fail(MP_ERR_ARGUMENT, "reference-arithmetic posteriors take a model without run lengths");
    std::vector<RefJob> jobs(pairs.size());
    int64_t cells = 0, slots = 0, live = 0;
    for (size_t k = 0; k < pairs.size(); k++) {
        const RefPair &q = pairs[k];
        if (q.lx < 0 || q.ly < 0 || q.xOff < 0 || q.yOff < 0 || q.xOff + q.lx > (int64_t) xs.size() ||
            q.yOff + q.ly > (int64_t) ys.size())
            return mp_fail(MP_ERR_ARGUMENT, "reference-arithmetic posteriors: pair %zu outside its symbols", k);
        const int64_t c = ((int64_t) q.lx + 1) * ((int64_t) q.ly + 1);
        if (c > kRefMaxCells)
            return mp_fail(MP_ERR_OVERFLOW, "reference-arithmetic posteriors: %lld cells exceed %lld", (long long) c,
                           (long long) kRefMaxCells);
        RefJob &jb = jobs[k];
        memset(&jb, 0, sizeof(jb));
        jb.xOff = q.xOff;
        jb.yOff = q.yOff;
        jb.lx = q.lx;
        jb.ly = q.ly;
        jb.flags = (q.raggedLeft ? 1 : 0) | (q.raggedRight ? 2 : 0) | (q.forward ? 4 : 0);
        jb.cellOff = cells;
        jb.outOff = slots;
        jb.liveOff = live;
        cells += c;
        slots += std::max<int64_t>((int64_t) q.lx * q.ly, 1);
        live += q.lx + q.ly + 2;
    }
    cudaSetDevice(e->device);
    DevBuf dJobs, dXs, dYs, dF, dB, dLive, dOut, dCount;
    PAIRS_TRY(dJobs.reserve(sizeof(RefJob) * jobs.size()));
    PAIRS_TRY(dXs.reserve(sizeof(uint16_t) * std::max<size_t>(xs.size(), 1)));
    PAIRS_TRY(dYs.reserve(sizeof(uint16_t) * std::max<size_t>(ys.size(), 1)));
    PAIRS_TRY(dF.reserve(sizeof(double) * 3 * (size_t) cells));
    PAIRS_TRY(dB.reserve(sizeof(double) * 3 * (size_t) cells));
    PAIRS_TRY(dLive.reserve((size_t) live));
    PAIRS_TRY(dOut.reserve(sizeof(int4) * (size_t) slots));
    PAIRS_TRY(dCount.reserve(sizeof(int32_t) * jobs.size()));
    cudaStream_t st = e->stream;
    cudaError_t ce = cudaMemcpyAsync(dJobs.p, jobs.data(), sizeof(RefJob) * jobs.size(), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && !xs.empty())
        ce = cudaMemcpyAsync(dXs.p, xs.data(), sizeof(uint16_t) * xs.size(), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && !ys.empty())
        ce = cudaMemcpyAsync(dYs.p, ys.data(), sizeof(uint16_t) * ys.size(), cudaMemcpyHostToDevice, st);
    RefArgs a;
    memset(&a, 0, sizeof(a));
    a.jobs = dJobs.as<RefJob>();
    a.nJobs = (int32_t) jobs.size();
    a.xs = dXs.as<uint16_t>();
    a.ys = dYs.as<uint16_t>();
    a.models = m->logModels.as<DevLogModel>();
    a.F = dF.as<double>();
    a.B = dB.as<double>();
    a.live = dLive.as<uint8_t>();
    a.out = dOut.as<int4>();
    a.count = dCount.as<int32_t>();
    a.threshold = p->threshold;
    a.minDiagsBetweenTraceBack = p->min_diags_between_traceback;
    a.traceBackDiagonals = p->traceback_diagonals;
    a.diagonalExpansion = p->diagonal_expansion;
    if (ce == cudaSuccess) {
        refMatchKernel<<<(a.nJobs + 31) / 32, 32, 0, st>>>(a);
        ce = cudaGetLastError();
    }
    std::vector<int32_t> count(jobs.size());
    std::vector<int4> tup((size_t) slots);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(count.data(), dCount.p, sizeof(int32_t) * count.size(), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(tup.data(), dOut.p, sizeof(int4) * tup.size(), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return mp_fail(MP_ERR_CUDA, "reference-arithmetic posteriors: %s", cudaGetErrorString(ce));
    // the sub-problem's list popped into the output (impl/pairwiseAligner.c:1062-1068): reversed
    for (size_t k = 0; k < jobs.size(); k++) {
        std::vector<RefTuple> &o = out[k];
        for (int32_t q = count[k] - 1; q >= 0; q--) {
            const int4 &t = tup[(size_t) (jobs[k].outOff + q)];
            o.push_back(RefTuple{t.x, t.y, t.z});
        }
    }
    return MP_OK;
}

extern "C" mp_status mp_match_pairs_reference(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                              int64_t *offsets, int32_t *weight, int32_t *x, int32_t *y, int64_t cap,
                                              int64_t *total) {
    if (!e || !m || !p || !b || !offsets || !total || b->n_jobs < 0)
        return mp_fail(MP_ERR_ARGUMENT, "mp_match_pairs_reference: NULL argument");
    const int64_t n = b->n_jobs;
    std::vector<RefPair> pairs((size_t) n);
    std::vector<uint16_t> xs(b->x_symbols, b->x_symbols + b->x_symbols_length),
        ys(b->y_symbols, b->y_symbols + (n > 0 ? b->y_offsets[n] : 0));
    for (int64_t j = 0; j < n; j++) {
        if (b->anchor_offsets && b->anchor_offsets[j + 1] != b->anchor_offsets[j])
            return mp_fail(MP_ERR_ARGUMENT, "mp_match_pairs_reference: job %lld has anchors", (long long) j);
        pairs[(size_t) j] = RefPair{b->x_begin[j], b->y_offsets[j], (int32_t) (b->x_end[j] - b->x_begin[j]),
                                    (int32_t) (b->y_offsets[j + 1] - b->y_offsets[j]),
                                    b->ragged_left ? b->ragged_left[j] != 0 : false,
                                    b->ragged_right ? b->ragged_right[j] != 0 : false,
                                    b->strand ? b->strand[j] != 0 : true};
    }
    std::vector<std::vector<RefTuple>> out;
    mp_status s = refMatchPairs(e, m, p, pairs, xs, ys, out);
    if (s != MP_OK) return s;
    offsets[0] = 0;
    for (int64_t j = 0; j < n; j++) offsets[j + 1] = offsets[j] + (int64_t) out[(size_t) j].size();
    *total = offsets[n];
    if (offsets[n] > cap) return mp_fail(MP_ERR_OVERFLOW, "mp_match_pairs_reference: %lld tuples, room for %lld",
                                         (long long) offsets[n], (long long) cap);
    for (int64_t j = 0; j < n; j++)
        for (size_t q = 0; q < out[(size_t) j].size(); q++) {
            const RefTuple &t = out[(size_t) j][q];
            const int64_t k = offsets[j] + (int64_t) q;
            if (weight) weight[k] = t.weight;
            if (x) x[k] = t.x;
            if (y) y[k] = t.y;
        }
    return MP_OK;
}
