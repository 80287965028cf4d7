// Internal definitions shared by the host planner (mp_api.cu) and the device
// kernels (mp_kernels.cu) of the realignment engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mp {

constexpr int kMaxRepeat = 51;                       // inc/margin.h:123
constexpr int kRepTable = 4 * kMaxRepeat * kMaxRepeat; // one strand's run-length table
constexpr int kProbOne = 10000000;                   // inc/pairwiseAligner.h:26

// Lowered state machine of one read strand in probability space (FP32).
struct DevModel {
    float t[9];            // transitions from*3+to (0 match, 1 gap-x, 2 gap-y)
    float start[3];
    float raggedStart[3];
    float end[3];
    float raggedEnd[3];
    float match[25];       // [xbase*5 + ybase], base 4 = 'N'
    float gapX[5];
    float gapY[5];
    int32_t runLength;     // symbols carry repeat counts
    int32_t strand;        // repeat-table strand flag (row = strand ? base : 3 - base)
    int32_t pad[2];
};

// Log-space state machine of one read strand in FP64, the values the reference's cells use
// (the bubble scorer reproduces the reference's arithmetic on them).
struct DevLogModel {
    double t[9];           // log transitions from*3+to
    double start[3];
    double raggedStart[3];
    double end[3];
    double raggedEnd[3];
    double match[25];      // log match emissions [xbase*5 + ybase]
    double gapX[5];
    double gapY[5];
    int32_t runLength;
    int32_t strand;
    int32_t noSwitch;      // both switch transitions (gap-x <-> gap-y) are log 0
    int32_t pad;
};

// Bubble-scoring launch: one thread per (allele, read substring) pair of a length class.
struct PairArgs {
    const int32_t *pairs;       // pair indices of this launch (a length class)
    int32_t nPairs;
    const int64_t *xOff, *yOff;
    const int32_t *xLen, *yLen;
    const uint8_t *strand;
    const uint16_t *xs, *ys;
    const DevLogModel *models;  // [0] forward strand, [1] reverse strand
    const double *repeatLog;    // [2][kRepTable] repeat_scale * log10 table, per model
    double *rows;               // generic class only: one row of 3 (lx+1) doubles per pair
    const int64_t *rowOff;      // generic class only: each pair's row (in doubles)
    double *out;                // ln P per pair (indexed by pair)
};

// One banded sub-problem (one split rectangle of one job).
struct Task {
    int64_t xOff;          // first X symbol of the sub-problem (device symbol buffer index)
    int64_t yOff;          // first Y symbol
    int64_t bandOff;       // first diagonal record in the band buffer (N+1 records)
    int64_t anchorOff;     // first anchor triple of the sub-problem (original coordinates)
    int64_t outOff[3];     // start of this task's output region per list
    int32_t cap[3];        // capacity per list (tuples)
    int32_t nAnchors;
    int32_t lx, ly;        // sub-problem lengths
    int32_t x1, y1;        // split origin (subtracted from anchors, added to outputs)
    int32_t xShift;        // job-level x shift added to outputs (reference crop start)
    int32_t flags;         // bit0 ragged left, bit1 ragged right, bit2 forward strand, bit3 dynamic expansion
    int32_t job;
    int32_t expansion;     // fixed expansion when not dynamic
    int32_t pad[2];
};

// Task flags.
constexpr int32_t kFlagRaggedLeft = 1, kFlagRaggedRight = 2, kFlagForward = 4, kFlagDynamic = 8,
                  kFlagForwardOnly = 16;  // likelihood only: one walk of the top block, no tuples

// Expected counts (adjoint) in global memory, per model m (0 forward strand, 1 reverse):
// [m*kExpPerModel + kExpTrans + from*3+to]   sum over cells of f_from * u_to / P (times t on the host)
// [m*kExpPerModel + kExpMatch + xb*5+yb]     posterior of the match state by (x base, y base)
// [m*kExpPerModel + kExpGapX + xb], [.. + kExpGapY + yb]
// [m*kExpPerModel + kExpStart + s], [.. + kExpEnd + s]  state posteriors at the first / last cell
// and, separately, [table][4][51][51] posteriors of the match state by repeat-table entry.
constexpr int kExpTrans = 0, kExpMatch = 9, kExpGapX = 34, kExpGapY = 39, kExpStart = 44, kExpEnd = 47,
              kExpPerModel = 50;

enum TaskStatus : int32_t {
    kTaskOk = 0,
    kTaskCapacity = 1,     // an output list needed more than its capacity (counts are exact)
    kTaskWindow = 2,       // band hull wider than the slot window of the class
    kTaskBand = 4,         // invalid diagonal (reference: exception)
    kTaskScratch = 8,      // checkpoint scratch too small
    kTaskSymbol = 16,      // a symbol's repeat count is >= kMaxRepeat
    kTaskRange = 32        // the walk's totals disagree: the scaled values lost their range
};

struct TaskOut {
    int32_t count[3];
    int32_t status;
    double logLik;         // natural log of the final segment's total probability
    int64_t cells;         // sum of band widths
};

// Kernel-wide parameters of a posterior launch.
struct DpArgs {
    const Task *tasks;
    const int32_t *order;       // task indices in queue order (longest first)
    int32_t nTasks;
    int32_t scratchBlocks;      // checkpoints available per task slot
    int32_t *queue;             // global work counter
    const uint16_t *xs;
    const uint16_t *ys;
    const int2 *band;           // (xmyL, xmyR) per diagonal
    const DevModel *models;     // [0] forward strand, [1] reverse strand
    const float *repeatProb;    // [2][4][51][51] exp(scale*log10 table), per model
    void *scratch;              // per task slot: checkpoints [block][window slot] (float4 or double4)
    int2 *scratchScalars;       // per task slot: (exponent, window) per checkpoint
    int4 *outT[3];              // per list: staged tuples (weight, x, y, 0) in per-task regions
    TaskOut *out;
    float threshold;
    int32_t minDiagsBetweenTraceBack;
    int32_t traceBackDiagonals;
    int32_t diagonalExpansion;
    int32_t sharedRepeat;       // both models use repeat table 0
    int32_t noSwitch;           // both models' switch transitions (gap-x <-> gap-y) are zero
    double *expect;             // adjoint only: [2][kExpPerModel]
    double *expectRep;          // adjoint only: [tables][kRepTable]
};

// Compaction: task regions of the staged tuples -> per-job final lists.
struct CompactArgs {
    const Task *tasks;
    const TaskOut *out;
    int32_t nTasks;
    const int64_t *dst[3];      // per list: first destination index of each task (NULL: 0)
    const int4 *src[3];         // staged tuples (DpArgs::outT)
    int32_t *w[3];
    int32_t *x[3];
    int32_t *y[3];
};

struct BandArgs {
    const Task *tasks;
    int32_t nTasks;
    const int32_t *anchors;     // triples, original job coordinates
    int2 *band;
    TaskOut *out;
};

}  // namespace mp
