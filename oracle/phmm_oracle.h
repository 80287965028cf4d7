/*
 * ORACLE B -- TEST INFRASTRUCTURE ONLY.
 *
 * An FP64 restatement of MarginPolish's anchored, banded 3-state pair-HMM
 * posterior pass (the schedule of impl/pairwiseAligner.c:81-269, :528-808,
 * :875-991, :1068-1130, with the model of impl/stateMachine.c:360-380,
 * :518-581, :632-689, :702-736 lowered to flat log tables). It is the
 * checker for the CUDA library, never part of it: only tests/, bench.py's
 * CPU-baseline leg and __graft_entry__.smoke() load it.
 *
 * Parity pin: with logAdd replaced by the reference's own logAdd (passed in
 * as a function pointer from the reference build) the outputs are required to
 * be bit-identical to the reference's getAlignedPairsWithIndelsUsingAnchors;
 * with the default exact log-sum (max + log1p(exp(-|a-b|))) it is the FP64
 * oracle for the 1e-4 posterior bound.
 */
#ifndef MP_PHMM_ORACLE_H_
#define MP_PHMM_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* States: 0 match, 1 gap-x (consumes x), 2 gap-y (consumes y). */
typedef struct {
    double trans[9];        /* log transition, index from*3+to */
    double start[3];        /* log boundary probabilities */
    double raggedStart[3];
    double end[3];
    double raggedEnd[3];
    double match[25];       /* log match emission by base [xb*5+yb]; base 4 = N */
    double gapX[5];         /* log gap-x emission by x base */
    double gapY[5];         /* log gap-y emission by y base */
    int64_t runLength;      /* 1: symbols carry repeat counts; base = symbol & 255 */
    int64_t strand;         /* run-length table strand flag (1 forward) */
    int64_t maxRepeat;      /* repeat table dimension (51) */
    double repeatScale;     /* multiplier of the log10 repeat table (2.3025) */
    const double *repeat10; /* [4][maxRepeat][maxRepeat] log10, [base][underlying][observed]; may be NULL */
} MpoModel;

typedef struct {
    double threshold;
    int64_t minDiagsBetweenTraceBack;
    int64_t traceBackDiagonals;
    int64_t diagonalExpansion;
    int64_t constraintDiagonalTrim;
    int64_t splitMatrixBiggerThanThis;
    int64_t dynamicAnchorExpansion;
    double gapGamma;
} MpoParams;

typedef double (*MpoLogAddFn)(double, double);

typedef struct {
    int64_t n[3];           /* match, gap-x, gap-y tuple counts */
    int64_t *t[3];          /* n[k]*3 int64 (weight, x, y), reference order */
    double logLikelihood;   /* sum over splits of the final segment's log total probability */
    int64_t cells;          /* sum of band widths over all split sub-problems (the GCUPS numerator) */
    int64_t nDense;         /* dense posterior records (when requested) */
    double *dense;          /* nDense*5: x, y, pM, pX, pY in emission order; -1 = not defined */
} MpoResult;

/* Full posterior pass of one job (getAlignedPairsWithIndelsUsingAnchors semantics). wantDense:
 * 0 none, 1 a record for every band cell of every posterior diagonal, 2 only the records of cells
 * with a posterior of at least threshold - 1e-3. */
MpoResult *mpo_align_with_indels(const MpoModel *model, const uint16_t *sx, int64_t lx, const uint16_t *sy,
                                 int64_t ly, const int64_t *anchors, int64_t nAnchors, const MpoParams *params,
                                 int raggedLeft, int raggedRight, MpoLogAddFn logAdd, int wantDense);

void mpo_result_free(MpoResult *r);

/* Band of one sub-problem: writes (xay, xmyL, xmyR) for d = 0..lX+lY. Returns 0, or -1 on an invalid diagonal. */
int mpo_band(const int64_t *anchors, int64_t nAnchors, int64_t lX, int64_t lY, int64_t expansion, int dynamic,
             int64_t *out);

/* Split rectangles (x1, y1, x2, y2); returns the count (writes at most cap). */
int64_t mpo_split_points(const int64_t *anchors, int64_t nAnchors, int64_t lX, int64_t lY, int64_t maxMatrixSize,
                         int raggedLeft, int raggedRight, int64_t *out, int64_t cap);

/* Log match / gap emissions of the lowered model for two symbols. */
double mpo_match_emission(const MpoModel *m, uint16_t cx, uint16_t cy);
double mpo_gap_x_emission(const MpoModel *m, uint16_t cx);
double mpo_gap_y_emission(const MpoModel *m, uint16_t cy);

/* Forward log-probability (computeForwardProbability, impl/pairwiseAligner.c:813-865): the
 * forward recursion over the band (band_construct with the fixed expansion when dynamic is 0,
 * as the reference; band_constructDynamic with the anchors' expansions when 1), total at the
 * last anti-diagonal with the (ragged) end probabilities. No splits, no traceback segments.
 * Returns 0 (LOG_ONE) for lx + ly = 0 and NaN on an invalid band. logAdd NULL = exact. */
double mpo_forward_probability(const MpoModel *model, const uint16_t *sx, int64_t lx, const uint16_t *sy,
                               int64_t ly, const int64_t *anchors, int64_t nAnchors, int64_t expansion, int dynamic,
                               int raggedLeft, int raggedRight, MpoLogAddFn logAdd);

/* Expected counts of one sub-problem by exact FP64 forward-backward over the whole band
 * (no traceback segments, no splits): out[0..8] transitions (from*3+to), out[9..33] match
 * posteriors by (x base, y base), out[34..38] gap-x by x base, out[39..43] gap-y by y base,
 * out[44..46] / out[47..49] state posteriors at the first / last cell,
 * out[50 .. 50 + 4*M*M) match posteriors by run-length table entry [row][rcx][rcy]
 * (M = model->maxRepeat; only when the model is run-length). Counts are added to out.
 * Returns ln P, NaN on an invalid band. */
double mpo_expectations(const MpoModel *model, const uint16_t *sx, int64_t lx, const uint16_t *sy, int64_t ly,
                        const int64_t *anchors, int64_t nAnchors, int64_t expansion, int dynamic, int raggedLeft,
                        int raggedRight, double *out);

/* Exact log-sum used by default. */
double mpo_logadd_exact(double a, double b);

/* Batched run over jobs with OpenMP (dynamic,1); counts is nJobs*3. */
int64_t mpo_align_batch(const MpoModel *modelFwd, const MpoModel *modelRev, int64_t nJobs,
                        const int64_t *xOffsets, const uint16_t *xSymbols, const int64_t *yOffsets,
                        const uint16_t *ySymbols, const int64_t *anchorOffsets, const int64_t *anchors,
                        const uint8_t *strand, const MpoParams *params, int nThreads, int64_t *counts,
                        double *logLikelihoods);

#ifdef __cplusplus
}
#endif

#endif
