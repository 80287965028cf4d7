/*
 * mpgpu_dropin.h -- drop-in replacements for MarginPolish's pair-HMM entry points.
 *
 * libmpgpu_dropin.so exports the reference's own signatures so that a MarginPolish
 * build can link it in place of impl/pairwiseAligner.c's posterior functions:
 *
 *   getAlignedPairsWithIndelsUsingAnchors   inc/pairwiseAligner.h:75-77 (impl/pairwiseAligner.c:1105-1130)
 *   getAlignedPairsUsingAnchors             inc/pairwiseAligner.h:73    (impl/pairwiseAligner.c:1088-1103)
 *   getAlignedPairsWithIndels               inc/pairwiseAligner.h:67-69 (impl/pairwiseAligner.c:1141-1149)
 *   getAlignedPairs                         inc/pairwiseAligner.h:60-61 (impl/pairwiseAligner.c:1132-1139)
 *   computeForwardProbability               inc/pairwiseAligner.h:54-55 (impl/pairwiseAligner.c:813-865)
 *   getExpectationsUsingAnchors             inc/pairwiseAligner.h:103-104 (impl/pairwiseAligner.c:1151-1156)
 *   getExpectations                         inc/pairwiseAligner.h:106 (impl/pairwiseAligner.c:1158-1164)
 *
 * The type declarations below restate the reference's public layouts
 * (inc/stateMachine.h:13-22, :40-48, :60-75, :96-124, :138-148; inc/pairwiseAligner.h:28-39)
 * so that objects built by the caller are read correctly. stList / stIntTuple
 * are the caller's sonLib; the library resolves stList_* / stIntTuple_* from the
 * host application at load time. The StateMachine is lowered to flat tables
 * through its public function pointers (cellCalculate, emission, boundary
 * probabilities), once per machine, and cached.
 *
 * Semantics: identical argument meaning and output order as the reference;
 * returned lists are newly allocated, own their stIntTuple elements and are
 * destroyed by the caller. Failures (no sm_100 device, malformed anchors,
 * unsupported machines) print the library's message and call exit(1), which
 * matches the reference's st_errAbort behaviour.
 *
 * Threading: the reference calls these from OpenMP threads, one chunk per thread
 * (marginPolish.c:436-439). Each calling thread gets its own engine -- its own CUDA
 * stream and device buffers, created on the thread's first call and released when
 * the thread exits -- and its own cache of lowered machines, so concurrent callers'
 * passes run side by side on the GPU. MPGPU_DEVICE selects the device (default 0).
 * A machine is recognised by its address and a fingerprint of its values; its tables
 * must not change in place once it has been passed in.
 */
#ifndef MPGPU_DROPIN_H_
#define MPGPU_DROPIN_H_

#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>

#include "mpgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct _stList stList;
typedef int64_t stIntTuple;

typedef struct _alphabet Alphabet;
typedef struct _emissions Emissions;
typedef uint16_t Symbol;

typedef struct _symbolString {
    Alphabet *alphabet;
    Symbol *sequence;
    int64_t length;
} SymbolString;

struct _alphabet {
    uint64_t alphabetSize;
    Symbol (*convertCharToSymbol)(char i);
    char (*convertSymbolToChar)(Symbol i);
    bool (*symbolsEqual)(Symbol, Symbol);
};

struct _emissions {
    Alphabet *alphabet;
    double (*emission)(Emissions *e, Symbol cX, Symbol cY);
    double (*gapEmissionX)(Emissions *e, Symbol cX);
    double (*gapEmissionY)(Emissions *e, Symbol cY);
    void (*printFn)(Emissions *e, FILE *f);
};

typedef enum { threeState = 2, threeStateAsymmetric = 3 } StateMachineType;
typedef enum { nucleotideEmissions = 0, nucleotideEmissionsSymmetric = 1 } EmissionType;

/* Expectation accumulator (inc/stateMachine.h:138-148); transitions[from * stateNumber + to]. */
typedef struct _hmm {
    StateMachineType type;
    EmissionType emissionsType;
    int64_t *emissionNoPerState;
    int64_t *emissionOffsetPerState;
    int64_t totalEmissions;
    double *transitions;
    double *emissions;
    double likelihood;
    int64_t stateNumber;
} Hmm;

typedef struct _stateMachine StateMachine;

struct _stateMachine {
    StateMachineType type;
    int64_t stateNumber;
    int64_t matchState;
    int64_t gapXState;
    int64_t gapYState;
    Emissions *emissions;
    double (*startStateProb)(StateMachine *sM, int64_t state);
    double (*endStateProb)(StateMachine *sM, int64_t state);
    double (*raggedEndStateProb)(StateMachine *sM, int64_t state);
    double (*raggedStartStateProb)(StateMachine *sM, int64_t state);
    void (*cellCalculate)(StateMachine *sM, double *current, double *lower, double *middle, double *upper,
                          Symbol cX, Symbol cY, void (*doTransition)(double *, double *, int64_t, int64_t, double,
                                                                     double, void *),
                          void *extraArgs);
    void (*printFn)(StateMachine *e, FILE *f);
};

typedef struct _pairwiseAlignmentBandingParameters {
    double threshold;
    int64_t minDiagsBetweenTraceBack;
    int64_t traceBackDiagonals;
    int64_t diagonalExpansion;
    int64_t constraintDiagonalTrim;
    int64_t splitMatrixBiggerThanThis;
    bool alignAmbiguityCharacters;
    float gapGamma;
    bool dynamicAnchorExpansion;
} PairwiseAlignmentParameters;

/* Reference signatures (see the file comment for the lines they replace). */
void getAlignedPairsWithIndelsUsingAnchors(StateMachine *sM, SymbolString sX, SymbolString sY, stList *anchorPairs,
                                           PairwiseAlignmentParameters *p, stList **alignedPairs, stList **gapXPairs,
                                           stList **gapYPairs, bool alignmentHasRaggedLeftEnd,
                                           bool alignmentHasRaggedRightEnd);
stList *getAlignedPairsUsingAnchors(StateMachine *sM, SymbolString sX, SymbolString sY, stList *anchorPairs,
                                    PairwiseAlignmentParameters *p, bool alignmentHasRaggedLeftEnd,
                                    bool alignmentHasRaggedRightEnd);
void getAlignedPairsWithIndels(StateMachine *sM, SymbolString sX, SymbolString sY, PairwiseAlignmentParameters *p,
                               stList **alignedPairs, stList **gapXPairs, stList **gapYPairs,
                               bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd);
stList *getAlignedPairs(StateMachine *sM, SymbolString sX, SymbolString sY, PairwiseAlignmentParameters *p,
                        bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd);
/* computeForwardProbability (impl/pairwiseAligner.c:813-865, inc/pairwiseAligner.h:54-55): ln P over
 * the band of band_construct, through mp_forward_batch. */
double computeForwardProbability(SymbolString sX, SymbolString sY, stList *anchorPairs, PairwiseAlignmentParameters *p,
                                 StateMachine *sM, bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd);
/* getExpectationsUsingAnchors (impl/pairwiseAligner.c:1151-1156, inc/pairwiseAligner.h:103-104): adds the
 * expected transition counts E[n_ij] (impl/pairwiseAligner.c:347-357) of the read to
 * hmmExpectations->transitions, through the adjoint pass mp_expectations_batch over the read's
 * band and split rectangles, and adds (lX + lY) * ln P to hmmExpectations->likelihood (the
 * reference adds its total once per posterior diagonal, impl/pairwiseAligner.c:674). Emission
 * expectations are left alone, as in the reference (:359-362). The counts are those of the whole
 * lattice; for a read whose band passes the reference's traceback points
 * (minDiagsBetweenTraceBack) the reference seeds each segment's backward at that point instead,
 * which moves its counts by the difference of those approximate posteriors. */
void getExpectationsUsingAnchors(StateMachine *sM, Hmm *hmmExpectations, SymbolString sX, SymbolString sY,
                                 stList *anchorPairs, PairwiseAlignmentParameters *p, bool alignmentHasRaggedLeftEnd,
                                 bool alignmentHasRaggedRightEnd);
/* getExpectations (impl/pairwiseAligner.c:1158-1164, inc/pairwiseAligner.h:106): the same without anchors. */
void getExpectations(StateMachine *sM, Hmm *hmmExpectations, SymbolString sX, SymbolString sY,
                     PairwiseAlignmentParameters *p, bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd);

/* Lowering of a caller's StateMachine to the flat description mp_model_create takes
 * (no device needed). repeat_out must hold 4*51*51 doubles; desc->repeat_log10 is set
 * to point at it when the machine carries run-length emissions. Returns MP_OK or
 * MP_ERR_ARGUMENT when the machine's emissions are not of the reference's form. */
mp_status mpd_lower_state_machine(StateMachine *sM, mp_model_desc *desc, double *repeat_out);

#ifdef __cplusplus
}
#endif

#endif
