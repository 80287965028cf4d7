/*
 * ORACLE A harness -- TEST INFRASTRUCTURE ONLY.
 *
 * Links against the reference's own impl/pairwiseAligner.c and
 * impl/stateMachine.c, compiled unmodified from the reference tree by
 * oracle/Makefile (output: oracle/_ref/libref_oracle.so), and exposes a flat
 * C API (plain pointers and sizes) that tests and the CPU baseline call via
 * ctypes. Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke()
 * load it, as the checker.
 *
 * The state machines are assembled exactly the way the reference's parser
 * does it (impl/parser.c:235-245 for the forward / reverse-complemented HMMs,
 * impl/parser.c:391-401 for the run-length emission swap).
 */
#include "margin.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* band_constructDynamic is defined non-static in impl/pairwiseAligner.c:120
 * but has no prototype in the public header. */
Band *band_constructDynamic(stList *anchorPairs, int64_t lX, int64_t lY);

#ifndef MP_REF_WITH_POLISHER  /* the POA oracle build links impl/polisher.c, which defines it */
/* ------------------------------------------------------------------------ */
/* Repeat-count table access.                                                */
/* impl/polisher.c (not compiled into the oracle) defines                    */
/* repeatSubMatrix_getLogProb; this is a restatement of its indexing rule    */
/* (impl/polisher.c:1756-1775): an 'N' base (alphabetSize-1) reads base 0,   */
/* the reverse strand reads the complement base's matrix (3-base), and the  */
/* flat index is base*M*M + underlying*M + observed.                         */
/* ------------------------------------------------------------------------ */
double repeatSubMatrix_getLogProb(RepeatSubMatrix *repeatSubMatrix, Symbol base, bool strand,
                                  int64_t observedRepeatCount, int64_t underlyingRepeatCount) {
    if (base == repeatSubMatrix->alphabet->alphabetSize - 1) {
        base = 0;
    }
    if (base >= repeatSubMatrix->alphabet->alphabetSize - 1) {
        st_errAbort("repeatSubMatrix_getLogProb: base 'N' not supported");
    }
    int64_t m = repeatSubMatrix->maximumRepeatLength;
    int64_t idx = (strand ? base : 3 - base) * m * m + underlyingRepeatCount * m + observedRepeatCount;
    if (idx < 0 || idx >= repeatSubMatrix->maxEntry) {
        st_errAbort("repeatSubMatrix_getLogProb: index %" PRIi64 " out of range", idx);
    }
    return repeatSubMatrix->logProbabilities[idx];
}
#endif

/* ------------------------------------------------------------------------ */
/* Model construction                                                        */
/* ------------------------------------------------------------------------ */

typedef struct {
    StateMachine *sM;
    RepeatSubMatrix *repeatSubMatrix; /* owned when non-NULL */
} RefoModel;

/*
 * hmmType: 2 (symmetric) or 3 (asymmetric); transitions: 9 probabilities
 * (from-major); emissions: 24 probabilities (16 match, 4 gap-x, 4 gap-y).
 * reverseComplement: apply nucleotideEmissions_reverseComplement (reverse
 * strand machine, impl/parser.c:243). repeatLog10: NULL or 4*51*51 log10
 * probabilities laid out [base][underlying][observed] for the forward strand;
 * strand: the strand flag handed to rleNucleotideEmissions_construct.
 */
void *refo_model_create(int hmmType, const double *transitions, const double *emissions, int reverseComplement,
                        const double *repeatLog10, int strand) {
    Hmm *hmm = hmm_constructEmpty(0.0, (StateMachineType) hmmType, nucleotideEmissions);
    for (int64_t i = 0; i < 9; i++) {
        hmm->transitions[i] = transitions[i];
    }
    for (int64_t i = 0; i < hmm->totalEmissions; i++) {
        hmm->emissions[i] = emissions[i];
    }
    RefoModel *m = st_calloc(1, sizeof(RefoModel));
    m->sM = hmm_getStateMachine(hmm);
    hmm_destruct(hmm);
    if (reverseComplement) {
        nucleotideEmissions_reverseComplement((NucleotideEmissions *) m->sM->emissions);
    }
    if (repeatLog10 != NULL) {
        RepeatSubMatrix *r = st_calloc(1, sizeof(RepeatSubMatrix));
        r->alphabet = alphabet_constructNucleotide();
        r->maximumRepeatLength = MAXIMUM_REPEAT_LENGTH;
        r->maxEntry = r->alphabet->alphabetSize * r->maximumRepeatLength * r->maximumRepeatLength;
        r->logProbabilities = st_calloc(r->maxEntry, sizeof(double));
        r->baseLogProbs_AT = st_calloc(r->maximumRepeatLength, sizeof(double));
        r->baseLogProbs_GC = st_calloc(r->maximumRepeatLength, sizeof(double));
        memcpy(r->logProbabilities, repeatLog10, sizeof(double) * 4 * MAXIMUM_REPEAT_LENGTH * MAXIMUM_REPEAT_LENGTH);
        m->repeatSubMatrix = r;
        m->sM->emissions = rleNucleotideEmissions_construct(m->sM->emissions, r, strand ? 1 : 0);
    }
    return m;
}

/* The code-default machine used by the reference's unit tests (stateMachine.c:598-630). */
void *refo_model_create_default(void) {
    RefoModel *m = st_calloc(1, sizeof(RefoModel));
    m->sM = stateMachine3_constructNucleotide(threeState);
    return m;
}

void refo_model_destroy(void *handle) {
    RefoModel *m = handle;
    if (m == NULL) {
        return;
    }
    stateMachine_destruct(m->sM);
    if (m->repeatSubMatrix != NULL) {
        alphabet_destruct(m->repeatSubMatrix->alphabet);
        free(m->repeatSubMatrix->logProbabilities);
        free(m->repeatSubMatrix->baseLogProbs_AT);
        free(m->repeatSubMatrix->baseLogProbs_GC);
        free(m->repeatSubMatrix);
    }
    free(m);
}

/* Evaluate the machine's emission / transition / boundary functions, so tests can
 * compare them with the flat tables the GPU library builds. */
double refo_model_match_emission(void *handle, int cx, int cy) {
    RefoModel *m = handle;
    return m->sM->emissions->emission(m->sM->emissions, (Symbol) cx, (Symbol) cy);
}

double refo_model_gap_x_emission(void *handle, int cx) {
    RefoModel *m = handle;
    return m->sM->emissions->gapEmissionX(m->sM->emissions, (Symbol) cx);
}

double refo_model_gap_y_emission(void *handle, int cy) {
    RefoModel *m = handle;
    return m->sM->emissions->gapEmissionY(m->sM->emissions, (Symbol) cy);
}

/* Records each (from, to, transition) the machine's cell function visits. */
static void recordTransition(double *fromCells, double *toCells, int64_t from, int64_t to, double eP, double tP,
                             void *extraArgs) {
    (void) fromCells;
    (void) toCells;
    (void) eP;
    ((double *) extraArgs)[from * 3 + to] = tP;
}

/* The 9 log transitions (from*3+to) as the reference's cellCalculate passes them. */
void refo_model_transitions(void *handle, double *out) {
    RefoModel *m = handle;
    double cur[3] = {0, 0, 0}, lower[3] = {0, 0, 0}, middle[3] = {0, 0, 0}, upper[3] = {0, 0, 0};
    m->sM->cellCalculate(m->sM, cur, lower, middle, upper, 0, 0, recordTransition, out);
}

/* boundary: 0 start, 1 ragged start, 2 end, 3 ragged end */
double refo_model_boundary(void *handle, int boundary, int state) {
    RefoModel *m = handle;
    switch (boundary) {
        case 0: return m->sM->startStateProb(m->sM, state);
        case 1: return m->sM->raggedStartStateProb(m->sM, state);
        case 2: return m->sM->endStateProb(m->sM, state);
        default: return m->sM->raggedEndStateProb(m->sM, state);
    }
}

/* ------------------------------------------------------------------------ */
/* Parameters                                                                */
/* ------------------------------------------------------------------------ */

typedef struct {
    double threshold;
    int64_t minDiagsBetweenTraceBack;
    int64_t traceBackDiagonals;
    int64_t diagonalExpansion;
    int64_t constraintDiagonalTrim;
    int64_t splitMatrixBiggerThanThis;
    int64_t dynamicAnchorExpansion;
    double gapGamma;
} RefoParams;

static PairwiseAlignmentParameters *toReferenceParams(const RefoParams *q) {
    PairwiseAlignmentParameters *p = pairwiseAlignmentBandingParameters_construct();
    p->threshold = q->threshold;
    p->minDiagsBetweenTraceBack = q->minDiagsBetweenTraceBack;
    p->traceBackDiagonals = q->traceBackDiagonals;
    p->diagonalExpansion = q->diagonalExpansion;
    p->constraintDiagonalTrim = q->constraintDiagonalTrim;
    p->splitMatrixBiggerThanThis = q->splitMatrixBiggerThanThis;
    p->dynamicAnchorExpansion = q->dynamicAnchorExpansion != 0;
    p->gapGamma = (float) q->gapGamma;
    p->alignAmbiguityCharacters = 0;
    return p;
}

/* Accessors for the POA oracle (oracle/ref_poa_harness.c). */
PairwiseAlignmentParameters *refo_params_to_reference(const RefoParams *q) {
    return toReferenceParams(q);
}

StateMachine *refo_model_state_machine(void *handle) {
    return ((RefoModel *) handle)->sM;
}

RepeatSubMatrix *refo_model_repeat_matrix(void *handle) {
    return ((RefoModel *) handle)->repeatSubMatrix;
}

static SymbolString toSymbolString(Alphabet *a, const uint16_t *s, int64_t n) {
    SymbolString ss;
    ss.alphabet = a;
    ss.sequence = st_malloc(sizeof(Symbol) * (n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) {
        ss.sequence[i] = s[i];
    }
    ss.length = n;
    return ss;
}

static stList *toAnchorList(const int64_t *anchors, int64_t nAnchors) {
    stList *l = stList_construct3(0, (void (*)(void *)) stIntTuple_destruct);
    for (int64_t i = 0; i < nAnchors; i++) {
        stList_append(l, stIntTuple_construct3(anchors[3 * i], anchors[3 * i + 1], anchors[3 * i + 2]));
    }
    return l;
}

/* ------------------------------------------------------------------------ */
/* Posterior pair lists                                                      */
/* ------------------------------------------------------------------------ */

typedef struct {
    int64_t n[3];     /* match, gap-x, gap-y */
    int64_t *t[3];    /* n[k] * 3 int64: weight, x, y (reference order) */
} RefoPairs;

static void flattenList(stList *l, int64_t *n, int64_t **t) {
    *n = stList_length(l);
    *t = st_malloc(sizeof(int64_t) * 3 * (*n > 0 ? *n : 1));
    for (int64_t i = 0; i < *n; i++) {
        stIntTuple *j = stList_get(l, i);
        (*t)[3 * i] = stIntTuple_get(j, 0);
        (*t)[3 * i + 1] = stIntTuple_get(j, 1);
        (*t)[3 * i + 2] = stIntTuple_get(j, 2);
    }
}

/* getAlignedPairsWithIndelsUsingAnchors (impl/pairwiseAligner.c:1105-1130) on one job. */
RefoPairs *refo_align_with_indels(void *model, const uint16_t *sx, int64_t lx, const uint16_t *sy, int64_t ly,
                                  const int64_t *anchors, int64_t nAnchors, const RefoParams *params,
                                  int raggedLeft, int raggedRight) {
    RefoModel *m = model;
    Alphabet *a = alphabet_constructNucleotide();
    SymbolString sX = toSymbolString(a, sx, lx), sY = toSymbolString(a, sy, ly);
    stList *anchorPairs = toAnchorList(anchors, nAnchors);
    PairwiseAlignmentParameters *p = toReferenceParams(params);
    stList *matches, *gapX, *gapY;
    getAlignedPairsWithIndelsUsingAnchors(m->sM, sX, sY, anchorPairs, p, &matches, &gapX, &gapY,
                                          raggedLeft != 0, raggedRight != 0);
    RefoPairs *r = st_calloc(1, sizeof(RefoPairs));
    flattenList(matches, &r->n[0], &r->t[0]);
    flattenList(gapX, &r->n[1], &r->t[1]);
    flattenList(gapY, &r->n[2], &r->t[2]);
    stList_destruct(matches);
    stList_destruct(gapX);
    stList_destruct(gapY);
    stList_destruct(anchorPairs);
    pairwiseAlignmentBandingParameters_destruct(p);
    symbolString_destruct(sX);
    symbolString_destruct(sY);
    alphabet_destruct(a);
    return r;
}

/* getAlignedPairsUsingAnchors (impl/pairwiseAligner.c:1088-1103): match list only. */
RefoPairs *refo_align(void *model, const uint16_t *sx, int64_t lx, const uint16_t *sy, int64_t ly,
                      const int64_t *anchors, int64_t nAnchors, const RefoParams *params,
                      int raggedLeft, int raggedRight) {
    RefoModel *m = model;
    Alphabet *a = alphabet_constructNucleotide();
    SymbolString sX = toSymbolString(a, sx, lx), sY = toSymbolString(a, sy, ly);
    stList *anchorPairs = toAnchorList(anchors, nAnchors);
    PairwiseAlignmentParameters *p = toReferenceParams(params);
    stList *matches = getAlignedPairsUsingAnchors(m->sM, sX, sY, anchorPairs, p, raggedLeft != 0, raggedRight != 0);
    RefoPairs *r = st_calloc(1, sizeof(RefoPairs));
    flattenList(matches, &r->n[0], &r->t[0]);
    r->t[1] = st_malloc(sizeof(int64_t));
    r->t[2] = st_malloc(sizeof(int64_t));
    stList_destruct(matches);
    stList_destruct(anchorPairs);
    pairwiseAlignmentBandingParameters_destruct(p);
    symbolString_destruct(sX);
    symbolString_destruct(sY);
    alphabet_destruct(a);
    return r;
}

void refo_pairs_free(RefoPairs *r) {
    if (r == NULL) {
        return;
    }
    for (int k = 0; k < 3; k++) {
        free(r->t[k]);
    }
    free(r);
}

/* ------------------------------------------------------------------------ */
/* Batched CPU run: OpenMP over jobs, schedule(dynamic,1), mirroring the     */
/* per-chunk parallel loop of marginPolish.c:436-439. Returns the pair       */
/* counts per job (nJobs*3) and optionally all tuples.                       */
/* ------------------------------------------------------------------------ */

int64_t refo_align_batch(void *modelFwd, void *modelRev, int64_t nJobs,
                         const int64_t *xOffsets, const uint16_t *xSymbols,
                         const int64_t *yOffsets, const uint16_t *ySymbols,
                         const int64_t *anchorOffsets, const int64_t *anchors,
                         const uint8_t *strand, const RefoParams *params, int nThreads,
                         int64_t *counts, int64_t **tuplesOut /* nullable: nJobs*3 malloc'd arrays */) {
#ifdef _OPENMP
    if (nThreads > 0) {
        omp_set_num_threads(nThreads);
    }
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t j = 0; j < nJobs; j++) {
        RefoPairs *r = refo_align_with_indels(strand[j] ? modelFwd : modelRev,
                                              xSymbols + xOffsets[j], xOffsets[j + 1] - xOffsets[j],
                                              ySymbols + yOffsets[j], yOffsets[j + 1] - yOffsets[j],
                                              anchors + 3 * anchorOffsets[j], anchorOffsets[j + 1] - anchorOffsets[j],
                                              params, 0, 0);
        for (int k = 0; k < 3; k++) {
            counts[3 * j + k] = r->n[k];
            if (tuplesOut != NULL) {
                tuplesOut[3 * j + k] = r->t[k];
                r->t[k] = NULL;
            }
        }
        refo_pairs_free(r);
    }
    return nJobs;
}

/* The same over chunks: OpenMP over chunks with schedule(dynamic,1), the reads of a chunk  */
/* aligned one after another by the thread that holds the chunk -- the parallel loop of     */
/* marginPolish.c:436-439 around poa_realign's per-read loop (impl/polisher.c:656-703).     */
/* Chunk c holds jobs chunkOffsets[c] .. chunkOffsets[c+1]-1. Fills counts (nJobs*3).       */
int64_t refo_align_chunks(void *modelFwd, void *modelRev, int64_t nChunks, const int64_t *chunkOffsets,
                          const int64_t *xOffsets, const uint16_t *xSymbols,
                          const int64_t *yOffsets, const uint16_t *ySymbols,
                          const int64_t *anchorOffsets, const int64_t *anchors,
                          const uint8_t *strand, const RefoParams *params, int nThreads, int64_t *counts) {
#ifdef _OPENMP
    if (nThreads > 0) {
        omp_set_num_threads(nThreads);
    }
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t c = 0; c < nChunks; c++) {
        for (int64_t j = chunkOffsets[c]; j < chunkOffsets[c + 1]; j++) {
            RefoPairs *r = refo_align_with_indels(strand[j] ? modelFwd : modelRev,
                                                  xSymbols + xOffsets[j], xOffsets[j + 1] - xOffsets[j],
                                                  ySymbols + yOffsets[j], yOffsets[j + 1] - yOffsets[j],
                                                  anchors + 3 * anchorOffsets[j],
                                                  anchorOffsets[j + 1] - anchorOffsets[j], params, 0, 0);
            for (int k = 0; k < 3; k++) {
                counts[3 * j + k] = r->n[k];
            }
            refo_pairs_free(r);
        }
    }
    return nChunks;
}

void refo_free(void *p) {
    free(p);
}

/* ------------------------------------------------------------------------ */
/* Geometry and small helpers                                                */
/* ------------------------------------------------------------------------ */

/* Writes (xay, xmyL, xmyR) for d = 0..lX+lY from band_construct (dynamic = 0,
 * impl/pairwiseAligner.c:175) or band_constructDynamic (:120). */
void refo_band(const int64_t *anchors, int64_t nAnchors, int64_t lX, int64_t lY, int64_t expansion, int dynamic,
               int64_t *out) {
    stList *anchorPairs = toAnchorList(anchors, nAnchors);
    Band *band = dynamic ? band_constructDynamic(anchorPairs, lX, lY) : band_construct(anchorPairs, lX, lY, expansion);
    BandIterator *it = bandIterator_construct(band);
    for (int64_t d = 0; d <= lX + lY; d++) {
        Diagonal g = bandIterator_getNext(it);
        out[3 * d] = g.xay;
        out[3 * d + 1] = g.xmyL;
        out[3 * d + 2] = g.xmyR;
    }
    bandIterator_destruct(it);
    band_destruct(band);
    stList_destruct(anchorPairs);
}

/* getSplitPoints (impl/pairwiseAligner.c:899-926); writes up to cap rectangles
 * (x1, y1, x2, y2) and returns the number of rectangles. */
int64_t refo_split_points(const int64_t *anchors, int64_t nAnchors, int64_t lX, int64_t lY, int64_t maxMatrixSize,
                          int raggedLeft, int raggedRight, int64_t *out, int64_t cap) {
    stList *anchorPairs = toAnchorList(anchors, nAnchors);
    stList *splits = getSplitPoints(anchorPairs, lX, lY, maxMatrixSize, raggedLeft != 0, raggedRight != 0);
    int64_t n = stList_length(splits);
    for (int64_t i = 0; i < n && i < cap; i++) {
        stIntTuple *t = stList_get(splits, i);
        for (int k = 0; k < 4; k++) {
            out[4 * i + k] = stIntTuple_get(t, k);
        }
    }
    stList_destruct(splits);
    stList_destruct(anchorPairs);
    return n;
}

double refo_logadd(double x, double y) {
    return logAdd(x, y);
}

/* computeForwardProbability (impl/pairwiseAligner.c:813-865). */
double refo_forward_probability(void *model, const uint16_t *sx, int64_t lx, const uint16_t *sy, int64_t ly,
                                const int64_t *anchors, int64_t nAnchors, const RefoParams *params,
                                int raggedLeft, int raggedRight) {
    RefoModel *m = model;
    Alphabet *a = alphabet_constructNucleotide();
    SymbolString sX = toSymbolString(a, sx, lx), sY = toSymbolString(a, sy, ly);
    stList *anchorPairs = toAnchorList(anchors, nAnchors);
    PairwiseAlignmentParameters *p = toReferenceParams(params);
    double lp = computeForwardProbability(sX, sY, anchorPairs, p, m->sM, raggedLeft != 0, raggedRight != 0);
    stList_destruct(anchorPairs);
    pairwiseAlignmentBandingParameters_destruct(p);
    symbolString_destruct(sX);
    symbolString_destruct(sY);
    alphabet_destruct(a);
    return lp;
}

/* getExpectationsUsingAnchors (impl/pairwiseAligner.c:1151-1156): transition
 * expected counts (9, from-major) and the reference's per-diagonal
 * "likelihood" accumulator. */
void refo_expectations(void *model, int hmmType, const uint16_t *sx, int64_t lx, const uint16_t *sy, int64_t ly,
                       const int64_t *anchors, int64_t nAnchors, const RefoParams *params,
                       int raggedLeft, int raggedRight, double *transitionsOut, double *likelihoodOut) {
    RefoModel *m = model;
    Alphabet *a = alphabet_constructNucleotide();
    SymbolString sX = toSymbolString(a, sx, lx), sY = toSymbolString(a, sy, ly);
    stList *anchorPairs = toAnchorList(anchors, nAnchors);
    PairwiseAlignmentParameters *p = toReferenceParams(params);
    Hmm *e = hmm_constructEmpty(0.0, (StateMachineType) hmmType, nucleotideEmissions);
    getExpectationsUsingAnchors(m->sM, e, sX, sY, anchorPairs, p, raggedLeft != 0, raggedRight != 0);
    for (int i = 0; i < 9; i++) {
        transitionsOut[i] = e->transitions[i];
    }
    *likelihoodOut = e->likelihood;
    hmm_destruct(e);
    stList_destruct(anchorPairs);
    pairwiseAlignmentBandingParameters_destruct(p);
    symbolString_destruct(sX);
    symbolString_destruct(sY);
    alphabet_destruct(a);
}

/* getMaximalExpectedAccuracyPairwiseAlignment (impl/pairwiseAligner.c:1279-1375)
 * on flat (weight, x, y) lists; writes up to cap tuples, returns the count. */
int64_t refo_mea(const int64_t *matches, int64_t nM, const int64_t *gapX, int64_t nX, const int64_t *gapY, int64_t nY,
                 int64_t lX, int64_t lY, double gapGamma, double *scoreOut, int64_t *out, int64_t cap) {
    stList *lm = stList_construct3(0, (void (*)(void *)) stIntTuple_destruct);
    stList *lx = stList_construct3(0, (void (*)(void *)) stIntTuple_destruct);
    stList *ly = stList_construct3(0, (void (*)(void *)) stIntTuple_destruct);
    for (int64_t i = 0; i < nM; i++) stList_append(lm, stIntTuple_construct3(matches[3 * i], matches[3 * i + 1], matches[3 * i + 2]));
    for (int64_t i = 0; i < nX; i++) stList_append(lx, stIntTuple_construct3(gapX[3 * i], gapX[3 * i + 1], gapX[3 * i + 2]));
    for (int64_t i = 0; i < nY; i++) stList_append(ly, stIntTuple_construct3(gapY[3 * i], gapY[3 * i + 1], gapY[3 * i + 2]));
    PairwiseAlignmentParameters *p = pairwiseAlignmentBandingParameters_construct();
    p->gapGamma = (float) gapGamma;
    stList *mea = getMaximalExpectedAccuracyPairwiseAlignment(lm, lx, ly, lX, lY, scoreOut, p);
    int64_t n = stList_length(mea);
    for (int64_t i = 0; i < n && i < cap; i++) {
        stIntTuple *t = stList_get(mea, i);
        for (int k = 0; k < 3; k++) out[3 * i + k] = stIntTuple_get(t, k);
    }
    stList_destruct(mea);
    stList_destruct(lm);
    stList_destruct(lx);
    stList_destruct(ly);
    pairwiseAlignmentBandingParameters_destruct(p);
    return n;
}
