/*
 * Drop-in implementations of the reference's pair-HMM entry points on top of
 * the C ABI in mpgpu.h (see mpgpu_dropin.h for the signatures replaced).
 *
 * stList / stIntTuple functions are the host application's sonLib; they are
 * declared here by their reference signatures and resolved at load time.
 */
#include "mpgpu_dropin.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* host sonLib (resolved at load time) */
extern stList *stList_construct3(int64_t length, void (*destructElement)(void *));
extern void stList_append(stList *list, void *item);
extern void *stList_get(stList *list, int64_t index);
extern int64_t stList_length(stList *list);
extern stIntTuple *stIntTuple_construct3(int64_t v1, int64_t v2, int64_t v3);
extern void stIntTuple_destruct(stIntTuple *t);
extern int64_t stIntTuple_get(stIntTuple *t, int64_t index);
extern int64_t stIntTuple_length(stIntTuple *t);

#define REP 51

static void recordTransition(double *fromCells, double *toCells, int64_t from, int64_t to, double eP, double tP,
                             void *extraArgs) {
    (void) fromCells;
    (void) toCells;
    (void) eP;
    ((double *) extraArgs)[from * 3 + to] = tP;
}

mp_status mpd_lower_state_machine(StateMachine *sM, mp_model_desc *d, double *rep) {
    if (sM == NULL || d == NULL || rep == NULL || sM->stateNumber != 3 || sM->emissions == NULL)
        return MP_ERR_ARGUMENT;
    memset(d, 0, sizeof(*d));
    double rec[9];
    for (int k = 0; k < 9; k++) rec[k] = NAN;
    double cur[3] = {0, 0, 0}, lower[3] = {0, 0, 0}, middle[3] = {0, 0, 0}, upper[3] = {0, 0, 0};
    sM->cellCalculate(sM, cur, lower, middle, upper, 0, 0, recordTransition, rec);
    for (int k = 0; k < 9; k++) {
        if (isnan(rec[k])) return MP_ERR_ARGUMENT;
        d->log_transitions[k] = rec[k];
    }
    for (int s = 0; s < 3; s++) {
        d->log_start[s] = sM->startStateProb(sM, s);
        d->log_ragged_start[s] = sM->raggedStartStateProb(sM, s);
        d->log_end[s] = sM->endStateProb(sM, s);
        d->log_ragged_end[s] = sM->raggedEndStateProb(sM, s);
    }
    Emissions *e = sM->emissions;
    double n44 = e->emission(e, 4, 4);
    int rle = 0;
    for (int b = 0; b < 4; b++) {
        if (e->emission(e, (Symbol) ((2 << 8) | b), (Symbol) ((2 << 8) | b)) != n44) rle = 1;
    }
    for (int b = 0; b < 5; b++) {
        d->log_gap_x[b] = e->gapEmissionX(e, (Symbol) b);
        d->log_gap_y[b] = e->gapEmissionY(e, (Symbol) b);
        for (int c = 0; c < 5; c++) d->log_match[b * 5 + c] = e->emission(e, (Symbol) b, (Symbol) c);
    }
    d->max_repeat = REP;
    d->strand = 1;
    d->run_length = rle;
    d->repeat_scale = 1.0;
    d->repeat_log10 = NULL;
    if (!rle) return MP_OK;
    /* run-length emission = match(xb, yb) + table(xb, rcX, rcY): decompose with rc 0 as the base point */
    for (int b = 0; b < 4; b++) {
        double base = e->emission(e, (Symbol) b, 0);
        for (int rx = 0; rx < REP; rx++) {
            for (int ry = 0; ry < REP; ry++) {
                rep[(b * REP + rx) * REP + ry] =
                    e->emission(e, (Symbol) ((rx << 8) | b), (Symbol) (ry << 8)) - base;
            }
        }
    }
    /* verify the decomposition on every symbol pair ('N' reads the base-0 table) */
    for (int xb = 0; xb < 5; xb++) {
        int row = xb == 4 ? 0 : xb;
        for (int yb = 0; yb < 5; yb++) {
            for (int rx = 0; rx < REP; rx++) {
                for (int ry = 0; ry < REP; ry++) {
                    double want = e->emission(e, (Symbol) ((rx << 8) | xb), (Symbol) ((ry << 8) | yb));
                    double got = d->log_match[xb * 5 + yb] + rep[(row * REP + rx) * REP + ry];
                    if (!(fabs(want - got) <= 1e-9 * (1.0 + fabs(want)))) return MP_ERR_ARGUMENT;
                }
            }
            if (e->gapEmissionX(e, (Symbol) ((3 << 8) | xb)) != d->log_gap_x[xb] ||
                e->gapEmissionY(e, (Symbol) ((3 << 8) | xb)) != d->log_gap_y[xb])
                return MP_ERR_ARGUMENT;
        }
    }
    d->repeat_log10 = rep;
    return MP_OK;
}

/* Each calling thread drives its own CUDA stream. CUDA maps streams onto a fixed number of
 * hardware work queues (8 by default), so with more calling threads than queues, unrelated
 * threads' kernels wait on one another. When the library is loaded -- before the host
 * application has created its CUDA context -- it asks for 32 queues, unless the application's
 * environment already sets CUDA_DEVICE_MAX_CONNECTIONS. */
__attribute__((constructor)) static void mpdRaiseHardwareQueues(void) {
    setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
}

/* ---------------- per-thread engine and lowered-machine cache ---------------- */

/* The reference's callers run one chunk per OpenMP thread (marginPolish.c:436-439), each thread
 * aligning its chunk's reads one after another. Every calling thread gets its own engine (its
 * own CUDA stream and device buffers) and its own cache of lowered machines, so concurrent
 * callers' passes run side by side on the GPU instead of queueing on one lock. */

#define FP_N (9 + 12 + 10 + 25 + REP)
typedef struct {
    StateMachine *sM;
    double fingerprint[FP_N];
    mp_model *model;
} CacheEntry;

#define CACHE_N 16
typedef struct {
    mp_engine *engine;
    CacheEntry cache[CACHE_N];
    int n;
} ThreadState;

static pthread_key_t gKey;
static pthread_once_t gKeyOnce = PTHREAD_ONCE_INIT;

static void destroyThreadState(void *p) {
    ThreadState *ts = p;
    if (ts == NULL) return;
    for (int i = 0; i < ts->n; i++) mp_model_destroy(ts->cache[i].model);
    mp_engine_destroy(ts->engine);
    free(ts);
}

static void makeKey(void) {
    pthread_key_create(&gKey, destroyThreadState);
}

static void die(const char *what) {
    fprintf(stderr, "mpgpu drop-in: %s: %s\n", what, mp_last_error());
    exit(1);
}

/* The calling thread's engine (created on its first call; MPGPU_DEVICE selects the device). */
static ThreadState *threadState(void) {
    pthread_once(&gKeyOnce, makeKey);
    ThreadState *ts = pthread_getspecific(gKey);
    if (ts != NULL) return ts;
    ts = calloc(1, sizeof(ThreadState));
    if (ts == NULL) die("out of memory");
    const char *dev = getenv("MPGPU_DEVICE");
    if (mp_engine_create(dev ? atoi(dev) : 0, &ts->engine) != MP_OK) die("mp_engine_create");
    pthread_setspecific(gKey, ts);
    return ts;
}

/* A machine is identified by its address and a fingerprint of its values: the 9 transitions, the
 * 12 start / end probabilities, the 10 gap emissions, the 25 base match emissions and the 51
 * run-length emissions of equal counts (bases taken in turn). A machine whose other run-length
 * entries change in place while its address stays the same is not detected: callers keep a
 * machine's tables fixed once it is built, as the reference's parser does. */
static void fingerprint(StateMachine *sM, double *fp) {
    double cur[3] = {0, 0, 0}, lower[3] = {0, 0, 0}, middle[3] = {0, 0, 0}, upper[3] = {0, 0, 0};
    sM->cellCalculate(sM, cur, lower, middle, upper, 0, 0, recordTransition, fp);
    int k = 9;
    for (int s = 0; s < 3; s++) {
        fp[k++] = sM->startStateProb(sM, s);
        fp[k++] = sM->endStateProb(sM, s);
        fp[k++] = sM->raggedStartStateProb(sM, s);
        fp[k++] = sM->raggedEndStateProb(sM, s);
    }
    Emissions *e = sM->emissions;
    for (int b = 0; b < 5; b++) {
        fp[k++] = e->gapEmissionX(e, (Symbol) b);
        fp[k++] = e->gapEmissionY(e, (Symbol) b);
    }
    for (int b = 0; b < 25; b++) fp[k++] = e->emission(e, (Symbol) (b / 5), (Symbol) (b % 5));
    for (int rc = 0; rc < REP; rc++) fp[k++] = e->emission(e, (Symbol) ((rc << 8) | (rc & 3)), (Symbol) ((rc << 8) | (rc & 3)));
}

static mp_model *modelFor(ThreadState *ts, StateMachine *sM) {
    double fp[FP_N];
    fingerprint(sM, fp);
    for (int i = 0; i < ts->n; i++) {
        if (ts->cache[i].sM == sM && memcmp(ts->cache[i].fingerprint, fp, sizeof(fp)) == 0) return ts->cache[i].model;
    }
    mp_model_desc d;
    double *rep = malloc(sizeof(double) * 4 * REP * REP);
    if (rep == NULL) die("out of memory");
    if (mpd_lower_state_machine(sM, &d, rep) != MP_OK) {
        fprintf(stderr, "mpgpu drop-in: state machine emissions are not of the supported 3-state form\n");
        exit(1);
    }
    mp_model *m = NULL;
    if (mp_model_create(ts->engine, &d, &d, &m) != MP_OK) die("mp_model_create");
    free(rep);
    if (ts->n == CACHE_N) {
        mp_model_destroy(ts->cache[0].model);
        memmove(ts->cache, ts->cache + 1, sizeof(CacheEntry) * (CACHE_N - 1));
        ts->n--;
    }
    ts->cache[ts->n].sM = sM;
    memcpy(ts->cache[ts->n].fingerprint, fp, sizeof(fp));
    ts->cache[ts->n].model = m;
    ts->n++;
    return m;
}

static stList *toList(const mp_result_view *v, int k) {
    stList *l = stList_construct3(0, (void (*)(void *)) stIntTuple_destruct);
    for (int64_t i = v->offsets[k][0]; i < v->offsets[k][1]; i++) {
        stList_append(l, stIntTuple_construct3(v->weight[k][i], v->x[k][i], v->y[k][i]));
    }
    return l;
}

static void toParams(const PairwiseAlignmentParameters *p, mp_params *q) {
    memset(q, 0, sizeof(*q));
    q->threshold = p->threshold;
    q->min_diags_between_traceback = p->minDiagsBetweenTraceBack;
    q->traceback_diagonals = p->traceBackDiagonals;
    q->diagonal_expansion = p->diagonalExpansion;
    q->constraint_diagonal_trim = p->constraintDiagonalTrim;
    q->split_matrix_bigger_than_this = p->splitMatrixBiggerThanThis;
    q->dynamic_anchor_expansion = p->dynamicAnchorExpansion ? 1 : 0;
    q->gap_gamma = p->gapGamma;
}

/* One job's host batch over the caller's symbol strings and anchor list. `an` receives the
 * anchors as int32 triples; with ownExpansion the anchors' third values are used (else the
 * default expansion, or 0 when zeroExpansion). */
typedef struct {
    mp_batch b;
    int32_t *an;
    uint16_t zero;
    int64_t xb, xe, yoff[2], aoff[2];
    uint8_t strand, rl, rr;
} OneJob;

static void oneJob(OneJob *j, SymbolString sX, SymbolString sY, stList *anchorPairs, int64_t defaultExpansion,
                   int zeroExpansion, bool raggedLeft, bool raggedRight) {
    int64_t nA = anchorPairs ? stList_length(anchorPairs) : 0;
    j->an = malloc(sizeof(int32_t) * 3 * (nA > 0 ? nA : 1));
    if (j->an == NULL) die("out of memory");
    for (int64_t i = 0; i < nA; i++) {
        stIntTuple *t = stList_get(anchorPairs, i);
        j->an[3 * i] = (int32_t) stIntTuple_get(t, 0);
        j->an[3 * i + 1] = (int32_t) stIntTuple_get(t, 1);
        j->an[3 * i + 2] = zeroExpansion ? 0
                                         : (int32_t) (stIntTuple_length(t) >= 3 ? stIntTuple_get(t, 2) : defaultExpansion);
    }
    j->zero = 0;
    j->xb = 0;
    j->xe = sX.length;
    j->yoff[0] = 0;
    j->yoff[1] = sY.length;
    j->aoff[0] = 0;
    j->aoff[1] = nA;
    j->strand = 1;
    j->rl = raggedLeft ? 1 : 0;
    j->rr = raggedRight ? 1 : 0;
    memset(&j->b, 0, sizeof(j->b));
    j->b.n_jobs = 1;
    j->b.x_begin = &j->xb;
    j->b.x_end = &j->xe;
    j->b.x_symbols_length = sX.length;
    j->b.x_symbols = sX.length > 0 ? sX.sequence : &j->zero;
    j->b.y_offsets = j->yoff;
    j->b.y_symbols = sY.length > 0 ? sY.sequence : &j->zero;
    j->b.anchor_offsets = j->aoff;
    j->b.anchors = j->an;
    j->b.strand = &j->strand;
    j->b.ragged_left = &j->rl;
    j->b.ragged_right = &j->rr;
}

/* computeForwardProbability (impl/pairwiseAligner.c:813-865). */
double computeForwardProbability(SymbolString sX, SymbolString sY, stList *anchorPairs, PairwiseAlignmentParameters *p,
                                 StateMachine *sM, bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd) {
    ThreadState *ts = threadState();
    mp_model *m = modelFor(ts, sM);
    OneJob j;
    /* band_construct ignores the anchors' own expansions */
    oneJob(&j, sX, sY, anchorPairs, 0, 1, alignmentHasRaggedLeftEnd, alignmentHasRaggedRightEnd);
    mp_params q;
    toParams(p, &q);
    double lp = 0.0;
    if (mp_forward_batch(ts->engine, m, &q, &j.b, &lp) != MP_OK) die("computeForwardProbability");
    free(j.an);
    return lp;
}

static void run(StateMachine *sM, SymbolString sX, SymbolString sY, stList *anchorPairs,
                PairwiseAlignmentParameters *p, stList **alignedPairs, stList **gapXPairs, stList **gapYPairs,
                bool raggedLeft, bool raggedRight) {
    ThreadState *ts = threadState();
    mp_model *m = modelFor(ts, sM);
    OneJob j;
    oneJob(&j, sX, sY, anchorPairs, p->diagonalExpansion, 0, raggedLeft, raggedRight);
    mp_params q;
    toParams(p, &q);
    mp_result *r = NULL;
    if (mp_realign_batch(ts->engine, m, &q, &j.b, &r) != MP_OK) die("getAlignedPairsWithIndelsUsingAnchors");
    mp_result_view v;
    mp_result_view_get(r, &v);
    if (alignedPairs) *alignedPairs = toList(&v, 0);
    if (gapXPairs) *gapXPairs = toList(&v, 1);
    if (gapYPairs) *gapYPairs = toList(&v, 2);
    mp_result_destroy(r);
    free(j.an);
}

/* getExpectationsUsingAnchors (impl/pairwiseAligner.c:1151-1156): adds to the caller's Hmm the
 * Baum-Welch transition expectations E[n_ij] = sum over cells of exp(f_i + t_ij + e_j + b_j - ln P)
 * (impl/pairwiseAligner.c:347-357), through mp_expectations_batch, and the reference's likelihood
 * term (its diagonalCalculationExpectations adds the total once per posterior diagonal, :674).
 * Emission expectations stay untouched: the reference has them disabled (:359-362). */
void getExpectationsUsingAnchors(StateMachine *sM, Hmm *hmmExpectations, SymbolString sX, SymbolString sY,
                                 stList *anchorPairs, PairwiseAlignmentParameters *p, bool alignmentHasRaggedLeftEnd,
                                 bool alignmentHasRaggedRightEnd) {
    if (hmmExpectations == NULL || hmmExpectations->stateNumber != 3 || hmmExpectations->transitions == NULL) {
        fprintf(stderr, "mpgpu drop-in: getExpectationsUsingAnchors needs a 3-state Hmm\n");
        exit(1);
    }
    ThreadState *ts = threadState();
    mp_model *m = modelFor(ts, sM);
    OneJob j;
    oneJob(&j, sX, sY, anchorPairs, p->diagonalExpansion, 0, alignmentHasRaggedLeftEnd, alignmentHasRaggedRightEnd);
    mp_params q;
    toParams(p, &q);
    mp_expectations *ex = malloc(sizeof(mp_expectations));
    if (ex == NULL) die("out of memory");
    double ll = 0.0;
    if (mp_expectations_batch(ts->engine, m, &q, &j.b, ex, &ll) != MP_OK) die("getExpectationsUsingAnchors");
    for (int i = 0; i < 9; i++) hmmExpectations->transitions[i] += ex->transitions[0][i];
    /* one total per posterior diagonal d = 1 .. lX + lY, every total being ln P */
    if (sX.length + sY.length > 0) hmmExpectations->likelihood += (double) (sX.length + sY.length) * ll;
    free(ex);
    free(j.an);
}

/* getExpectations (impl/pairwiseAligner.c:1158-1164): the same without anchors. */
void getExpectations(StateMachine *sM, Hmm *hmmExpectations, SymbolString sX, SymbolString sY,
                     PairwiseAlignmentParameters *p, bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd) {
    getExpectationsUsingAnchors(sM, hmmExpectations, sX, sY, NULL, p, alignmentHasRaggedLeftEnd,
                                alignmentHasRaggedRightEnd);
}

void getAlignedPairsWithIndelsUsingAnchors(StateMachine *sM, SymbolString sX, SymbolString sY, stList *anchorPairs,
                                           PairwiseAlignmentParameters *p, stList **alignedPairs, stList **gapXPairs,
                                           stList **gapYPairs, bool alignmentHasRaggedLeftEnd,
                                           bool alignmentHasRaggedRightEnd) {
    run(sM, sX, sY, anchorPairs, p, alignedPairs, gapXPairs, gapYPairs, alignmentHasRaggedLeftEnd,
        alignmentHasRaggedRightEnd);
}

stList *getAlignedPairsUsingAnchors(StateMachine *sM, SymbolString sX, SymbolString sY, stList *anchorPairs,
                                    PairwiseAlignmentParameters *p, bool alignmentHasRaggedLeftEnd,
                                    bool alignmentHasRaggedRightEnd) {
    stList *m = NULL;
    run(sM, sX, sY, anchorPairs, p, &m, NULL, NULL, alignmentHasRaggedLeftEnd, alignmentHasRaggedRightEnd);
    return m;
}

void getAlignedPairsWithIndels(StateMachine *sM, SymbolString sX, SymbolString sY, PairwiseAlignmentParameters *p,
                               stList **alignedPairs, stList **gapXPairs, stList **gapYPairs,
                               bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd) {
    run(sM, sX, sY, NULL, p, alignedPairs, gapXPairs, gapYPairs, alignmentHasRaggedLeftEnd,
        alignmentHasRaggedRightEnd);
}

stList *getAlignedPairs(StateMachine *sM, SymbolString sX, SymbolString sY, PairwiseAlignmentParameters *p,
                        bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd) {
    stList *m = NULL;
    run(sM, sX, sY, NULL, p, &m, NULL, NULL, alignmentHasRaggedLeftEnd, alignmentHasRaggedRightEnd);
    return m;
}
