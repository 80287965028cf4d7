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

/* ---------------- process-wide engine and lowered-machine cache ---------------- */

typedef struct {
    StateMachine *sM;
    double fingerprint[12];
    mp_model *model;
} CacheEntry;

static pthread_mutex_t gLock = PTHREAD_MUTEX_INITIALIZER;
static mp_engine *gEngine = NULL;
static CacheEntry gCache[64];
static int gCacheN = 0;

static void die(const char *what) {
    fprintf(stderr, "mpgpu drop-in: %s: %s\n", what, mp_last_error());
    exit(1);
}

static void fingerprint(StateMachine *sM, double *fp) {
    double cur[3] = {0, 0, 0}, lower[3] = {0, 0, 0}, middle[3] = {0, 0, 0}, upper[3] = {0, 0, 0};
    sM->cellCalculate(sM, cur, lower, middle, upper, 0, 0, recordTransition, fp);
    Emissions *e = sM->emissions;
    fp[9] = e->emission(e, (Symbol) ((3 << 8) | 1), (Symbol) ((5 << 8) | 2));
    fp[10] = e->gapEmissionX(e, 2);
    fp[11] = e->gapEmissionY(e, 3);
}

static mp_model *modelFor(StateMachine *sM) {
    double fp[12];
    fingerprint(sM, fp);
    for (int i = 0; i < gCacheN; i++) {
        if (gCache[i].sM == sM && memcmp(gCache[i].fingerprint, fp, sizeof(fp)) == 0) return gCache[i].model;
    }
    mp_model_desc d;
    double *rep = malloc(sizeof(double) * 4 * REP * REP);
    if (rep == NULL) die("out of memory");
    if (mpd_lower_state_machine(sM, &d, rep) != MP_OK) {
        fprintf(stderr, "mpgpu drop-in: state machine emissions are not of the supported 3-state form\n");
        exit(1);
    }
    mp_model *m = NULL;
    if (mp_model_create(gEngine, &d, &d, &m) != MP_OK) die("mp_model_create");
    free(rep);
    if (gCacheN == 64) {
        mp_model_destroy(gCache[0].model);
        memmove(gCache, gCache + 1, sizeof(CacheEntry) * 63);
        gCacheN--;
    }
    gCache[gCacheN].sM = sM;
    memcpy(gCache[gCacheN].fingerprint, fp, sizeof(fp));
    gCache[gCacheN].model = m;
    gCacheN++;
    return m;
}

static void ensureEngine(void) {
    if (gEngine != NULL) return;
    const char *dev = getenv("MPGPU_DEVICE");
    if (mp_engine_create(dev ? atoi(dev) : 0, &gEngine) != MP_OK) die("mp_engine_create");
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

/* computeForwardProbability (impl/pairwiseAligner.c:813-865). */
double computeForwardProbability(SymbolString sX, SymbolString sY, stList *anchorPairs, PairwiseAlignmentParameters *p,
                                 StateMachine *sM, bool alignmentHasRaggedLeftEnd, bool alignmentHasRaggedRightEnd) {
    pthread_mutex_lock(&gLock);
    ensureEngine();
    mp_model *m = modelFor(sM);
    int64_t nA = anchorPairs ? stList_length(anchorPairs) : 0;
    int32_t *an = malloc(sizeof(int32_t) * 3 * (nA > 0 ? nA : 1));
    if (an == NULL) die("out of memory");
    for (int64_t i = 0; i < nA; i++) {
        stIntTuple *t = stList_get(anchorPairs, i);
        an[3 * i] = (int32_t) stIntTuple_get(t, 0);
        an[3 * i + 1] = (int32_t) stIntTuple_get(t, 1);
        an[3 * i + 2] = 0;  /* band_construct ignores the anchors' own expansions */
    }
    uint16_t zero = 0;
    int64_t xb = 0, xe = sX.length, yoff[2] = {0, sY.length}, aoff[2] = {0, nA};
    uint8_t strand = 1, rl = alignmentHasRaggedLeftEnd ? 1 : 0, rr = alignmentHasRaggedRightEnd ? 1 : 0;
    mp_batch b;
    memset(&b, 0, sizeof(b));
    b.n_jobs = 1;
    b.x_begin = &xb;
    b.x_end = &xe;
    b.x_symbols_length = sX.length;
    b.x_symbols = sX.length > 0 ? sX.sequence : &zero;
    b.y_offsets = yoff;
    b.y_symbols = sY.length > 0 ? sY.sequence : &zero;
    b.anchor_offsets = aoff;
    b.anchors = an;
    b.strand = &strand;
    b.ragged_left = &rl;
    b.ragged_right = &rr;
    mp_params q;
    toParams(p, &q);
    double lp = 0.0;
    if (mp_forward_batch(gEngine, m, &q, &b, &lp) != MP_OK) die("computeForwardProbability");
    free(an);
    pthread_mutex_unlock(&gLock);
    return lp;
}

static void run(StateMachine *sM, SymbolString sX, SymbolString sY, stList *anchorPairs,
                PairwiseAlignmentParameters *p, stList **alignedPairs, stList **gapXPairs, stList **gapYPairs,
                bool raggedLeft, bool raggedRight) {
    pthread_mutex_lock(&gLock);
    ensureEngine();
    mp_model *m = modelFor(sM);
    int64_t nA = anchorPairs ? stList_length(anchorPairs) : 0;
    int32_t *an = malloc(sizeof(int32_t) * 3 * (nA > 0 ? nA : 1));
    if (an == NULL) die("out of memory");
    for (int64_t i = 0; i < nA; i++) {
        stIntTuple *t = stList_get(anchorPairs, i);
        an[3 * i] = (int32_t) stIntTuple_get(t, 0);
        an[3 * i + 1] = (int32_t) stIntTuple_get(t, 1);
        an[3 * i + 2] = (int32_t) (stIntTuple_length(t) >= 3 ? stIntTuple_get(t, 2) : p->diagonalExpansion);
    }
    uint16_t zero = 0;
    int64_t xb = 0, xe = sX.length, yoff[2] = {0, sY.length}, aoff[2] = {0, nA};
    uint8_t strand = 1, rl = raggedLeft ? 1 : 0, rr = raggedRight ? 1 : 0;
    mp_batch b;
    memset(&b, 0, sizeof(b));
    b.n_jobs = 1;
    b.x_begin = &xb;
    b.x_end = &xe;
    b.x_symbols_length = sX.length;
    b.x_symbols = sX.length > 0 ? sX.sequence : &zero;
    b.y_offsets = yoff;
    b.y_symbols = sY.length > 0 ? sY.sequence : &zero;
    b.anchor_offsets = aoff;
    b.anchors = an;
    b.strand = &strand;
    b.ragged_left = &rl;
    b.ragged_right = &rr;
    mp_params q;
    toParams(p, &q);
    mp_result *r = NULL;
    if (mp_realign_batch(gEngine, m, &q, &b, &r) != MP_OK) die("getAlignedPairsWithIndelsUsingAnchors");
    mp_result_view v;
    mp_result_view_get(r, &v);
    if (alignedPairs) *alignedPairs = toList(&v, 0);
    if (gapXPairs) *gapXPairs = toList(&v, 1);
    if (gapYPairs) *gapYPairs = toList(&v, 2);
    mp_result_destroy(r);
    free(an);
    pthread_mutex_unlock(&gLock);
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
