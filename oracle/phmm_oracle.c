/*
 * ORACLE B -- TEST INFRASTRUCTURE ONLY (see phmm_oracle.h).
 *
 * FP64 log-space restatement of the reference's banded posterior schedule.
 * Every routine names the reference lines it follows. Operation order inside
 * a cell (which neighbour first, which state first, the grouping
 * f + (e + t)) follows the reference, so that swapping in the reference's
 * approximate logAdd reproduces its output bit for bit.
 */
#include "phmm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define NEG_INF (-INFINITY)

/* Integer probability scale (inc/pairwiseAligner.h:26). */
#define PROB_ONE_INT 10000000

double mpo_logadd_exact(double a, double b) {
    if (a < b) {
        double t = a;
        a = b;
        b = t;
    }
    if (b == NEG_INF) {
        return a;
    }
    return a + log1p(exp(b - a));
}

/* ------------------------------------------------------------------ */
/* Emissions (impl/stateMachine.c:360-380 nucleotide, :708-722 RLE)    */
/* ------------------------------------------------------------------ */

static int symbolBase(const MpoModel *m, uint16_t s) {
    int b = m->runLength ? (s & 255) : s;
    return b >= 4 ? 4 : b;
}

double mpo_match_emission(const MpoModel *m, uint16_t cx, uint16_t cy) {
    int xb = symbolBase(m, cx), yb = symbolBase(m, cy);
    double e = m->match[xb * 5 + yb];
    if (m->runLength && m->repeat10 != NULL) {
        int64_t M = m->maxRepeat;
        int64_t rx = cx >> 8, ry = cy >> 8;
        int b = xb == 4 ? 0 : xb; /* 'N' reads the A table (impl/polisher.c:1758) */
        int row = m->strand ? b : 3 - b;
        if (rx >= M || ry >= M) {
            fprintf(stderr, "oracle: repeat count out of range (%d, %d)\n", (int) rx, (int) ry);
            abort();
        }
        e = e + m->repeatScale * m->repeat10[(row * M + rx) * M + ry];
    }
    return e;
}

double mpo_gap_x_emission(const MpoModel *m, uint16_t cx) {
    return m->gapX[symbolBase(m, cx)];
}

double mpo_gap_y_emission(const MpoModel *m, uint16_t cy) {
    return m->gapY[symbolBase(m, cy)];
}

/* ------------------------------------------------------------------ */
/* Band geometry (impl/pairwiseAligner.c:86-173)                        */
/* ------------------------------------------------------------------ */

static int64_t clampCoordinate(int64_t z, int64_t lZ) {
    return z < 0 ? 0 : (z > lZ ? lZ : z);
}

/* One anti-diagonal of the box (xL, yL)-(xU, yU): band_setCurrentDiagonal. */
static int boxDiagonal(int64_t d, int64_t xL, int64_t yL, int64_t xU, int64_t yU, int64_t *lo, int64_t *hi) {
    int64_t l = xL - yL, h = xU - yU;
    if ((d + l) & 1) l++;
    if ((d + h) & 1) h++;
    int64_t x = (d + l) / 2;
    if (x < xL) l += 2 * (xL - x);
    int64_t y = (d - l) / 2;
    if (yL < y) l += 2 * (y - yL);
    x = (d + h) / 2;
    if (xU < x) h -= 2 * (x - xU);
    y = (d - h) / 2;
    if (y < yU) h -= 2 * (yU - y);
    if (l > h) {
        return -1;
    }
    *lo = l;
    *hi = h;
    return 0;
}

int mpo_band(const int64_t *anchors, int64_t nAnchors, int64_t lX, int64_t lY, int64_t expansion, int dynamic,
             int64_t *out) {
    int64_t xL = 0, yL = 0, xU = 0, yU = 0;
    int64_t e = dynamic ? 0 : expansion;
    int64_t nx = 0, ny = 0, k = 0;
    for (int64_t d = 0; d <= lX + lY; d++) {
        int64_t lo, hi;
        if (boxDiagonal(d, xL, yL, xU, yU, &lo, &hi) != 0) {
            return -1;
        }
        out[3 * d] = d;
        out[3 * d + 1] = lo;
        out[3 * d + 2] = hi;
        if (d == nx + ny) { /* reached the next anchor: it becomes the previous one */
            int64_t px = nx, py = ny;
            if (k < nAnchors) {
                nx = anchors[3 * k] + 1; /* matrix coordinates are sequence + 1 */
                ny = anchors[3 * k + 1] + 1;
                if (dynamic) {
                    e = anchors[3 * k + 2];
                }
                k++;
            } else {
                nx = lX;
                ny = lY;
            }
            int64_t pxay = px + py, pxmy = px - py, nxay = nx + ny, nxmy = nx - ny;
            xL = clampCoordinate((pxay + (pxmy - e)) / 2, lX);
            yL = clampCoordinate((nxay - (nxmy - e)) / 2, lY);
            xU = clampCoordinate((nxay + (nxmy + e)) / 2, lX);
            yU = clampCoordinate((pxay - (pxmy + e)) / 2, lY);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Split rectangles (impl/pairwiseAligner.c:875-926)                    */
/* ------------------------------------------------------------------ */

static int splitAtGap(int64_t *x1, int64_t *y1, int64_t x2, int64_t y2, int64_t x3, int64_t y3, int64_t maxSize,
                      int skip, int64_t *out, int64_t cap, int64_t *n) {
    int64_t gx = x3 - x2, gy = y3 - y2;
    if (gx * gy > maxSize) {
        int64_t side = (int64_t) sqrt((double) maxSize);
        int64_t hX = gx / 2 > side ? side : gx / 2;
        int64_t hY = gy / 2 > side ? side : gy / 2;
        if (!skip) {
            if (*n < cap) {
                out[4 * *n] = *x1;
                out[4 * *n + 1] = *y1;
                out[4 * *n + 2] = x2 + hX;
                out[4 * *n + 3] = y2 + hY;
            }
            (*n)++;
        }
        *x1 = x3 - hX;
        *y1 = y3 - hY;
        return 1;
    }
    return 0;
}

int64_t mpo_split_points(const int64_t *anchors, int64_t nAnchors, int64_t lX, int64_t lY, int64_t maxMatrixSize,
                         int raggedLeft, int raggedRight, int64_t *out, int64_t cap) {
    int64_t x1 = 0, y1 = 0, x2 = 0, y2 = 0, n = 0;
    for (int64_t i = 0; i < nAnchors; i++) {
        int64_t x3 = anchors[3 * i], y3 = anchors[3 * i + 1];
        splitAtGap(&x1, &y1, x2, y2, x3, y3, maxMatrixSize, raggedLeft && i == 0, out, cap, &n);
        x2 = x3 + 1;
        y2 = y3 + 1;
    }
    int split = splitAtGap(&x1, &y1, x2, y2, lX, lY, maxMatrixSize, raggedLeft && nAnchors == 0, out, cap, &n);
    if (!split || !raggedRight) {
        if (n < cap) {
            out[4 * n] = x1;
            out[4 * n + 1] = y1;
            out[4 * n + 2] = lX;
            out[4 * n + 3] = lY;
        }
        n++;
    }
    return n;
}

/* ------------------------------------------------------------------ */
/* Growable tuple buffers                                              */
/* ------------------------------------------------------------------ */

typedef struct {
    int64_t n, cap;
    int64_t *t;
} TupleBuf;

static void tupleAppend(TupleBuf *b, int64_t w, int64_t x, int64_t y) {
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 256;
        b->t = realloc(b->t, sizeof(int64_t) * 3 * b->cap);
        if (b->t == NULL) {
            abort();
        }
    }
    b->t[3 * b->n] = w;
    b->t[3 * b->n + 1] = x;
    b->t[3 * b->n + 2] = y;
    b->n++;
}

typedef struct {
    int64_t n, cap;
    double *v;
    double floor; /* records are kept when one of the cell's posteriors is at least this */
} DenseBuf;

static void denseAppend(DenseBuf *b, double x, double y, double pm, double px, double py) {
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 1024;
        b->v = realloc(b->v, sizeof(double) * 5 * b->cap);
        if (b->v == NULL) {
            abort();
        }
    }
    double *r = b->v + 5 * b->n;
    r[0] = x;
    r[1] = y;
    r[2] = pm;
    r[3] = px;
    r[4] = py;
    b->n++;
}

/* ------------------------------------------------------------------ */
/* One banded sub-problem: getPosteriorProbsWithBanding                */
/* (impl/pairwiseAligner.c:687-808) with the indel posterior callback  */
/* diagonalCalculationPosteriorProbs (:622-664).                       */
/* ------------------------------------------------------------------ */

typedef struct {
    const MpoModel *m;
    const MpoParams *p;
    MpoLogAddFn add;
    const uint16_t *sx, *sy;
    int64_t lx, ly, N;
    int64_t *lo, *hi, *off; /* band per diagonal; flat cell offset per diagonal */
    double *F, *B;          /* cells*3 log values */
    char *bLive;            /* backward diagonal currently allocated (reference: non-NULL) */
} Sub;

static inline double *cellOf(const Sub *s, double *base, int64_t d, int64_t xmy) {
    if (d < 0 || d > s->N || xmy < s->lo[d] || xmy > s->hi[d]) {
        return NULL;
    }
    return base + 3 * (s->off[d] + (xmy - s->lo[d]) / 2);
}

static inline uint16_t xSymbolAt(const Sub *s, int64_t d, int64_t xmy) {
    int64_t x = (d + xmy) / 2;
    return x > 0 ? s->sx[x - 1] : 4; /* the reference's x = 0 placeholder (:528-532) */
}

static inline uint16_t ySymbolAt(const Sub *s, int64_t d, int64_t xmy) {
    int64_t y = (d - xmy) / 2;
    return y > 0 ? s->sy[y - 1] : 4;
}

static void resetDiagonal(Sub *s, double *base, int64_t d) {
    double *c = base + 3 * s->off[d];
    int64_t n = 3 * ((s->hi[d] - s->lo[d]) / 2 + 1);
    for (int64_t i = 0; i < n; i++) {
        c[i] = NEG_INF;
    }
}

static void setDiagonal(Sub *s, double *base, int64_t d, const double *v) {
    for (int64_t xmy = s->lo[d]; xmy <= s->hi[d]; xmy += 2) {
        double *c = cellOf(s, base, d, xmy);
        c[0] = v[0];
        c[1] = v[1];
        c[2] = v[2];
    }
}

/* Forward cell update (stateMachine3_cellCalculate with doTransitionForward). */
static void forwardDiagonal(Sub *s, int64_t d) {
    const double *t = s->m->trans;
    for (int64_t xmy = s->lo[d]; xmy <= s->hi[d]; xmy += 2) {
        double *cur = cellOf(s, s->F, d, xmy);
        double *lower = cellOf(s, s->F, d - 1, xmy - 1);
        double *middle = d >= 2 ? cellOf(s, s->F, d - 2, xmy) : NULL;
        double *upper = cellOf(s, s->F, d - 1, xmy + 1);
        uint16_t cx = xSymbolAt(s, d, xmy), cy = ySymbolAt(s, d, xmy);
        if (lower != NULL) {
            double e = mpo_gap_x_emission(s->m, cx);
            cur[1] = s->add(cur[1], lower[0] + (e + t[0 * 3 + 1]));
            cur[1] = s->add(cur[1], lower[1] + (e + t[1 * 3 + 1]));
            cur[1] = s->add(cur[1], lower[2] + (e + t[2 * 3 + 1]));
        }
        if (middle != NULL) {
            double e = mpo_match_emission(s->m, cx, cy);
            cur[0] = s->add(cur[0], middle[0] + (e + t[0 * 3 + 0]));
            cur[0] = s->add(cur[0], middle[1] + (e + t[1 * 3 + 0]));
            cur[0] = s->add(cur[0], middle[2] + (e + t[2 * 3 + 0]));
        }
        if (upper != NULL) {
            double e = mpo_gap_y_emission(s->m, cy);
            cur[2] = s->add(cur[2], upper[0] + (e + t[0 * 3 + 2]));
            cur[2] = s->add(cur[2], upper[2] + (e + t[2 * 3 + 2]));
            cur[2] = s->add(cur[2], upper[1] + (e + t[1 * 3 + 2]));
        }
    }
}

/* Backward push from diagonal d into d-1 and d-2 (doTransitionBackward). */
static void backwardDiagonal(Sub *s, int64_t d) {
    const double *t = s->m->trans;
    int live1 = d - 1 >= 0 && s->bLive[d - 1];
    int live2 = d - 2 >= 0 && s->bLive[d - 2];
    for (int64_t xmy = s->lo[d]; xmy <= s->hi[d]; xmy += 2) {
        double *cur = cellOf(s, s->B, d, xmy);
        double *lower = live1 ? cellOf(s, s->B, d - 1, xmy - 1) : NULL;
        double *middle = live2 ? cellOf(s, s->B, d - 2, xmy) : NULL;
        double *upper = live1 ? cellOf(s, s->B, d - 1, xmy + 1) : NULL;
        uint16_t cx = xSymbolAt(s, d, xmy), cy = ySymbolAt(s, d, xmy);
        if (lower != NULL) {
            double e = mpo_gap_x_emission(s->m, cx);
            lower[0] = s->add(lower[0], cur[1] + (e + t[0 * 3 + 1]));
            lower[1] = s->add(lower[1], cur[1] + (e + t[1 * 3 + 1]));
            lower[2] = s->add(lower[2], cur[1] + (e + t[2 * 3 + 1]));
        }
        if (middle != NULL) {
            double e = mpo_match_emission(s->m, cx, cy);
            middle[0] = s->add(middle[0], cur[0] + (e + t[0 * 3 + 0]));
            middle[1] = s->add(middle[1], cur[0] + (e + t[1 * 3 + 0]));
            middle[2] = s->add(middle[2], cur[0] + (e + t[2 * 3 + 0]));
        }
        if (upper != NULL) {
            double e = mpo_gap_y_emission(s->m, cy);
            upper[0] = s->add(upper[0], cur[2] + (e + t[0 * 3 + 2]));
            upper[2] = s->add(upper[2], cur[2] + (e + t[2 * 3 + 2]));
            upper[1] = s->add(upper[1], cur[2] + (e + t[1 * 3 + 2]));
        }
    }
}

static double cellDot(const Sub *s, const double *a, const double *b) {
    double v = a[0] + b[0];
    v = s->add(v, a[1] + b[1]);
    v = s->add(v, a[2] + b[2]);
    return v;
}

/* diagonalCalculationTotalProbability (:567-584). */
static double totalProbability(Sub *s, int64_t d) {
    double total = NEG_INF;
    for (int64_t xmy = s->lo[d]; xmy <= s->hi[d]; xmy += 2) {
        total = s->add(total, cellDot(s, cellOf(s, s->F, d, xmy), cellOf(s, s->B, d, xmy)));
    }
    if (d + 1 <= s->N && s->bLive[d + 1] && d - 1 >= 0) {
        const double *t = s->m->trans;
        double crossing = NEG_INF;
        for (int64_t xmy = s->lo[d + 1]; xmy <= s->hi[d + 1]; xmy += 2) {
            double mcell[3] = {NEG_INF, NEG_INF, NEG_INF};
            double *middle = cellOf(s, s->F, d - 1, xmy);
            if (middle != NULL) {
                double e = mpo_match_emission(s->m, xSymbolAt(s, d + 1, xmy), ySymbolAt(s, d + 1, xmy));
                mcell[0] = s->add(mcell[0], middle[0] + (e + t[0 * 3 + 0]));
                mcell[0] = s->add(mcell[0], middle[1] + (e + t[1 * 3 + 0]));
                mcell[0] = s->add(mcell[0], middle[2] + (e + t[2 * 3 + 0]));
            }
            crossing = s->add(crossing, cellDot(s, mcell, cellOf(s, s->B, d + 1, xmy)));
        }
        total = s->add(total, crossing);
    }
    return total;
}

/* addPosteriorProb (:586-595). */
static void addPosterior(const MpoParams *p, TupleBuf *b, int64_t x, int64_t y, double prob) {
    if (prob >= p->threshold) {
        if (prob > 1.0) {
            prob = 1.0;
        }
        prob = floor(prob * PROB_ONE_INT);
        tupleAppend(b, (int64_t) prob, x - 1, y - 1);
    }
}

static void posteriorDiagonal(Sub *s, int64_t d, double total, TupleBuf *out, DenseBuf *dense) {
    for (int64_t xmy = s->lo[d]; xmy <= s->hi[d]; xmy += 2) {
        int64_t x = (d + xmy) / 2, y = (d - xmy) / 2;
        double *f = cellOf(s, s->F, d, xmy), *b = cellOf(s, s->B, d, xmy);
        double pm = -1.0, px = -1.0, py = -1.0;
        if (x > 0 && y > 0) {
            pm = exp((f[0] + b[0]) - total);
            addPosterior(s->p, &out[0], x, y, pm);
        }
        if (x > 0) {
            px = exp((f[1] + b[1]) - total);
            addPosterior(s->p, &out[1], x, y, px);
        }
        if (y > 0) {
            py = exp((f[2] + b[2]) - total);
            addPosterior(s->p, &out[2], x, y, py);
        }
        if (dense != NULL && (pm >= dense->floor || px >= dense->floor || py >= dense->floor)) {
            denseAppend(dense, (double) (x - 1), (double) (y - 1), pm, px, py);
        }
    }
}

/* Returns 0 on success, -1 on an invalid band. Appends emissions to out[3]
 * in the reference's emission order; *logLik is the final segment's log total. */
static int runSubProblem(const MpoModel *m, const MpoParams *p, MpoLogAddFn add, const uint16_t *sx, int64_t lx,
                         const uint16_t *sy, int64_t ly, const int64_t *anchors, int64_t nAnchors, int raggedLeft,
                         int raggedRight, TupleBuf *out, DenseBuf *dense, double *logLik, int64_t *cells) {
    Sub s;
    memset(&s, 0, sizeof(s));
    s.m = m;
    s.p = p;
    s.add = add;
    s.sx = sx;
    s.sy = sy;
    s.lx = lx;
    s.ly = ly;
    s.N = lx + ly;
    *logLik = 0.0;
    if (s.N == 0) {
        *cells = 0;
        return 0;
    }
    int64_t *band = malloc(sizeof(int64_t) * 3 * (s.N + 1));
    if (mpo_band(anchors, nAnchors, lx, ly, p->diagonalExpansion, p->dynamicAnchorExpansion != 0, band) != 0) {
        free(band);
        return -1;
    }
    s.lo = malloc(sizeof(int64_t) * (s.N + 1));
    s.hi = malloc(sizeof(int64_t) * (s.N + 1));
    s.off = malloc(sizeof(int64_t) * (s.N + 2));
    int64_t total = 0;
    for (int64_t d = 0; d <= s.N; d++) {
        s.lo[d] = band[3 * d + 1];
        s.hi[d] = band[3 * d + 2];
        s.off[d] = total;
        total += (s.hi[d] - s.lo[d]) / 2 + 1;
    }
    s.off[s.N + 1] = total;
    *cells = total;
    free(band);
    s.F = malloc(sizeof(double) * 3 * total);
    s.B = malloc(sizeof(double) * 3 * total);
    s.bLive = calloc(s.N + 2, 1);
    for (int64_t i = 0; i < 3 * total; i++) {
        s.F[i] = NEG_INF;
        s.B[i] = NEG_INF;
    }
    setDiagonal(&s, s.F, 0, raggedLeft ? m->raggedStart : m->start);

    int64_t tracedBackTo = 0;
    for (int64_t d = 1; d <= s.N; d++) {
        forwardDiagonal(&s, d);
        int atEnd = d == s.N;
        int width = (int) ((s.hi[d] - s.lo[d]) / 2 + 1);
        int tracebackPoint = d >= tracedBackTo + p->minDiagsBetweenTraceBack && width <= p->diagonalExpansion * 2 + 1;
        if (!(atEnd || tracebackPoint)) {
            continue;
        }
        setDiagonal(&s, s.B, d, (atEnd && raggedRight) ? m->raggedEnd : m->end);
        s.bLive[d] = 1;
        if (d > tracedBackTo + 1) {
            resetDiagonal(&s, s.B, d - 1);
            s.bLive[d - 1] = 1;
        }
        int64_t tracedBackFrom = d - (atEnd ? 0 : p->traceBackDiagonals + 1);
        double totalLog = NEG_INF;
        int64_t posteriorsThisWalk = 0;
        for (int64_t d2 = d; d2 > tracedBackTo; d2--) {
            if (d2 > tracedBackTo + 2) {
                resetDiagonal(&s, s.B, d2 - 2);
                s.bLive[d2 - 2] = 1;
            }
            if (d2 > tracedBackTo + 1) {
                backwardDiagonal(&s, d2);
            }
            if (d2 <= tracedBackFrom) {
                if (posteriorsThisWalk++ % 10 == 0) {
                    totalLog = totalProbability(&s, d2);
                    if (atEnd && posteriorsThisWalk == 1) {
                        *logLik = totalLog;
                    }
                }
                posteriorDiagonal(&s, d2, totalLog, out, dense);
            }
            if (d2 + 1 <= s.N) {
                s.bLive[d2 + 1] = 0;
            }
        }
        for (int64_t k = tracedBackTo; k <= d; k++) {
            s.bLive[k] = 0;
        }
        tracedBackTo = tracedBackFrom;
    }
    free(s.lo);
    free(s.hi);
    free(s.off);
    free(s.F);
    free(s.B);
    free(s.bLive);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Forward likelihood and expected counts over a whole band            */
/* ------------------------------------------------------------------ */

/* Band + full forward matrix of one sub-problem; returns 0, -1 on an invalid band. */
static int fullForward(Sub *s, const MpoModel *m, MpoLogAddFn add, const uint16_t *sx, int64_t lx, const uint16_t *sy,
                       int64_t ly, const int64_t *anchors, int64_t nAnchors, int64_t expansion, int dynamic,
                       int raggedLeft) {
    memset(s, 0, sizeof(*s));
    s->m = m;
    s->add = add;
    s->sx = sx;
    s->sy = sy;
    s->lx = lx;
    s->ly = ly;
    s->N = lx + ly;
    int64_t *band = malloc(sizeof(int64_t) * 3 * (s->N + 1));
    if (mpo_band(anchors, nAnchors, lx, ly, expansion, dynamic, band) != 0) {
        free(band);
        return -1;
    }
    s->lo = malloc(sizeof(int64_t) * (s->N + 1));
    s->hi = malloc(sizeof(int64_t) * (s->N + 1));
    s->off = malloc(sizeof(int64_t) * (s->N + 2));
    int64_t total = 0;
    for (int64_t d = 0; d <= s->N; d++) {
        s->lo[d] = band[3 * d + 1];
        s->hi[d] = band[3 * d + 2];
        s->off[d] = total;
        total += (s->hi[d] - s->lo[d]) / 2 + 1;
    }
    s->off[s->N + 1] = total;
    free(band);
    s->F = malloc(sizeof(double) * 3 * total);
    s->B = malloc(sizeof(double) * 3 * total);
    s->bLive = calloc(s->N + 2, 1);
    for (int64_t i = 0; i < 3 * total; i++) {
        s->F[i] = NEG_INF;
        s->B[i] = NEG_INF;
    }
    setDiagonal(s, s->F, 0, raggedLeft ? m->raggedStart : m->start);
    for (int64_t d = 1; d <= s->N; d++) {
        forwardDiagonal(s, d);
    }
    return 0;
}

static void freeSub(Sub *s) {
    free(s->lo);
    free(s->hi);
    free(s->off);
    free(s->F);
    free(s->B);
    free(s->bLive);
}

double mpo_forward_probability(const MpoModel *model, const uint16_t *sx, int64_t lx, const uint16_t *sy,
                               int64_t ly, const int64_t *anchors, int64_t nAnchors, int64_t expansion, int dynamic,
                               int raggedLeft, int raggedRight, MpoLogAddFn logAdd) {
    if (logAdd == NULL) {
        logAdd = mpo_logadd_exact;
    }
    if (lx + ly == 0) {
        return 0.0;
    }
    Sub s;
    if (fullForward(&s, model, logAdd, sx, lx, sy, ly, anchors, nAnchors, expansion, dynamic, raggedLeft) != 0) {
        freeSub(&s);
        return NAN;
    }
    /* diagonalCalculationTotalProbability at the last diagonal: no diagonal follows it */
    setDiagonal(&s, s.B, s.N, raggedRight ? model->raggedEnd : model->end);
    s.bLive[s.N] = 1;
    double total = totalProbability(&s, s.N);
    freeSub(&s);
    return total;
}

/* Run-length table entry of a match emission (the index mpo_match_emission reads), -1 if none. */
static int64_t repeatEntry(const MpoModel *m, uint16_t cx, uint16_t cy) {
    if (!m->runLength || m->repeat10 == NULL) {
        return -1;
    }
    int64_t M = m->maxRepeat;
    int xb = symbolBase(m, cx);
    int b = xb == 4 ? 0 : xb;
    int row = m->strand ? b : 3 - b;
    return (row * M + (cx >> 8)) * M + (cy >> 8);
}

double mpo_expectations(const MpoModel *model, const uint16_t *sx, int64_t lx, const uint16_t *sy, int64_t ly,
                        const int64_t *anchors, int64_t nAnchors, int64_t expansion, int dynamic, int raggedLeft,
                        int raggedRight, double *out) {
    if (lx + ly == 0) {
        return 0.0;
    }
    Sub s;
    if (fullForward(&s, model, mpo_logadd_exact, sx, lx, sy, ly, anchors, nAnchors, expansion, dynamic,
                    raggedLeft) != 0) {
        freeSub(&s);
        return NAN;
    }
    for (int64_t d = 0; d <= s.N; d++) {
        s.bLive[d] = 1;
    }
    setDiagonal(&s, s.B, s.N, raggedRight ? model->raggedEnd : model->end);
    for (int64_t d = s.N; d >= 1; d--) {
        backwardDiagonal(&s, d);
    }
    const double P = totalProbability(&s, s.N);
    const double *t = model->trans;
    {  /* state posteriors at the first and the last cell */
        const double *f0 = cellOf(&s, s.F, 0, 0), *b0 = cellOf(&s, s.B, 0, 0);
        const double *fN = cellOf(&s, s.F, s.N, lx - ly), *bN = cellOf(&s, s.B, s.N, lx - ly);
        for (int k = 0; k < 3; k++) {
            if (f0 != NULL && b0 != NULL) out[44 + k] += exp(f0[k] + b0[k] - P);
            if (fN != NULL && bN != NULL) out[47 + k] += exp(fN[k] + bN[k] - P);
        }
    }
    for (int64_t d = 1; d <= s.N; d++) {
        for (int64_t xmy = s.lo[d]; xmy <= s.hi[d]; xmy += 2) {
            const int64_t x = (d + xmy) / 2, y = (d - xmy) / 2;
            const double *b = cellOf(&s, s.B, d, xmy), *f = cellOf(&s, s.F, d, xmy);
            const double *lower = cellOf(&s, s.F, d - 1, xmy - 1);
            const double *middle = d >= 2 ? cellOf(&s, s.F, d - 2, xmy) : NULL;
            const double *upper = cellOf(&s, s.F, d - 1, xmy + 1);
            const uint16_t cx = xSymbolAt(&s, d, xmy), cy = ySymbolAt(&s, d, xmy);
            /* transitions into this cell (cell_calculateExpectation, impl/pairwiseAligner.c:347-369) */
            for (int i = 0; i < 3; i++) {
                if (lower != NULL) {
                    out[i * 3 + 1] += exp(lower[i] + t[i * 3 + 1] + mpo_gap_x_emission(model, cx) + b[1] - P);
                }
                if (middle != NULL) {
                    out[i * 3 + 0] += exp(middle[i] + t[i * 3 + 0] + mpo_match_emission(model, cx, cy) + b[0] - P);
                }
                if (upper != NULL) {
                    out[i * 3 + 2] += exp(upper[i] + t[i * 3 + 2] + mpo_gap_y_emission(model, cy) + b[2] - P);
                }
            }
            /* state posteriors by emitted symbols */
            const int xb = symbolBase(model, cx), yb = symbolBase(model, cy);
            if (x > 0 && y > 0) {
                const double pm = exp(f[0] + b[0] - P);
                out[9 + xb * 5 + yb] += pm;
                const int64_t r = repeatEntry(model, cx, cy);
                if (r >= 0) {
                    out[50 + r] += pm;
                }
            }
            if (x > 0) {
                out[34 + xb] += exp(f[1] + b[1] - P);
            }
            if (y > 0) {
                out[39 + yb] += exp(f[2] + b[2] - P);
            }
        }
    }
    freeSub(&s);
    return P;
}

/* ------------------------------------------------------------------ */
/* Public job entry: splits + coordinate correction                    */
/* (getPosteriorProbsWithBandingSplittingAlignmentsByLargeGaps :942-991,*/
/*  pairCoordinateCorrectionFn :1077-1086)                              */
/* ------------------------------------------------------------------ */

MpoResult *mpo_align_with_indels(const MpoModel *model, const uint16_t *sx, int64_t lx, const uint16_t *sy,
                                 int64_t ly, const int64_t *anchors, int64_t nAnchors, const MpoParams *params,
                                 int raggedLeft, int raggedRight, MpoLogAddFn logAdd, int wantDense) {
    if (logAdd == NULL) {
        logAdd = mpo_logadd_exact;
    }
    int64_t nSplits = mpo_split_points(anchors, nAnchors, lx, ly, params->splitMatrixBiggerThanThis, raggedLeft,
                                       raggedRight, NULL, 0);
    int64_t *splits = malloc(sizeof(int64_t) * 4 * (nSplits > 0 ? nSplits : 1));
    mpo_split_points(anchors, nAnchors, lx, ly, params->splitMatrixBiggerThanThis, raggedLeft, raggedRight, splits,
                     nSplits);
    MpoResult *r = calloc(1, sizeof(MpoResult));
    TupleBuf final[3];
    memset(final, 0, sizeof(final));
    DenseBuf dense;
    memset(&dense, 0, sizeof(dense));
    /* wantDense 1: every band cell of every posterior diagonal; 2: only cells with a posterior
     * within 1e-3 of the threshold or above it (enough to check emitted tuples and completeness
     * on long reads) */
    dense.floor = wantDense == 2 ? params->threshold - 1e-3 : -HUGE_VAL;
    int64_t *subAnchors = malloc(sizeof(int64_t) * 3 * (nAnchors > 0 ? nAnchors : 1));
    int64_t j = 0;
    int failed = 0;
    for (int64_t i = 0; i < nSplits && !failed; i++) {
        int64_t x1 = splits[4 * i], y1 = splits[4 * i + 1], x2 = splits[4 * i + 2], y2 = splits[4 * i + 3];
        int64_t nSub = 0;
        while (j < nAnchors) {
            int64_t x = anchors[3 * j], y = anchors[3 * j + 1];
            if (x + y >= x2 + y2) {
                break;
            }
            subAnchors[3 * nSub] = x - x1;
            subAnchors[3 * nSub + 1] = y - y1;
            subAnchors[3 * nSub + 2] = anchors[3 * j + 2];
            nSub++;
            j++;
        }
        TupleBuf sub[3];
        memset(sub, 0, sizeof(sub));
        double ll = 0.0;
        int64_t cells = 0;
        int64_t denseStart = dense.n;
        if (runSubProblem(model, params, logAdd, sx + x1, x2 - x1, sy + y1, y2 - y1, subAnchors, nSub,
                          raggedLeft || i > 0, raggedRight || i < nSplits - 1, sub, wantDense ? &dense : NULL, &ll,
                          &cells) != 0) {
            failed = 1;
        }
        r->logLikelihood += ll;
        r->cells += cells;
        for (int k = 0; k < 3; k++) {
            for (int64_t q = sub[k].n - 1; q >= 0; q--) { /* pop-reverse into the output */
                tupleAppend(&final[k], sub[k].t[3 * q], sub[k].t[3 * q + 1] + x1, sub[k].t[3 * q + 2] + y1);
            }
            free(sub[k].t);
        }
        /* dense records of this split are in sub-problem coordinates: shift them */
        for (int64_t q = denseStart; q < dense.n; q++) {
            dense.v[5 * q] += (double) x1;
            dense.v[5 * q + 1] += (double) y1;
        }
    }
    free(subAnchors);
    free(splits);
    for (int k = 0; k < 3; k++) {
        r->n[k] = final[k].n;
        r->t[k] = final[k].t != NULL ? final[k].t : malloc(sizeof(int64_t));
    }
    r->nDense = dense.n;
    r->dense = dense.v;
    if (failed) {
        r->cells = -1;
    }
    return r;
}

void mpo_result_free(MpoResult *r) {
    if (r == NULL) {
        return;
    }
    for (int k = 0; k < 3; k++) {
        free(r->t[k]);
    }
    free(r->dense);
    free(r);
}

int64_t mpo_align_batch(const MpoModel *modelFwd, const MpoModel *modelRev, int64_t nJobs,
                        const int64_t *xOffsets, const uint16_t *xSymbols, const int64_t *yOffsets,
                        const uint16_t *ySymbols, const int64_t *anchorOffsets, const int64_t *anchors,
                        const uint8_t *strand, const MpoParams *params, int nThreads, int64_t *counts,
                        double *logLikelihoods) {
#ifdef _OPENMP
    if (nThreads > 0) {
        omp_set_num_threads(nThreads);
    }
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t j = 0; j < nJobs; j++) {
        MpoResult *r = mpo_align_with_indels(strand[j] ? modelFwd : modelRev, xSymbols + xOffsets[j],
                                             xOffsets[j + 1] - xOffsets[j], ySymbols + yOffsets[j],
                                             yOffsets[j + 1] - yOffsets[j], anchors + 3 * anchorOffsets[j],
                                             anchorOffsets[j + 1] - anchorOffsets[j], params, 0, 0, NULL, 0);
        for (int k = 0; k < 3; k++) {
            counts[3 * j + k] = r->n[k];
        }
        if (logLikelihoods != NULL) {
            logLikelihoods[j] = r->logLikelihood;
        }
        mpo_result_free(r);
    }
    return nJobs;
}
