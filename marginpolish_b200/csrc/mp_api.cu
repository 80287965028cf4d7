// C ABI of the realignment engine: model lowering, batch planning (splits,
// kernel variants, length-sorted queues), device memory and launches.
//
// Reference behaviour restated here (integer logic, bit-exact):
//  * split rectangles  -- getSplitPoints / getSplitPointsP (impl/pairwiseAligner.c:875-926)
//  * anchor re-basing  -- getPosteriorProbsWithBandingSplittingAlignmentsByLargeGaps (:942-991)
//  * band geometry     -- band_constructDynamic / band_construct (:96-226), mirrored by the band kernel
//  * crop range        -- getAlignedPairsWithIndelsCroppingReference (impl/polisher.c:613-628)
#include "../../include/mpgpu.h"
#include "mp_internal.h"
#include "mp_host.h"

#include <sched.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace mp {
int variantCount();
bool variantShape(int v, int *C, int *L, int *K);
bool variantIsF64(int v);
int variantMaxWarps(int v, int nTables);
cudaError_t launchVariant(int v, const DpArgs &a, int blocks, int warps, cudaStream_t s);
int adjointVariantCount();
bool adjointVariantShape(int v, int *C, int *L, int *K);
int adjointVariantMaxWarps(int v, int nTables);
cudaError_t launchAdjointVariant(int v, const DpArgs &a, int blocks, int warps, cudaStream_t s);
cudaError_t launchBand(const BandArgs &a, cudaStream_t s);
cudaError_t launchCompact(const CompactArgs &a, cudaStream_t s);
cudaError_t launchStatusCopy(const TaskOut *src, TaskOut *dst, int n, cudaStream_t s);
}  // namespace mp

using namespace mp;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

static thread_local std::string g_lastError;

static mp_status failf(mp_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return s;
}

#define CUDA_TRY(expr)                                                                              \
    do {                                                                                            \
        cudaError_t _e = (expr);                                                                    \
        if (_e != cudaSuccess) return failf(MP_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

#define MP_TRY(expr)                   \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

mp_status mp_fail(mp_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return s;
}

extern "C" const char *mp_last_error(void) {
    return g_lastError.c_str();
}

extern "C" const char *mp_version(void) {
    return "mpgpu 0.1 (sm_100a)";
}

extern "C" mp_status mp_engine_create(int device, mp_engine **out) {
    if (!out) return failf(MP_ERR_ARGUMENT, "mp_engine_create: out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        return failf(MP_ERR_CUDA, "no CUDA device available (%s)", e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
    }
    if (device < 0 || device >= n) return failf(MP_ERR_ARGUMENT, "device %d out of range (%d devices)", device, n);
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        return failf(MP_ERR_CUDA, "device %d is sm_%d%d; this library is built for sm_100a only", device, prop.major,
                     prop.minor);
    }
    mp_engine *eng = new mp_engine();
    eng->device = device;
    eng->scratchBudget = (size_t) ((double) prop.totalGlobalMem * 0.5);
    eng->smCount = prop.multiProcessorCount;
    eng->ccMajor = prop.major;
    eng->ccMinor = prop.minor;
    e = cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&eng->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&eng->ev1);
    if (e != cudaSuccess) {
        delete eng;
        return failf(MP_ERR_CUDA, "stream/event creation failed: %s", cudaGetErrorString(e));
    }
    *out = eng;
    return MP_OK;
}

extern "C" void mp_engine_destroy(mp_engine *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    mp_device_batch_destroy(e->oneShot);
    mp_device_batch_destroy(e->forwardShot);
    mp_device_batch_destroy(e->adjointShot);
    e->oneShot = e->forwardShot = e->adjointShot = nullptr;
    for (int k = 0; k < mp_engine::kPipeSlots; k++) {
        mp_device_batch_destroy(e->pipe[k]);  // destroys its own stream
        e->pipe[k] = nullptr;
    }
    if (e->outStream) cudaStreamDestroy(e->outStream);
    mp_node_scratch_free(e->nodeScratch);
    e->nodeScratch = nullptr;
    mp_indel_scratch_free(e->indelScratch);
    e->indelScratch = nullptr;
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

extern "C" mp_status mp_engine_release_buffers(mp_engine *e) {
    if (!e) return failf(MP_ERR_ARGUMENT, "engine is NULL");
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    CUDA_TRY(cudaSetDevice(e->device));
    mp_device_batch_destroy(e->oneShot);
    mp_device_batch_destroy(e->forwardShot);
    mp_device_batch_destroy(e->adjointShot);
    e->oneShot = e->forwardShot = e->adjointShot = nullptr;
    for (int k = 0; k < mp_engine::kPipeSlots; k++) {
        mp_device_batch_destroy(e->pipe[k]);
        e->pipe[k] = nullptr;
    }
    return MP_OK;
}

extern "C" mp_status mp_engine_info(const mp_engine *e, int *sm, int *ma, int *mi) {
    if (!e) return failf(MP_ERR_ARGUMENT, "engine is NULL");
    if (sm) *sm = e->smCount;
    if (ma) *ma = e->ccMajor;
    if (mi) *mi = e->ccMinor;
    return MP_OK;
}

extern "C" mp_status mp_engine_set_tuning(mp_engine *e, const mp_tuning *t) {
    if (!e || !t) return failf(MP_ERR_ARGUMENT, "engine or tuning is NULL");
    if (t->lanes_per_task != 0 && t->lanes_per_task != 32 && t->lanes_per_task != 16 && t->lanes_per_task != 8)
        return failf(MP_ERR_ARGUMENT, "lanes_per_task must be 0, 32, 16 or 8 (got %d)", t->lanes_per_task);
    if (t->warps_per_block < 0 || t->blocks_per_sm < 0)
        return failf(MP_ERR_ARGUMENT, "negative tuning value");
    e->tuning = *t;
    return MP_OK;
}

extern "C" mp_status mp_engine_set_graph_capture(mp_engine *e, int enable) {
    if (!e) return failf(MP_ERR_ARGUMENT, "engine is NULL");
    e->graphs = enable != 0;
    return MP_OK;
}

static float probOf(double logp) {
    return (float) std::exp(logp);
}

static mp_status lowerModel(const mp_model_desc *d, DevModel &m, float *rp) {
    if (!d) return failf(MP_ERR_ARGUMENT, "model description is NULL");
    for (int k = 0; k < 9; k++) {
        if (std::isnan(d->log_transitions[k]) || d->log_transitions[k] > 1e-9)
            return failf(MP_ERR_ARGUMENT, "log transition %d is not a log probability (%g)", k, d->log_transitions[k]);
        m.t[k] = probOf(d->log_transitions[k]);
    }
    for (int k = 0; k < 3; k++) {
        m.start[k] = probOf(d->log_start[k]);
        m.raggedStart[k] = probOf(d->log_ragged_start[k]);
        m.end[k] = probOf(d->log_end[k]);
        m.raggedEnd[k] = probOf(d->log_ragged_end[k]);
    }
    for (int k = 0; k < 25; k++) {
        if (std::isnan(d->log_match[k])) return failf(MP_ERR_ARGUMENT, "log match emission %d is NaN", k);
        m.match[k] = probOf(d->log_match[k]);
    }
    for (int k = 0; k < 5; k++) {
        m.gapX[k] = probOf(d->log_gap_x[k]);
        m.gapY[k] = probOf(d->log_gap_y[k]);
    }
    m.runLength = d->run_length ? 1 : 0;
    m.strand = d->strand ? 1 : 0;
    if (m.runLength) {
        if (d->max_repeat != kMaxRepeat)
            return failf(MP_ERR_ARGUMENT, "max_repeat must be %d (got %d)", kMaxRepeat, d->max_repeat);
        if (!d->repeat_log10) return failf(MP_ERR_ARGUMENT, "run-length model needs repeat_log10");
        for (int i = 0; i < kRepTable; i++) {
            double v = d->repeat_log10[i];
            if (std::isnan(v)) return failf(MP_ERR_ARGUMENT, "repeat table entry %d is NaN", i);
            rp[i] = (float) std::exp(d->repeat_scale * v);
        }
    } else {
        for (int i = 0; i < kRepTable; i++) rp[i] = 1.0f;
    }
    return MP_OK;
}

extern "C" mp_status mp_model_create(mp_engine *e, const mp_model_desc *fwd, const mp_model_desc *rev,
                                     mp_model **out) {
    if (!e || !out) return failf(MP_ERR_ARGUMENT, "engine or out is NULL");
    *out = nullptr;
    mp_model *m = new mp_model();
    m->engine = e;
    std::vector<float> rp(2 * kRepTable);
    mp_status s = lowerModel(fwd, m->host[0], rp.data());
    if (s == MP_OK) s = lowerModel(rev, m->host[1], rp.data() + kRepTable);
    if (s == MP_OK) {
        for (int k = 0; k < 9; k++) {
            m->logT[0][k] = fwd->log_transitions[k];
            m->logT[1][k] = rev->log_transitions[k];
        }
    }
    if (s == MP_OK) {
        m->sharedRepeat = memcmp(rp.data(), rp.data() + kRepTable, sizeof(float) * kRepTable) == 0 ? 1 : 0;
        m->noSwitch = (m->host[0].t[1 * 3 + 2] == 0.0f && m->host[0].t[2 * 3 + 1] == 0.0f &&
                       m->host[1].t[1 * 3 + 2] == 0.0f && m->host[1].t[2 * 3 + 1] == 0.0f) ? 1 : 0;
        std::vector<double> lrp(2 * kRepTable);
        mp_model_lower_log(fwd, m->logHost[0], lrp.data());
        mp_model_lower_log(rev, m->logHost[1], lrp.data() + kRepTable);
        cudaSetDevice(e->device);
        s = m->models.reserve(sizeof(DevModel) * 2);
        if (s == MP_OK) s = m->repeat.reserve(sizeof(float) * 2 * kRepTable);
        if (s == MP_OK) s = m->logModels.reserve(sizeof(mp::DevLogModel) * 2);
        if (s == MP_OK) s = m->logRepeat.reserve(sizeof(double) * 2 * kRepTable);
        if (s == MP_OK) {
            cudaError_t ce = cudaMemcpy(m->models.p, m->host, sizeof(DevModel) * 2, cudaMemcpyHostToDevice);
            if (ce == cudaSuccess) ce = cudaMemcpy(m->repeat.p, rp.data(), sizeof(float) * 2 * kRepTable, cudaMemcpyHostToDevice);
            if (ce == cudaSuccess)
                ce = cudaMemcpy(m->logModels.p, m->logHost, sizeof(mp::DevLogModel) * 2, cudaMemcpyHostToDevice);
            if (ce == cudaSuccess)
                ce = cudaMemcpy(m->logRepeat.p, lrp.data(), sizeof(double) * 2 * kRepTable, cudaMemcpyHostToDevice);
            if (ce != cudaSuccess) s = failf(MP_ERR_CUDA, "model upload failed: %s", cudaGetErrorString(ce));
        }
    }
    if (s != MP_OK) {
        delete m;
        return s;
    }
    *out = m;
    return MP_OK;
}

extern "C" void mp_model_destroy(mp_model *m) {
    if (!m) return;
    if (m->engine) cudaSetDevice(m->engine->device);
    delete m;
}

// ---------------------------------------------------------------------------
// geometry helpers (host)
// ---------------------------------------------------------------------------

static int64_t clampCoord(int64_t z, int64_t lz) {
    return z < 0 ? 0 : (z > lz ? lz : z);
}

static bool boxDiagonalHost(int64_t d, int64_t xL, int64_t yL, int64_t xU, int64_t yU, int64_t &lo, int64_t &hi) {
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
    lo = l;
    hi = h;
    return l <= h;
}

extern "C" mp_status mp_band(const int32_t *anchors, int64_t nA, int64_t lx, int64_t ly, int64_t expansion,
                             int dynamic, int64_t *out) {
    if (lx < 0 || ly < 0 || (!anchors && nA > 0) || !out) return failf(MP_ERR_ARGUMENT, "mp_band: bad arguments");
    int64_t xL = 0, yL = 0, xU = 0, yU = 0, e = dynamic ? 0 : expansion, nx = 0, ny = 0, k = 0;
    for (int64_t d = 0; d <= lx + ly; d++) {
        int64_t lo, hi;
        if (!boxDiagonalHost(d, xL, yL, xU, yU, lo, hi))
            return failf(MP_ERR_ARGUMENT, "invalid diagonal %lld (xmyL %lld > xmyR %lld)", (long long) d,
                         (long long) lo, (long long) hi);
        out[3 * d] = d;
        out[3 * d + 1] = lo;
        out[3 * d + 2] = hi;
        if (d == nx + ny) {
            int64_t px = nx, py = ny;
            if (k < nA) {
                nx = anchors[3 * k] + 1;
                ny = anchors[3 * k + 1] + 1;
                if (dynamic) e = anchors[3 * k + 2];
                k++;
            } else {
                nx = lx;
                ny = ly;
            }
            int64_t pxay = px + py, pxmy = px - py, nxay = nx + ny, nxmy = nx - ny;
            xL = clampCoord((pxay + (pxmy - e)) / 2, lx);
            yL = clampCoord((nxay - (nxmy - e)) / 2, ly);
            xU = clampCoord((nxay + (nxmy + e)) / 2, lx);
            yU = clampCoord((pxay - (pxmy + e)) / 2, ly);
        }
    }
    return MP_OK;
}

struct SplitRect {
    int64_t x1, y1, x2, y2;
};

static bool splitGap(int64_t &x1, int64_t &y1, int64_t x2, int64_t y2, int64_t x3, int64_t y3, int64_t maxSize,
                     bool skip, std::vector<SplitRect> &out) {
    int64_t gx = x3 - x2, gy = y3 - y2;
    if (gx * gy > maxSize) {
        int64_t side = (int64_t) std::sqrt((double) maxSize);
        int64_t hX = gx / 2 > side ? side : gx / 2;
        int64_t hY = gy / 2 > side ? side : gy / 2;
        if (!skip) out.push_back({x1, y1, x2 + hX, y2 + hY});
        x1 = x3 - hX;
        y1 = y3 - hY;
        return true;
    }
    return false;
}

static void splitPoints(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, int64_t maxSize, bool raggedL,
                        bool raggedR, std::vector<SplitRect> &out) {
    // every gap between anchors is a sub-rectangle of the matrix: none can exceed maxSize when
    // the whole matrix does not, and then the matrix is one rectangle
    if (lx * ly <= maxSize) {
        out.push_back({0, 0, lx, ly});
        return;
    }
    int64_t x1 = 0, y1 = 0, x2 = 0, y2 = 0;
    for (int64_t i = 0; i < nA; i++) {
        int64_t x3 = an[3 * i], y3 = an[3 * i + 1];
        splitGap(x1, y1, x2, y2, x3, y3, maxSize, raggedL && i == 0, out);
        x2 = x3 + 1;
        y2 = y3 + 1;
    }
    bool split = splitGap(x1, y1, x2, y2, lx, ly, maxSize, raggedL && nA == 0, out);
    if (!split || !raggedR) out.push_back({x1, y1, lx, ly});
}

extern "C" mp_status mp_split_points(const int32_t *anchors, int64_t nA, int64_t lx, int64_t ly, int64_t maxSize,
                                     int raggedL, int raggedR, int64_t *out, int64_t cap, int64_t *nOut) {
    if (lx < 0 || ly < 0 || (!anchors && nA > 0)) return failf(MP_ERR_ARGUMENT, "mp_split_points: bad arguments");
    std::vector<SplitRect> r;
    splitPoints(anchors, nA, lx, ly, maxSize, raggedL != 0, raggedR != 0, r);
    for (size_t i = 0; i < r.size() && (int64_t) i < cap; i++) {
        out[4 * i] = r[i].x1;
        out[4 * i + 1] = r[i].y1;
        out[4 * i + 2] = r[i].x2;
        out[4 * i + 3] = r[i].y2;
    }
    if (nOut) *nOut = (int64_t) r.size();
    return MP_OK;
}

extern "C" mp_status mp_crop_range(const int32_t *anchors, int64_t nA, int64_t tlen, int64_t rlen, int64_t *start,
                                   int64_t *end) {
    if (!start || !end) return failf(MP_ERR_ARGUMENT, "mp_crop_range: NULL output");
    int64_t s = 0, e = tlen;
    if (nA > 0) {
        s = (int64_t) anchors[0] - anchors[1];
        s = s < 0 ? 0 : s;
        e = 1 + (int64_t) anchors[3 * (nA - 1)] + (rlen - anchors[3 * (nA - 1) + 1]);
        e = e > tlen ? tlen : e;
    }
    if (s < 0 || s >= tlen || e < 0 || e > tlen)
        return failf(MP_ERR_ARGUMENT, "crop range [%lld, %lld) outside template of length %lld", (long long) s,
                     (long long) e, (long long) tlen);
    *start = s;
    *end = e;
    return MP_OK;
}

// ---------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------

// Kernel variants (C slots per lane, L lanes per task; see mp_posterior.cu). A task
// runs in the first variant of the engine's preference list whose window holds its
// band hull: S - 2C >= hull slots, S = L*C. Every list has ascending capacities.
static const int kPrefAuto[] = {0, 3, 4, 5, 6};  // measured fastest on the batched workload
static const int kPref32[] = {0, 3, 4, 5, 6};
static const int kPref16[] = {1, 0, 3, 4, 5, 6};
static const int kPref8[] = {2, 1, 0, 3, 4, 5, 6};
static const int kMaxHullSlots = 8 * 32 - 2 * 8;  // widest variant

static int variantCapacity(int v) {
    int C = 0, L = 0, K = 0;
    if (!variantShape(v, &C, &L, &K)) return 0;
    return L * C - 2 * C;
}

// Variant for a task needing `slots` window slots under lane preference `lanes`
// (32, 16, 8 or 0 = automatic); -1 when none is wide enough.
static int pickVariant(int lanes, int64_t slots) {
    const int *list = kPrefAuto;
    int n = (int) (sizeof(kPrefAuto) / sizeof(int));
    if (lanes == 32) {
        list = kPref32;
        n = (int) (sizeof(kPref32) / sizeof(int));
    } else if (lanes == 16) {
        list = kPref16;
        n = (int) (sizeof(kPref16) / sizeof(int));
    } else if (lanes == 8) {
        list = kPref8;
        n = (int) (sizeof(kPref8) / sizeof(int));
    }
    for (int i = 0; i < n; i++)
        if (slots <= variantCapacity(list[i])) return list[i];
    return -1;
}

// The engine's choice for a posterior task: the autotuned variant of the task's hull class
// when the engine is tuned and lanes_per_task is automatic, else the built-in preference.
static int pickTunedVariant(const mp_engine *e, int64_t slots) {
    if (e->tuning.lanes_per_task == 0) {
        for (size_t c = 0; c < e->tunedBound.size(); c++) {
            if (slots <= e->tunedBound[c]) {
                const int v = e->tunedVariant[c];
                if (v >= 0 && slots <= variantCapacity(v)) return v;
                break;
            }
        }
    }
    return pickVariant(e->tuning.lanes_per_task, slots);
}

// FP64 variants (one task per warp), narrowest window that holds the hull; -1 if none.
static int pickVariantF64(int64_t slots) {
    for (int v = 0; v < variantCount(); v++) {
        if (!variantIsF64(v)) continue;
        if (slots <= variantCapacity(v)) return v;
    }
    return -1;
}

// Bytes of one checkpoint slot of a variant (float4 or double4).
static size_t chkElemBytes(int v) {
    return variantIsF64(v) ? 32 : 16;
}

// Adjoint variants (one task per warp), narrowest window that holds the hull; -1 if none.
static int pickAdjointVariant(int64_t slots) {
    for (int v = 0; v < adjointVariantCount(); v++) {
        int C = 0, L = 0, K = 0;
        adjointVariantShape(v, &C, &L, &K);
        if (slots <= L * C - 2 * C) return v;
    }
    return -1;
}

static int adjointMaxHull() {
    int C = 0, L = 0, K = 0;
    adjointVariantShape(adjointVariantCount() - 1, &C, &L, &K);
    return L * C - 2 * C;
}

// Upper bound (in window slots) of the hull of 5 consecutive anti-diagonal bands:
// the union of up to three consecutive anchor boxes, clipped to the matrix.
static int64_t hullSlotBound(const int32_t *an, int64_t nA, int64_t x1, int64_t y1, int64_t lx, int64_t ly,
                             bool dynamic, int64_t fixedExp) {
    int64_t best = 1;
    int64_t lo1 = 0, hi1 = 0, lo2 = 0, hi2 = 0;  // previous two boxes (diagonal 0 seeds them)
    for (int64_t k = 0; k <= nA; k++) {
        int64_t px = 0, py = 0, nx, ny, e;
        if (k > 0) {
            px = an[3 * (k - 1)] - x1 + 1;
            py = an[3 * (k - 1) + 1] - y1 + 1;
        }
        if (k < nA) {
            nx = an[3 * k] - x1 + 1;
            ny = an[3 * k + 1] - y1 + 1;
            e = dynamic ? an[3 * k + 2] : fixedExp;
        } else {
            nx = lx;
            ny = ly;
            e = dynamic ? (nA > 0 ? an[3 * (nA - 1) + 2] : 0) : fixedExp;
        }
        int64_t lo = std::max(px - ny - e, -ly), hi = std::min(nx - py + e, lx);
        int64_t L = std::min(lo, std::min(lo1, lo2)), H = std::max(hi, std::max(hi1, hi2));
        int64_t span = ((H >> 1) - (L >> 1)) + 1;
        best = std::max(best, span);
        lo2 = lo1;
        hi2 = hi1;
        lo1 = lo;
        hi1 = hi;
    }
    return best;
}

// One pass over a job's anchors for the common case of a single rectangle: validation
// (strictly increasing, in range, even non-negative expansions when dynamic) and the hull bound
// of hullSlotBound(an, nA, 0, 0, lx, ly, ...), without branches in the loop. Returns -1 when an
// anchor is invalid (the caller then reports it through validateJob).
static int64_t scanSingleRect(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, bool dynamic, int64_t fixedExp) {
    int64_t lo1 = 0, hi1 = 0, lo2 = 0, hi2 = 0, best = 1;
    int64_t px = 0, py = 0;  // previous anchor + 1 (0 before the first)
    int64_t prevX = -1, prevY = -1;
    unsigned bad = 0;
    for (int64_t k = 0; k < nA; k++) {
        const int64_t x = an[3 * k], y = an[3 * k + 1], ex = an[3 * k + 2];
        bad |= (unsigned) (x <= prevX) | (unsigned) (y <= prevY) | (unsigned) (x >= lx) | (unsigned) (y >= ly);
        if (dynamic) bad |= (unsigned) (ex < 0) | (unsigned) (ex & 1);
        const int64_t e = dynamic ? ex : fixedExp;
        const int64_t nx = x + 1, ny = y + 1;
        const int64_t lo = std::max(px - ny - e, -ly), hi = std::min(nx - py + e, lx);
        const int64_t L = std::min(lo, std::min(lo1, lo2)), H = std::max(hi, std::max(hi1, hi2));
        best = std::max(best, ((H >> 1) - (L >> 1)) + 1);
        lo2 = lo1, hi2 = hi1, lo1 = lo, hi1 = hi;
        px = nx, py = ny, prevX = x, prevY = y;
    }
    {  // the box from the last anchor to the end
        const int64_t e = dynamic ? (nA > 0 ? (int64_t) an[3 * (nA - 1) + 2] : 0) : fixedExp;
        const int64_t lo = std::max(px - ly - e, -ly), hi = std::min(lx - py + e, lx);
        const int64_t L = std::min(lo, std::min(lo1, lo2)), H = std::max(hi, std::max(hi1, hi2));
        best = std::max(best, ((H >> 1) - (L >> 1)) + 1);
    }
    return bad ? -1 : best;
}

namespace mp {
int64_t splitCount(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, int64_t maxSize, bool raggedL, bool raggedR) {
    std::vector<SplitRect> r;
    splitPoints(an, nA, lx, ly, maxSize, raggedL, raggedR, r);
    return (int64_t) r.size();
}

void splitRects(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, int64_t maxSize, bool raggedL, bool raggedR,
                std::vector<SplitRectH> &out) {
    std::vector<SplitRect> r;
    splitPoints(an, nA, lx, ly, maxSize, raggedL, raggedR, r);
    out.clear();
    for (const SplitRect &q : r) out.push_back(SplitRectH{q.x1, q.y1, q.x2, q.y2});
}

int64_t hullSlots(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, bool dynamic, int64_t fixedExp) {
    return hullSlotBound(an, nA, 0, 0, lx, ly, dynamic, fixedExp);
}

int64_t hullSlotsRect(const int32_t *an, int64_t nA, int64_t x1, int64_t y1, int64_t lx, int64_t ly, bool dynamic,
                      int64_t fixedExp) {
    return hullSlotBound(an, nA, x1, y1, lx, ly, dynamic, fixedExp);
}
}  // namespace mp

struct PlannedTask {
    Task t;
    int32_t hull;  // window slots the band hull needs
};

// What a batch computes: the posterior pass (tuples), the forward likelihood only
// (computeForwardProbability), or the adjoint (expected counts).
enum BatchMode { kModePosterior = 0, kModeForward = 1, kModeAdjoint = 2 };

struct mp_device_batch {
    int mode = kModePosterior;
    mp_engine *e = nullptr;
    int device = -1;
    const mp_model *m = nullptr;
    mp_params p{};
    int64_t nJobs = 0;
    std::vector<Task> tasks;
    std::vector<int32_t> hull;          // per task: window slots needed (raised by window retries)
    std::vector<uint8_t> f64;           // per task: computed in FP64 (likelihood-only mode, or range retry)
    std::vector<int> var;               // per task: kernel variant of the current run
    std::vector<int64_t> jobFirstTask;  // n_jobs+1
    int64_t totalDiags = 0;
    int64_t outCap[3] = {0, 0, 0};
    // device
    DevBuf xs, ys, anchors, dTasks, band, dOut, outT[3];  // outT: staged tuples per list
    DevBuf orders, queue, scratch, scratchScal;
    DevBuf expect, expectRep;  // adjoint accumulators (FP64)
    DevBuf fetchDst[3], fetchW[3], fetchX[3], fetchY[3];  // compaction staging (reused)
    PinBuf stageTasks, stageOrders, stageDst[3];           // page-locked staging of the small uploads
    PinBuf stageIn[3];     // small inputs (templates, reads, anchors) from pageable caller memory
    PinBuf stageFetch;     // small results on their way to pageable result arrays
    std::vector<int> varOrderOff;  // per variant offset into orders
    std::vector<int> varCount;
    std::vector<int64_t> varMaxN;
    std::vector<TaskOut> hostOut;
    int launchesPerRun = 0;
    int forceVariant = -1;  // autotuner: every posterior task in this variant ...
    int forceWarps = 0;     // ... at this many warps per block
    int forceBlocks = 0;    // ... in at most this many persistent blocks
    size_t scratchBudget = 0;  // checkpoint bytes this batch may hold (0: the engine's budget)
    bool ran = false;
    float bandMs = 0.0f, posteriorMs = 0.0f;
    cudaEvent_t evBand = nullptr;
    cudaStream_t stream = nullptr;          // the batch's stream (the engine's unless a pipelined call set one)
    bool ownStream = false;                 // `stream` was created for this batch
    // pipelined slots: tuple copies run on their own stream, so that the slot's next inputs and
    // kernels do not queue behind them; evCopied guards the staging lists until they are copied
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evCompacted = nullptr, evCopied = nullptr;
    cudaEvent_t evUploaded = nullptr;       // pipelined slots: this slice's input copies are done
    cudaEvent_t evSync = nullptr;           // blocking-sync event the host waits on (sleeps, no spin)
    cudaEvent_t evKernels = nullptr;        // pipelined slots: the run's kernels are done
    cudaEvent_t evStatus = nullptr;         // pipelined slots: the run's statuses are on the host
    cudaEvent_t evReady = nullptr;          // pipelined slots: the run's tuples are compacted
    cudaStream_t outStream = nullptr;       // pipelined slots: the engine's stream of tuple copies
    bool copyPending = false;
    TaskOut *pinOut = nullptr;              // page-locked, mapped copy of the task statuses
    TaskOut *pinOutDev = nullptr;           // its device address (written by a small kernel)
    size_t pinOutCap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graphExec = nullptr;  // the pass's launches (engine graph capture on)
    std::vector<unsigned char> graphKey;  // their arguments when captured
    int graphCaptures = 0;
    ~mp_device_batch() {
        if (graphExec) cudaGraphExecDestroy(graphExec);
        if (evBand) cudaEventDestroy(evBand);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (pinOut) cudaFreeHost(pinOut);
        if (ownStream && stream) cudaStreamDestroy(stream);
        if (copyStream) cudaStreamDestroy(copyStream);
        if (evCompacted) cudaEventDestroy(evCompacted);
        if (evCopied) cudaEventDestroy(evCopied);
        if (evUploaded) cudaEventDestroy(evUploaded);
        if (evSync) cudaEventDestroy(evSync);
        if (evKernels) cudaEventDestroy(evKernels);
        if (evStatus) cudaEventDestroy(evStatus);
        if (evReady) cudaEventDestroy(evReady);
    }
};

// Waits until everything queued on `st` has run. The host thread polls an event, yielding its
// core for the first polls and then sleeping 20 us between them, instead of spinning in the
// runtime: callers that drive the engine from as many threads as the host has cores (the
// drop-in's OpenMP callers, each with its own engine) leave the cores to the threads still
// planning and filling their calls, while a lone caller still sees its work end promptly.
static cudaError_t waitStream(mp_device_batch *db, cudaStream_t st) {
    if (!db->evSync) {
        const cudaError_t e = cudaEventCreateWithFlags(&db->evSync, cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaEventRecord(db->evSync, st);
    if (e != cudaSuccess) return e;
    for (int polls = 0; (e = cudaEventQuery(db->evSync)) == cudaErrorNotReady; polls++) {
        if (polls < 32) {
            sched_yield();
        } else {
            struct timespec ts = {0, 20000};
            nanosleep(&ts, nullptr);
        }
    }
    return e;
}

static mp_status validateJob(const mp_batch *b, int64_t j, const mp_params *p, bool dynamic) {
    int64_t lx = b->x_end[j] - b->x_begin[j];
    int64_t ly = b->y_offsets[j + 1] - b->y_offsets[j];
    if (b->x_begin[j] < 0 || b->x_end[j] > b->x_symbols_length || lx < 0)
        return failf(MP_ERR_ARGUMENT, "job %lld: template range [%lld, %lld) invalid", (long long) j,
                     (long long) b->x_begin[j], (long long) b->x_end[j]);
    if (ly < 0) return failf(MP_ERR_ARGUMENT, "job %lld: negative read length", (long long) j);
    if (lx + ly > (int64_t) 1 << 30) return failf(MP_ERR_ARGUMENT, "job %lld: sequences too long", (long long) j);
    int64_t a0 = b->anchor_offsets[j], a1 = b->anchor_offsets[j + 1];
    if (a1 < a0) return failf(MP_ERR_ARGUMENT, "job %lld: anchor offsets decrease", (long long) j);
    int64_t px = -1, py = -1;
    for (int64_t i = a0; i < a1; i++) {
        int64_t x = b->anchors[3 * i], y = b->anchors[3 * i + 1], ex = b->anchors[3 * i + 2];
        if (x <= px || y <= py || x >= lx || y >= ly)
            return failf(MP_ERR_ARGUMENT, "job %lld: anchor %lld (%lld, %lld) not strictly increasing / in range",
                         (long long) j, (long long) (i - a0), (long long) x, (long long) y);
        if (dynamic && (ex < 0 || (ex & 1)))
            return failf(MP_ERR_ARGUMENT, "job %lld: anchor %lld expansion %lld must be even and >= 0",
                         (long long) j, (long long) (i - a0), (long long) ex);
        px = x;
        py = y;
    }
    (void) p;
    return MP_OK;
}

namespace mp {
mp_status validateAnchors(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, bool dynamic, int64_t job) {
    int64_t px = -1, py = -1;
    for (int64_t i = 0; i < nA; i++) {
        int64_t x = an[3 * i], y = an[3 * i + 1], ex = an[3 * i + 2];
        if (x <= px || y <= py || x >= lx || y >= ly)
            return failf(MP_ERR_ARGUMENT, "job %lld: anchor %lld (%lld, %lld) not strictly increasing / in range",
                         (long long) job, (long long) i, (long long) x, (long long) y);
        if (dynamic && (ex < 0 || (ex & 1)))
            return failf(MP_ERR_ARGUMENT, "job %lld: anchor %lld expansion %lld must be even and >= 0",
                         (long long) job, (long long) i, (long long) ex);
        px = x;
        py = y;
    }
    return MP_OK;
}
}  // namespace mp

static mp_status validateParams(const mp_params *p) {
    if (!p) return failf(MP_ERR_ARGUMENT, "params is NULL");
    if (!(p->threshold >= 0.0 && p->threshold <= 1.0))
        return failf(MP_ERR_ARGUMENT, "threshold %g outside [0, 1]", p->threshold);
    if (p->threshold <= 0.0) return failf(MP_ERR_ARGUMENT, "threshold 0 (emit every cell) is not supported");
    if (p->traceback_diagonals < 1) return failf(MP_ERR_ARGUMENT, "traceback_diagonals must be >= 1");
    if (p->diagonal_expansion < 0 || (p->diagonal_expansion & 1))
        return failf(MP_ERR_ARGUMENT, "diagonal_expansion must be even and >= 0");
    if (p->min_diags_between_traceback < 2) return failf(MP_ERR_ARGUMENT, "min_diags_between_traceback must be >= 2");
    if (p->traceback_diagonals + 1 >= p->min_diags_between_traceback)
        return failf(MP_ERR_ARGUMENT, "traceback_diagonals + 1 must be < min_diags_between_traceback");
    return MP_OK;
}

namespace mp {
mp_status validateParamsStruct(const mp_params *p) {
    return validateParams(p);
}
}  // namespace mp

static mp_status planBatch(mp_device_batch *db, const mp_batch *b) {
    const int64_t nJobs = b->n_jobs;
    const mp_params *p = &db->p;
    unsigned nThreads = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    if (nJobs < 64) nThreads = 1;
    std::vector<std::vector<PlannedTask>> perThread(nThreads);
    std::vector<std::vector<int64_t>> perThreadJobCount(nThreads);
    std::vector<mp_status> statuses(nThreads, MP_OK);
    std::vector<std::string> errors(nThreads);
    int64_t chunk = (nJobs + nThreads - 1) / nThreads;
    // the forward likelihood uses band_construct (fixed expansion, no splits)
    const bool forward = db->mode == kModeForward;
    const bool dynamic = !forward && p->dynamic_anchor_expansion != 0;
    auto work = [&](unsigned t) {
        int64_t j0 = t * chunk, j1 = std::min(nJobs, j0 + chunk);
        std::vector<SplitRect> rects;
        for (int64_t j = j0; j < j1; j++) {
            int64_t lx = b->x_end[j] - b->x_begin[j];
            int64_t ly = b->y_offsets[j + 1] - b->y_offsets[j];
            const int32_t *an = b->anchors + 3 * b->anchor_offsets[j];
            int64_t nA = b->anchor_offsets[j + 1] - b->anchor_offsets[j];
            bool rL = b->ragged_left ? b->ragged_left[j] != 0 : false;
            bool rR = b->ragged_right ? b->ragged_right[j] != 0 : false;
            // one rectangle (no split possible): validation and hull bound in one pass; the
            // general path validates first and bounds each rectangle's hull separately
            const bool whole = forward || lx * ly <= p->split_matrix_bigger_than_this;
            const bool shapeOk = b->x_begin[j] >= 0 && b->x_end[j] <= b->x_symbols_length && lx >= 0 && ly >= 0 &&
                                 lx + ly <= ((int64_t) 1 << 30) && b->anchor_offsets[j + 1] >= b->anchor_offsets[j];
            int64_t wholeHull = -1;
            if (whole && shapeOk)
                wholeHull = scanSingleRect(an, nA, lx, ly, dynamic, p->diagonal_expansion);
            if (wholeHull < 0) {
                mp_status s = validateJob(b, j, p, dynamic);
                if (s != MP_OK) {
                    statuses[t] = s;
                    errors[t] = g_lastError;
                    return;
                }
            }
            rects.clear();
            if (whole) rects.push_back(SplitRect{0, 0, lx, ly});
            else splitPoints(an, nA, lx, ly, p->split_matrix_bigger_than_this, rL, rR, rects);
            int64_t ai = 0;
            int64_t count = 0;
            for (size_t i = 0; i < rects.size(); i++) {
                const SplitRect &r = rects[i];
                int64_t first = ai;
                if (rects.size() == 1) {
                    ai = nA;  // every anchor lies in the only rectangle
                } else {
                    while (ai < nA) {
                        int64_t x = an[3 * ai], y = an[3 * ai + 1];
                        if (x + y >= r.x2 + r.y2) break;
                        ai++;
                    }
                }
                PlannedTask pt;
                memset(&pt, 0, sizeof(pt));
                Task &tk = pt.t;
                tk.lx = (int32_t) (r.x2 - r.x1);
                tk.ly = (int32_t) (r.y2 - r.y1);
                tk.xOff = b->x_begin[j] + r.x1;
                tk.yOff = b->y_offsets[j] + r.y1;
                tk.anchorOff = b->anchor_offsets[j] + first;
                tk.nAnchors = (int32_t) (ai - first);
                tk.x1 = (int32_t) r.x1;
                tk.y1 = (int32_t) r.y1;
                tk.xShift = b->x_shift ? (int32_t) b->x_shift[j] : 0;
                bool tl = rL || i > 0, tr = rR || i + 1 < rects.size();
                tk.flags = (tl ? kFlagRaggedLeft : 0) | (tr ? kFlagRaggedRight : 0) |
                           ((b->strand && b->strand[j]) ? kFlagForward : 0) | (dynamic ? kFlagDynamic : 0) |
                           (forward ? kFlagForwardOnly : 0);
                tk.job = (int32_t) j;
                tk.expansion = (int32_t) p->diagonal_expansion;
                int64_t slots = wholeHull >= 0 ? wholeHull
                                               : hullSlotBound(an + 3 * first, tk.nAnchors, r.x1, r.y1, tk.lx, tk.ly,
                                                               dynamic, p->diagonal_expansion);
                pt.hull = (int32_t) std::min<int64_t>(slots, 1 << 30);
                const int64_t maxHull = db->mode == kModeAdjoint ? adjointMaxHull() : kMaxHullSlots;
                if (slots > maxHull) {
                    statuses[t] = failf(MP_ERR_OVERFLOW,
                                        "job %lld: band hull of %lld slots exceeds the widest kernel window (%lld)",
                                        (long long) j, (long long) slots, (long long) maxHull);
                    errors[t] = g_lastError;
                    return;
                }
                perThread[t].push_back(pt);
                count++;
            }
            perThreadJobCount[t].push_back(count);
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nThreads; t++) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
    for (unsigned t = 0; t < nThreads; t++) {
        if (statuses[t] != MP_OK) {
            g_lastError = errors[t];
            return statuses[t];
        }
    }
    // assemble in job order
    db->tasks.clear();
    db->hull.clear();
    db->jobFirstTask.assign(1, 0);
    for (unsigned t = 0; t < nThreads; t++) {
        for (auto &pt : perThread[t]) {
            db->tasks.push_back(pt.t);
            db->hull.push_back(pt.hull);
        }
        for (int64_t c : perThreadJobCount[t]) db->jobFirstTask.push_back(db->jobFirstTask.back() + c);
    }
    // band / output offsets
    int64_t bandOff = 0;
    int64_t outOff[3] = {0, 0, 0};
    for (auto &tk : db->tasks) {
        int64_t N = (int64_t) tk.lx + tk.ly;
        tk.bandOff = bandOff;
        bandOff += N + 1;
        // capacity: measured densities are ~0.7 match and ~0.4-0.55 gap tuples per anti-diagonal
        // at threshold 0.01, higher in repetitive sequence; overflowing tasks are re-run with their
        // exact counts (a synchronous round trip, so the margins are generous: staging is 16 B per
        // entry, ~4 GB for a 77 M-diagonal batch)
        int32_t capM = (int32_t) (N + N / 2 + 64), capX = (int32_t) (N + 64), capY = (int32_t) (N + 64);
        int32_t caps[3] = {capM, capX, capY};
        if (db->mode != kModePosterior) caps[0] = caps[1] = caps[2] = 0;  // no tuples
        for (int k = 0; k < 3; k++) {
            tk.cap[k] = caps[k];
            tk.outOff[k] = outOff[k];
            outOff[k] += caps[k];
        }
    }
    db->totalDiags = bandOff;
    // the likelihood-only mode has no second total to check its range against: FP64 throughout
    db->f64.assign(db->tasks.size(), db->mode == kModeForward ? 1 : 0);
    for (int k = 0; k < 3; k++) db->outCap[k] = outOff[k];
    return MP_OK;
}

static int modeVariantCapacity(const mp_device_batch *db, int v) {
    if (db->mode != kModeAdjoint) return variantCapacity(v);
    int C = 0, L = 0, K = 0;
    if (!adjointVariantShape(v, &C, &L, &K)) return 0;
    return L * C - 2 * C;
}

static int modeMaxHullSlots(const mp_device_batch *db) {
    return db->mode == kModeAdjoint ? adjointMaxHull() : kMaxHullSlots;
}

// Zeroes the adjoint's FP64 accumulators (2 models' small tables, then the repeat tables).
static mp_status zeroExpectations(mp_device_batch *db) {
    MP_TRY(db->expect.reserve(sizeof(double) * 2 * kExpPerModel));
    MP_TRY(db->expectRep.reserve(sizeof(double) * 2 * kRepTable));
    CUDA_TRY(cudaMemsetAsync(db->expect.p, 0, sizeof(double) * 2 * kExpPerModel, db->stream));
    CUDA_TRY(cudaMemsetAsync(db->expectRep.p, 0, sizeof(double) * 2 * kRepTable, db->stream));
    return MP_OK;
}

// Picks each task's kernel variant under the engine's tuning and builds the
// per-variant length-sorted queues for the tasks in `subset`.
static int modeVariantCount(const mp_device_batch *db) {
    return db->mode == kModeAdjoint ? adjointVariantCount() : variantCount();
}

static bool modeVariantShape(const mp_device_batch *db, int v, int *C, int *L, int *K) {
    return db->mode == kModeAdjoint ? adjointVariantShape(v, C, L, K) : variantShape(v, C, L, K);
}

static mp_status buildQueues(mp_device_batch *db, const std::vector<int32_t> &subset, std::vector<int32_t> &orderHost) {
    const int nV = modeVariantCount(db);
    db->varOrderOff.assign(nV + 1, 0);
    db->varCount.assign(nV, 0);
    db->varMaxN.assign(nV, 0);
    db->var.resize(db->tasks.size(), -1);
    std::vector<std::vector<int32_t>> per(nV);
    for (int32_t t : subset) {
        const int v = db->mode == kModeAdjoint ? pickAdjointVariant(db->hull[t])
                      : db->f64[t]           ? pickVariantF64(db->hull[t])
                      : db->forceVariant >= 0 ? db->forceVariant
                                              : pickTunedVariant(db->e, db->hull[t]);
        if (v < 0)
            return failf(MP_ERR_OVERFLOW, "job %d: band wider than the widest kernel window", db->tasks[t].job);
        db->var[t] = v;
        per[v].push_back(t);
        int64_t N = (int64_t) db->tasks[t].lx + db->tasks[t].ly;
        db->varMaxN[v] = std::max(db->varMaxN[v], N);
    }
    orderHost.clear();
    for (int v = 0; v < nV; v++) {
        auto &q = per[v];
        std::stable_sort(q.begin(), q.end(), [&](int32_t x, int32_t y) {
            return (db->tasks[x].lx + db->tasks[x].ly) > (db->tasks[y].lx + db->tasks[y].ly);
        });
        db->varOrderOff[v] = (int) orderHost.size();
        db->varCount[v] = (int) q.size();
        orderHost.insert(orderHost.end(), q.begin(), q.end());
    }
    db->varOrderOff[nV] = (int) orderHost.size();
    return MP_OK;
}

static mp_status upload(DevBuf &buf, const void *src, size_t bytes, cudaStream_t s) {
    MP_TRY(buf.reserve(bytes));
    if (bytes) CUDA_TRY(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, s));
    return MP_OK;
}

// Transfers at most this many bytes go through the batch's page-locked staging when the
// caller's memory is pageable: the host copy is cheap, and a pageable transfer would go
// through the driver's own staging, which many calling threads share and queue on.
constexpr size_t kStageMax = (size_t) 8 << 20;

// upload() of a host vector through a page-locked staging buffer: the copy is DMA in stream
// order and the host returns at once. The staging buffer is rewritten by the next staged
// upload of the same purpose, which the batch's call sequence issues only after a
// synchronisation of this stream.
static mp_status uploadStaged(DevBuf &buf, PinBuf &stage, const void *src, size_t bytes, cudaStream_t s) {
    MP_TRY(buf.reserve(bytes));
    if (!bytes) return MP_OK;
    MP_TRY(stage.reserve(bytes));
    memcpy(stage.p, src, bytes);
    CUDA_TRY(cudaMemcpyAsync(buf.p, stage.p, bytes, cudaMemcpyHostToDevice, s));
    return MP_OK;
}

// Pageable host memory (not page-locked, not registered with CUDA).
static bool pageable(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return at.type == cudaMemoryTypeUnregistered;
}

static mp_status uploadSmall(DevBuf &buf, PinBuf &stage, const void *src, size_t bytes, cudaStream_t s) {
    return bytes > 0 && bytes <= kStageMax && pageable(src) ? uploadStaged(buf, stage, src, bytes, s)
                                                            : upload(buf, src, bytes, s);
}

// Plans a batch into `db` and uploads it, reusing the device buffers db already holds
// (they only grow).
static mp_status batchReset(mp_engine *e, mp_device_batch *db, const mp_model *m, const mp_params *p,
                            const mp_batch *b, bool syncInputs = true) {
    MP_TRY(validateParams(p));
    if (b->n_jobs < 0) return failf(MP_ERR_ARGUMENT, "negative job count");
    if (b->n_jobs > 0 && (!b->x_begin || !b->x_end || !b->y_offsets || !b->anchor_offsets || !b->strand))
        return failf(MP_ERR_ARGUMENT, "batch arrays missing");
    CUDA_TRY(cudaSetDevice(e->device));
    db->e = e;
    db->device = e->device;
    if (!db->stream) db->stream = e->stream;
    if (!db->ev0) CUDA_TRY(cudaEventCreate(&db->ev0));
    if (!db->ev1) CUDA_TRY(cudaEventCreate(&db->ev1));
    db->m = m;
    db->p = *p;
    db->nJobs = b->n_jobs;
    db->ran = false;
    db->hostOut.clear();
    MP_TRY(planBatch(db, b));
    cudaStream_t st = db->stream;
    int64_t ny = b->n_jobs > 0 ? b->y_offsets[b->n_jobs] : 0;
    int64_t na = b->n_jobs > 0 ? b->anchor_offsets[b->n_jobs] : 0;
    MP_TRY(uploadSmall(db->xs, db->stageIn[0], b->x_symbols, sizeof(uint16_t) * b->x_symbols_length, st));
    MP_TRY(uploadSmall(db->ys, db->stageIn[1], b->y_symbols, sizeof(uint16_t) * ny, st));
    MP_TRY(uploadSmall(db->anchors, db->stageIn[2], b->anchors, sizeof(int32_t) * 3 * na, st));
    MP_TRY(uploadStaged(db->dTasks, db->stageTasks, db->tasks.data(), sizeof(Task) * db->tasks.size(), st));
    MP_TRY(db->band.reserve(sizeof(int4) * std::max<int64_t>(db->totalDiags, 1)));
    MP_TRY(db->dOut.reserve(sizeof(TaskOut) * std::max<size_t>(db->tasks.size(), 1)));
    for (int k = 0; k < 3; k++) {
        MP_TRY(db->outT[k].reserve(sizeof(int4) * std::max<int64_t>(db->outCap[k], 1)));
    }
    MP_TRY(db->queue.reserve(sizeof(int32_t) * variantCount()));
    // the caller's host arrays may be reused as soon as this returns (unless the caller keeps
    // them valid until its own synchronisation)
    if (syncInputs) CUDA_TRY(waitStream(db, st));
    return MP_OK;
}

extern "C" mp_status mp_device_batch_create(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                            mp_device_batch **out) {
    if (!e || !m || !p || !b || !out) return failf(MP_ERR_ARGUMENT, "mp_device_batch_create: NULL argument");
    *out = nullptr;
    mp_device_batch *db = new mp_device_batch();
    mp_status s = batchReset(e, db, m, p, b);
    if (s != MP_OK) {
        delete db;
        return s;
    }
    *out = db;
    return MP_OK;
}

extern "C" mp_status mp_device_batch_reset(mp_engine *e, mp_device_batch *db, const mp_params *p, const mp_batch *b) {
    if (!e || !db || !p || !b) return failf(MP_ERR_ARGUMENT, "mp_device_batch_reset: NULL argument");
    return batchReset(e, db, db->m, p, b);
}

// The posterior launches of the current queues: one persistent launch per variant with
// tasks, with its grid, block and kernel arguments.
struct QueueLaunch {
    int v, blocks, warps;
    DpArgs a;
};

// Plans the posterior launches for the current queues. Scratch for all variants is reserved
// here, before any launch: every task slot (warp x tasks per warp) owns checkpoints for the
// longest task.
static mp_status planQueues(mp_device_batch *db, std::vector<QueueLaunch> &plan) {
    mp_engine *e = db->e;
    cudaStream_t st = db->stream;
    plan.clear();
    const int nV = modeVariantCount(db);
    const bool adj = db->mode == kModeAdjoint;
    std::vector<int> blocksOf(nV, 0), warpsOf(nV, 0), scratchBlocksOf(nV, 0);
    size_t needScratch = 0, needScal = 0;
    for (int v = 0; v < nV; v++) {
        if (db->varCount[v] == 0) continue;
        int C = 0, L = 0, K = 0;
        modeVariantShape(db, v, &C, &L, &K);
        const int G = 32 / L;
        const int nTables = db->m->sharedRepeat ? 1 : 2;
        const int maxW = adj ? adjointVariantMaxWarps(v, nTables) : variantMaxWarps(v, nTables);
        if (maxW < 1) return failf(MP_ERR_OVERFLOW, "kernel variant %d does not fit in shared memory", v);
        int warps = e->tuning.warps_per_block > 0 ? std::min(e->tuning.warps_per_block, maxW) : maxW;
        if (!adj && db->forceWarps > 0) warps = std::min(db->forceWarps, maxW);
        else if (!adj && e->tuning.warps_per_block == 0 && v < (int) e->tunedWarps.size() && e->tunedWarps[v] > 0)
            warps = std::min(e->tunedWarps[v], maxW);
        const int blocksPerSm = e->tuning.blocks_per_sm > 0 ? e->tuning.blocks_per_sm : 1;
        const int loads = (db->varCount[v] + G - 1) / G;  // warp-loads of G tasks
        const int maxBlocks = (loads + warps - 1) / warps;  // no more warps than loads
        int blocks = std::max(1, std::min(e->smCount * blocksPerSm, maxBlocks));
        if (!adj && db->forceBlocks > 0) blocks = std::min(blocks, db->forceBlocks);
        const int scratchBlocks = (int) (db->varMaxN[v] / K + 2);
        const size_t elem = adj ? sizeof(float4) : chkElemBytes(v);
        // every task slot holds checkpoints for the variant's longest task: within the budget,
        // fewer persistent blocks (long reads in wide windows need ~1 KB per anti-diagonal)
        {
            const size_t perSlot = (size_t) scratchBlocks * (size_t) (C * L) * elem + sizeof(int2) * scratchBlocks;
            const size_t budget = db->scratchBudget ? db->scratchBudget : e->scratchBudget;
            const size_t perBlock = perSlot * (size_t) warps * (size_t) G;
            if (budget > 0 && perBlock > 0) blocks = std::max(1, std::min(blocks, (int) std::min<size_t>(budget / perBlock, 1 << 20)));
        }
        const size_t slots = (size_t) blocks * warps * G;
        needScratch = std::max(needScratch, (size_t) scratchBlocks * (size_t) (C * L) * elem * slots);
        needScal = std::max(needScal, sizeof(int2) * (size_t) scratchBlocks * slots);
        blocksOf[v] = blocks;
        warpsOf[v] = warps;
        scratchBlocksOf[v] = scratchBlocks;
    }
    if (needScratch > db->scratch.bytes || needScal > db->scratchScal.bytes) {
        CUDA_TRY(cudaStreamSynchronize(st));
        MP_TRY(db->scratch.reserve(needScratch));
        MP_TRY(db->scratchScal.reserve(needScal));
    }
    for (int v = 0; v < nV; v++) {
        if (db->varCount[v] == 0) continue;
        DpArgs a;
        memset(&a, 0, sizeof(a));
        a.tasks = db->dTasks.as<Task>();
        a.order = db->orders.as<int32_t>() + db->varOrderOff[v];
        a.nTasks = db->varCount[v];
        a.scratchBlocks = scratchBlocksOf[v];
        a.queue = db->queue.as<int32_t>() + v;
        a.xs = db->xs.as<uint16_t>();
        a.ys = db->ys.as<uint16_t>();
        a.band = db->band.as<int2>();
        a.models = db->m->models.as<DevModel>();
        a.repeatProb = db->m->repeat.as<float>();
        a.scratch = db->scratch.as<float4>();
        a.scratchScalars = db->scratchScal.as<int2>();
        for (int k = 0; k < 3; k++) a.outT[k] = db->outT[k].as<int4>();
        a.out = db->dOut.as<TaskOut>();
        a.threshold = (float) db->p.threshold;
        a.minDiagsBetweenTraceBack = (int32_t) std::min<int64_t>(db->p.min_diags_between_traceback, 1 << 30);
        a.traceBackDiagonals = (int32_t) db->p.traceback_diagonals;
        a.diagonalExpansion = (int32_t) std::min<int64_t>(db->p.diagonal_expansion, 1 << 29);
        a.sharedRepeat = db->m->sharedRepeat;
        a.noSwitch = db->m->noSwitch;
        a.expect = db->expect.as<double>();
        a.expectRep = db->expectRep.as<double>();
        plan.push_back(QueueLaunch{v, blocksOf[v], warpsOf[v], a});
    }
    return MP_OK;
}

// Issues planned posterior launches (stream-ordered only: capturable into a CUDA graph).
static mp_status issueQueues(mp_device_batch *db, const std::vector<QueueLaunch> &plan) {
    cudaStream_t st = db->stream;
    const bool adj = db->mode == kModeAdjoint;
    CUDA_TRY(cudaMemsetAsync(db->queue.p, 0, sizeof(int32_t) * modeVariantCount(db), st));
    for (const QueueLaunch &q : plan) {
        if (adj) CUDA_TRY(launchAdjointVariant(q.v, q.a, q.blocks, q.warps, st));
        else CUDA_TRY(launchVariant(q.v, q.a, q.blocks, q.warps, st));
        db->launchesPerRun++;
    }
    return MP_OK;
}

static mp_status launchQueues(mp_device_batch *db) {
    std::vector<QueueLaunch> plan;
    MP_TRY(planQueues(db, plan));
    return issueQueues(db, plan);
}

// Appends the bytes of a trivially copyable value to a launch signature.
template <class T>
static void keyAppend(std::vector<unsigned char> &key, const T &v) {
    const unsigned char *b = reinterpret_cast<const unsigned char *>(&v);
    key.insert(key.end(), b, b + sizeof(T));
}

// Issues a run's launches and the copy of its task statuses on the batch's stream, without
// waiting for them.
static mp_status runIssue(mp_engine *e, mp_device_batch *db) {
    CUDA_TRY(cudaSetDevice(e->device));
    cudaStream_t st = db->stream;
    const int nTasks = (int) db->tasks.size();
    db->launchesPerRun = 0;
    std::vector<int32_t> all(nTasks), orderHost;
    for (int i = 0; i < nTasks; i++) all[i] = i;
    MP_TRY(buildQueues(db, all, orderHost));
    MP_TRY(uploadStaged(db->orders, db->stageOrders, orderHost.data(), sizeof(int32_t) * std::max<size_t>(orderHost.size(), 1), st));
    if (!db->evBand) CUDA_TRY(cudaEventCreate(&db->evBand));
    BandArgs ba;
    memset(&ba, 0, sizeof(ba));
    ba.tasks = db->dTasks.as<Task>();
    ba.nTasks = nTasks;
    ba.anchors = db->anchors.as<int32_t>();
    ba.band = db->band.as<int2>();
    ba.out = db->dOut.as<TaskOut>();
    if (db->mode == kModeAdjoint) {
        MP_TRY(db->expect.reserve(sizeof(double) * 2 * kExpPerModel));
        MP_TRY(db->expectRep.reserve(sizeof(double) * 2 * kRepTable));
    }
    std::vector<QueueLaunch> plan;
    MP_TRY(planQueues(db, plan));
    // the pass's launches: band kernels, then (adjoint: zeroed accumulators) the queues
    auto issuePass = [&](bool capturing) -> mp_status {
        CUDA_TRY(launchBand(ba, st));
        db->launchesPerRun += nTasks > 0 ? 2 : 0;
        // inside a capture, an event record becomes a graph node only when marked external
        if (capturing) CUDA_TRY(cudaEventRecordWithFlags(db->evBand, st, cudaEventRecordExternal));
        else CUDA_TRY(cudaEventRecord(db->evBand, st));
        if (db->mode == kModeAdjoint) MP_TRY(zeroExpectations(db));
        return issueQueues(db, plan);
    };
    if (e->graphs && !db->ownStream) {
        // One CUDA graph per batch (the pipelined slices of mp_realign_batch_into change every
        // call and run direct): replayed while the launches are identical (repeated runs),
        // re-captured and updated in place when they change.
        std::vector<unsigned char> key;
        keyAppend(key, db->mode);
        keyAppend(key, ba);
        for (const QueueLaunch &q : plan) {
            keyAppend(key, q.v);
            keyAppend(key, q.blocks);
            keyAppend(key, q.warps);
            keyAppend(key, q.a);
        }
        if (!db->graphExec || key != db->graphKey) {
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            const mp_status cs = issuePass(true);
            const cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (cs != MP_OK) {
                if (g) cudaGraphDestroy(g);
                return cs;
            }
            CUDA_TRY(ce);
            bool updated = false;
            if (db->graphExec) {
                cudaGraphExecUpdateResultInfo info;
                updated = cudaGraphExecUpdate(db->graphExec, g, &info) == cudaSuccess;
                if (!updated) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(db->graphExec);
                    db->graphExec = nullptr;
                }
            }
            if (!updated) {
                const cudaError_t ie = cudaGraphInstantiate(&db->graphExec, g, 0);
                cudaGraphDestroy(g);
                CUDA_TRY(ie);
            } else {
                cudaGraphDestroy(g);
            }
            db->graphKey = key;
            db->graphCaptures++;
        }
        db->launchesPerRun = (nTasks > 0 ? 2 : 0) + (int) plan.size();
        CUDA_TRY(cudaEventRecord(db->ev0, st));
        CUDA_TRY(cudaGraphLaunch(db->graphExec, st));
        CUDA_TRY(cudaEventRecord(db->ev1, st));
    } else {
        CUDA_TRY(cudaEventRecord(db->ev0, st));
        MP_TRY(issuePass(false));
        CUDA_TRY(cudaEventRecord(db->ev1, st));
    }
    // statuses, into page-locked memory so that the copy does not wait on the host
    // The statuses go to mapped page-locked memory through a small kernel: a copy would queue on
    // the copy engine behind earlier slices' tuple copies, and the host would learn late that
    // this run has ended.
    if ((size_t) nTasks > db->pinOutCap) {
        if (db->pinOut) cudaFreeHost(db->pinOut);
        db->pinOut = nullptr;
        db->pinOutDev = nullptr;
        db->pinOutCap = 0;
        CUDA_TRY(cudaHostAlloc(&db->pinOut, sizeof(TaskOut) * (size_t) nTasks, cudaHostAllocMapped | cudaHostAllocPortable));
        CUDA_TRY(cudaHostGetDevicePointer((void **) &db->pinOutDev, db->pinOut, 0));
        db->pinOutCap = (size_t) nTasks;
    }
    // pipelined slots: on the high-priority copy stream, so that the status copy is not queued
    // behind other slices' posterior kernels
    cudaStream_t ss = st;
    if (db->copyStream) {
        CUDA_TRY(cudaEventRecord(db->evKernels, st));
        CUDA_TRY(cudaStreamWaitEvent(db->copyStream, db->evKernels, 0));
        ss = db->copyStream;
    }
    if (nTasks) CUDA_TRY(launchStatusCopy(db->dOut.as<TaskOut>(), db->pinOutDev, nTasks, ss));
    if (db->copyStream) CUDA_TRY(cudaEventRecord(db->evStatus, ss));
    return MP_OK;
}

// Waits for an issued run, re-runs the tasks that need it (capacity, window, range, scratch)
// and marks the batch ran.
static mp_status runFinish(mp_engine *e, mp_device_batch *db, float *kernelMs) {
    cudaStream_t st = db->stream;
    const int nTasks = (int) db->tasks.size();
    std::vector<int32_t> orderHost;
    CUDA_TRY(waitStream(db, db->copyStream ? db->copyStream : st));  // the statuses are written there
    db->hostOut.assign(db->pinOut, db->pinOut + nTasks);
    float ms = 0.0f;
    CUDA_TRY(cudaEventElapsedTime(&ms, db->ev0, db->ev1));
    CUDA_TRY(cudaEventElapsedTime(&db->bandMs, db->ev0, db->evBand));
    CUDA_TRY(cudaEventElapsedTime(&db->posteriorMs, db->evBand, db->ev1));
    // retries: capacity overflows (exact counts known), window overflows (next wider variant), scratch
    for (int round = 0; round < 4; round++) {
        std::vector<int32_t> retry;
        bool changed = false;
        for (int t = 0; t < nTasks; t++) {
            TaskOut &o = db->hostOut[t];
            if (o.status & kTaskBand) {
                return failf(MP_ERR_ARGUMENT, "job %d: invalid band diagonal (anchors inconsistent with lengths)",
                             db->tasks[t].job);
            }
            if (o.status & kTaskSymbol) {
                return failf(MP_ERR_ARGUMENT, "job %d: a symbol's repeat count is >= %d", db->tasks[t].job,
                             kMaxRepeat);
            }
            if (o.status & kTaskRange) {
                // FP32 lost the range (wide band of weakly related sequences): again in FP64
                if (db->mode == kModeAdjoint || db->f64[t])
                    return failf(MP_ERR_OVERFLOW,
                                 "job %d: the band's probabilities exceed the range of the %s scaled "
                                 "arithmetic", db->tasks[t].job, db->f64[t] ? "FP64" : "FP32");
                db->f64[t] = 1;
                o.status &= ~kTaskRange;
                retry.push_back(t);
                changed = true;
                continue;
            }
            if (o.status & (kTaskCapacity | kTaskWindow | kTaskScratch)) {
                if (o.status & kTaskWindow) {
                    const int cap = modeVariantCapacity(db, db->var[t]);
                    if (cap >= modeMaxHullSlots(db))
                        return failf(MP_ERR_OVERFLOW, "job %d: band wider than the widest kernel window", db->tasks[t].job);
                    db->hull[t] = std::max(db->hull[t], cap + 1);
                }
                if (o.status & kTaskCapacity) {
                    for (int k = 0; k < 3; k++) {
                        if (o.count[k] > db->tasks[t].cap[k]) {
                            // new region at the end of the list buffer
                            db->tasks[t].cap[k] = o.count[k] + 16;
                            db->tasks[t].outOff[k] = db->outCap[k];
                            db->outCap[k] += db->tasks[t].cap[k];
                        }
                    }
                }
                retry.push_back(t);
                changed = true;
            }
        }
        if (!changed) break;
        if (db->mode == kModeAdjoint) {
            // the accumulators already hold the failed tasks' partial sums: run every task again
            retry.clear();
            for (int t = 0; t < nTasks; t++) retry.push_back(t);
            MP_TRY(zeroExpectations(db));
        }
        // grow output buffers (preserving contents)
        for (int k = 0; k < 3; k++) {
            size_t need = sizeof(int4) * db->outCap[k];
            if (need > db->outT[k].bytes) {
                DevBuf *bb = &db->outT[k];
                void *np = nullptr;
                CUDA_TRY(cudaMalloc(&np, need));
                CUDA_TRY(cudaMemcpyAsync(np, bb->p, bb->bytes, cudaMemcpyDeviceToDevice, st));
                CUDA_TRY(cudaStreamSynchronize(st));
                cudaFree(bb->p);
                bb->p = np;
                bb->bytes = need;
            }
        }
        MP_TRY(upload(db->dTasks, db->tasks.data(), sizeof(Task) * nTasks, st));
        // reset statuses of retried tasks (band flags stay valid)
        for (int32_t t : retry) db->hostOut[t].status = 0;
        CUDA_TRY(cudaMemcpyAsync(db->dOut.p, db->hostOut.data(), sizeof(TaskOut) * nTasks, cudaMemcpyHostToDevice, st));
        MP_TRY(buildQueues(db, retry, orderHost));
        MP_TRY(upload(db->orders, orderHost.data(), sizeof(int32_t) * std::max<size_t>(orderHost.size(), 1), st));
        CUDA_TRY(cudaEventRecord(db->ev0, st));
        MP_TRY(launchQueues(db));
        CUDA_TRY(cudaEventRecord(db->ev1, st));
        CUDA_TRY(cudaMemcpyAsync(db->hostOut.data(), db->dOut.p, sizeof(TaskOut) * nTasks, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        float ms2 = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms2, db->ev0, db->ev1));
        ms += ms2;
        db->posteriorMs += ms2;
    }
    for (int t = 0; t < nTasks; t++) {
        if (db->hostOut[t].status != 0)
            return failf(MP_ERR_OVERFLOW, "job %d: task status %d after retries", db->tasks[t].job, db->hostOut[t].status);
    }
    if (kernelMs) *kernelMs = ms;
    db->ran = true;
    return MP_OK;
}

extern "C" mp_status mp_device_batch_run(mp_engine *e, mp_device_batch *db, float *kernelMs) {
    if (!e || !db) return failf(MP_ERR_ARGUMENT, "mp_device_batch_run: NULL argument");
    MP_TRY(runIssue(e, db));
    return runFinish(e, db, kernelMs);
}

// The plain form of the same computation, for comparison: band kernels for the batch,
// then one posterior launch per task (one block of one warp, no persistent queue), in
// batch order, for the first max_tasks tasks. Returns the CUDA-event time of the
// posterior launches and the cells of the tasks run.
extern "C" mp_status mp_device_batch_run_plain(mp_engine *e, mp_device_batch *db, int64_t max_tasks, float *kernel_ms,
                                               int64_t *cells) {
    if (!e || !db) return failf(MP_ERR_ARGUMENT, "mp_device_batch_run_plain: NULL argument");
    CUDA_TRY(cudaSetDevice(e->device));
    cudaStream_t st = db->stream;
    const int nTasks = (int) db->tasks.size();
    const int n = (int) std::max<int64_t>(0, std::min<int64_t>(max_tasks, nTasks));
    std::vector<int32_t> all(nTasks), orderHost;
    for (int i = 0; i < nTasks; i++) all[i] = i;
    MP_TRY(buildQueues(db, all, orderHost));
    std::vector<int32_t> ident(std::max(nTasks, 1));
    for (int i = 0; i < nTasks; i++) ident[i] = i;
    MP_TRY(upload(db->orders, ident.data(), sizeof(int32_t) * ident.size(), st));
    BandArgs ba;
    ba.tasks = db->dTasks.as<Task>();
    ba.nTasks = nTasks;
    ba.anchors = db->anchors.as<int32_t>();
    ba.band = db->band.as<int2>();
    ba.out = db->dOut.as<TaskOut>();
    if (nTasks) CUDA_TRY(launchBand(ba, st));
    // scratch for one warp, sized for the longest task run
    size_t needScratch = 0, needScal = 0;
    int64_t maxN = 0;
    for (int t = 0; t < n; t++) maxN = std::max<int64_t>(maxN, (int64_t) db->tasks[t].lx + db->tasks[t].ly);
    for (int v = 0; v < variantCount(); v++) {
        int C = 0, L = 0, K = 0;
        variantShape(v, &C, &L, &K);
        needScratch = std::max(needScratch, (size_t) (maxN / K + 2) * (size_t) (C * L) * chkElemBytes(v) * (32 / L));
        needScal = std::max(needScal, sizeof(int2) * (size_t) (maxN / K + 2) * (32 / L));
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    MP_TRY(db->scratch.reserve(needScratch));
    MP_TRY(db->scratchScal.reserve(needScal));
    MP_TRY(db->queue.reserve(sizeof(int32_t) * std::max(n, 1)));
    CUDA_TRY(cudaMemsetAsync(db->queue.p, 0, sizeof(int32_t) * std::max(n, 1), st));
    CUDA_TRY(cudaEventRecord(db->ev0, st));
    for (int t = 0; t < n; t++) {
        int C = 0, L = 0, K = 0;
        const int v = db->var[t];
        variantShape(v, &C, &L, &K);
        DpArgs a;
        memset(&a, 0, sizeof(a));
        a.tasks = db->dTasks.as<Task>();
        a.order = db->orders.as<int32_t>() + t;
        a.nTasks = 1;
        a.scratchBlocks = (int32_t) (maxN / K + 2);
        a.queue = db->queue.as<int32_t>() + t;
        a.xs = db->xs.as<uint16_t>();
        a.ys = db->ys.as<uint16_t>();
        a.band = db->band.as<int2>();
        a.models = db->m->models.as<DevModel>();
        a.repeatProb = db->m->repeat.as<float>();
        a.scratch = db->scratch.as<float4>();
        a.scratchScalars = db->scratchScal.as<int2>();
        for (int k = 0; k < 3; k++) a.outT[k] = db->outT[k].as<int4>();
        a.out = db->dOut.as<TaskOut>();
        a.threshold = (float) db->p.threshold;
        a.minDiagsBetweenTraceBack = (int32_t) std::min<int64_t>(db->p.min_diags_between_traceback, 1 << 30);
        a.traceBackDiagonals = (int32_t) db->p.traceback_diagonals;
        a.diagonalExpansion = (int32_t) std::min<int64_t>(db->p.diagonal_expansion, 1 << 29);
        a.sharedRepeat = db->m->sharedRepeat;
        a.noSwitch = db->m->noSwitch;
        CUDA_TRY(launchVariant(v, a, 1, 1, st));
    }
    CUDA_TRY(cudaEventRecord(db->ev1, st));
    std::vector<TaskOut> host(std::max(nTasks, 1));
    if (nTasks) CUDA_TRY(cudaMemcpyAsync(host.data(), db->dOut.p, sizeof(TaskOut) * nTasks, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.0f;
    CUDA_TRY(cudaEventElapsedTime(&ms, db->ev0, db->ev1));
    int64_t c = 0;
    for (int t = 0; t < n; t++) {
        if (host[t].status != 0)
            return failf(MP_ERR_OVERFLOW, "job %d: task status %d in the plain run", db->tasks[t].job, host[t].status);
        c += host[t].cells;
    }
    db->ran = false;  // the batch's results now hold only the plain run's tasks
    if (kernel_ms) *kernel_ms = ms;
    if (cells) *cells = c;
    return MP_OK;
}

extern "C" mp_status mp_device_batch_timing(const mp_device_batch *db, float *bandMs, float *posteriorMs) {
    if (!db) return failf(MP_ERR_ARGUMENT, "batch is NULL");
    if (bandMs) *bandMs = db->bandMs;
    if (posteriorMs) *posteriorMs = db->posteriorMs;
    return MP_OK;
}

namespace mp {
cudaError_t launchFmaProbe(float *out, int blocks, int threads, int iters, cudaStream_t s);
cudaError_t launchDpProbe(double *out, int blocks, int threads, int iters, cudaStream_t s);
}

extern "C" mp_status mp_measure_fp32_peak(mp_engine *e, double *tflops) {
    if (!e || !tflops) return failf(MP_ERR_ARGUMENT, "mp_measure_fp32_peak: NULL argument");
    CUDA_TRY(cudaSetDevice(e->device));
    DevBuf out;
    const int threads = 512, blocksPerSm = 4, iters = 4096;
    const int blocks = e->smCount * blocksPerSm;
    MP_TRY(out.reserve(sizeof(float) * blocks * threads));
    cudaStream_t st = e->stream;
    for (int w = 0; w < 3; w++) CUDA_TRY(launchFmaProbe(out.as<float>(), blocks, threads, iters, st));
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        CUDA_TRY(cudaEventRecord(e->ev0, st));
        CUDA_TRY(launchFmaProbe(out.as<float>(), blocks, threads, iters, st));
        CUDA_TRY(cudaEventRecord(e->ev1, st));
        CUDA_TRY(cudaEventSynchronize(e->ev1));
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
        best = std::min(best, ms);
    }
    // 16 independent FMA chains per thread, `iters` rounds each
    double flops = 2.0 * 16.0 * iters * (double) blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return MP_OK;
}

extern "C" mp_status mp_measure_fp64_peak(mp_engine *e, double *gops) {
    if (!e || !gops) return failf(MP_ERR_ARGUMENT, "mp_measure_fp64_peak: NULL argument");
    CUDA_TRY(cudaSetDevice(e->device));
    DevBuf out;
    const int threads = 256, blocksPerSm = 4, iters = 1024;
    const int blocks = e->smCount * blocksPerSm;
    MP_TRY(out.reserve(sizeof(double) * blocks * threads));
    cudaStream_t st = e->stream;
    for (int w = 0; w < 3; w++) CUDA_TRY(launchDpProbe(out.as<double>(), blocks, threads, iters, st));
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        CUDA_TRY(cudaEventRecord(e->ev0, st));
        CUDA_TRY(launchDpProbe(out.as<double>(), blocks, threads, iters, st));
        CUDA_TRY(cudaEventRecord(e->ev1, st));
        CUDA_TRY(cudaEventSynchronize(e->ev1));
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
        best = std::min(best, ms);
    }
    const double ops = 16.0 * iters * (double) blocks * threads;
    *gops = ops / (best * 1e-3) / 1e9;
    return MP_OK;
}

extern "C" mp_status mp_device_batch_stats(const mp_device_batch *db, int64_t *cells, int64_t *nTasks,
                                           int32_t *launches) {
    if (!db) return failf(MP_ERR_ARGUMENT, "batch is NULL");
    int64_t c = 0;
    for (auto &o : db->hostOut) c += o.cells;
    if (cells) *cells = c;
    if (nTasks) *nTasks = (int64_t) db->tasks.size();
    if (launches) *launches = db->launchesPerRun;
    return MP_OK;
}

// ---------------------------------------------------------------------------
// results
// ---------------------------------------------------------------------------

struct mp_result {
    int64_t nJobs = 0;
    std::vector<int64_t> off[3];
    int64_t n[3] = {0, 0, 0};
    std::unique_ptr<int32_t[]> w[3], x[3], y[3];
    std::vector<double> logLik;
    std::vector<int64_t> cells;
    int64_t totalCells = 0;
    double deviceMs = 0.0;
};

// Per-job offsets of the compacted tuple lists and the per-task destinations.
static void fetchLayout(const mp_device_batch *db, int64_t total[3], std::vector<int64_t> dst[3],
                        int64_t *const off[3], double *logLik, int64_t *cells) {
    const int nTasks = (int) db->tasks.size();
    for (int k = 0; k < 3; k++) {
        total[k] = 0;
        dst[k].resize(std::max(nTasks, 1));
        if (off[k]) off[k][0] = 0;
    }
    for (int64_t j = 0; j < db->nJobs; j++) {
        double ll = 0.0;
        int64_t c = 0;
        for (int64_t t = db->jobFirstTask[j]; t < db->jobFirstTask[j + 1]; t++) {
            const TaskOut &o = db->hostOut[t];
            for (int k = 0; k < 3; k++) {
                dst[k][t] = total[k];
                total[k] += o.count[k];
            }
            ll += o.logLik;
            c += o.cells;
        }
        for (int k = 0; k < 3; k++)
            if (off[k]) off[k][j + 1] = total[k];
        if (logLik) logLik[j] = ll;
        if (cells) cells[j] = c;
    }
}

// Compacts every task's tuples into the batch's staging lists and queues their copies into
// the caller's host arrays (page-locked ones are copied by DMA at full link speed), without
// waiting for them. The batch's jobs are jobs j0.. of the caller's arrays and its tuples of
// list k start at tuple base[k]; a list whose tuples would pass cap[k] (cap may be NULL: no
// limit) is not copied. total[k] receives the batch's tuple counts.
static mp_status fetchIssue(mp_engine *e, mp_device_batch *db, const mp_output *out, int64_t j0,
                            const int64_t base[3], const int64_t *cap, int64_t total[3]) {
    if (!db->ran) return failf(MP_ERR_STATE, "fetch before a successful run");
    CUDA_TRY(cudaSetDevice(e->device));
    cudaStream_t st = db->stream;
    const int nTasks = (int) db->tasks.size();
    std::vector<int64_t> dst[3], off[3];
    int64_t *offp[3];
    for (int k = 0; k < 3; k++) {
        off[k].assign(db->nJobs + 1, 0);
        offp[k] = off[k].data();
    }
    fetchLayout(db, total, dst, offp, out->log_likelihood ? out->log_likelihood + j0 : nullptr,
                out->cells ? out->cells + j0 : nullptr);
    bool copy[3];
    for (int k = 0; k < 3; k++) {
        if (out->offsets[k])
            for (int64_t j = 0; j <= db->nJobs; j++) out->offsets[k][j0 + j] = base[k] + off[k][j];
        copy[k] = total[k] > 0 && (!cap || base[k] + total[k] <= cap[k]);
        if (copy[k] && (!out->weight[k] || !out->x[k] || !out->y[k]))
            return failf(MP_ERR_ARGUMENT, "output arrays of list %d missing", k);
        // the previous fetch's copies out of the staging lists must be done before they are reused
        if (k == 0 && db->copyPending) CUDA_TRY(cudaStreamWaitEvent(st, db->evCopied, 0));
        MP_TRY(uploadStaged(db->fetchDst[k], db->stageDst[k], dst[k].data(), sizeof(int64_t) * dst[k].size(), st));
        const size_t n = sizeof(int32_t) * std::max<int64_t>(total[k], 1);
        MP_TRY(db->fetchW[k].reserve(n));
        MP_TRY(db->fetchX[k].reserve(n));
        MP_TRY(db->fetchY[k].reserve(n));
    }
    // With a copy stream (pipelined slots), the compaction runs there too, at high priority, so
    // that it is not queued behind later slices' posterior kernels.
    cudaStream_t cs = st;
    if (db->copyStream) {
        CUDA_TRY(cudaEventRecord(db->evCompacted, st));
        CUDA_TRY(cudaStreamWaitEvent(db->copyStream, db->evCompacted, 0));
        cs = db->copyStream;
    }
    if (nTasks > 0) {
        CompactArgs ca;
        ca.tasks = db->dTasks.as<Task>();
        ca.out = db->dOut.as<TaskOut>();
        ca.nTasks = nTasks;
        for (int k = 0; k < 3; k++) {
            ca.dst[k] = db->fetchDst[k].as<int64_t>();
            ca.src[k] = db->outT[k].as<int4>();
            ca.w[k] = db->fetchW[k].as<int32_t>();
            ca.x[k] = db->fetchX[k].as<int32_t>();
            ca.y[k] = db->fetchY[k].as<int32_t>();
        }
        CUDA_TRY(launchCompact(ca, cs));
    }
    // the pipelined slots' tuple copies all go to the engine's one copy stream, so that the
    // slices' tuples leave in slice order at the link's full speed
    if (db->outStream) {
        CUDA_TRY(cudaEventRecord(db->evReady, cs));
        CUDA_TRY(cudaStreamWaitEvent(db->outStream, db->evReady, 0));
        cs = db->outStream;
    }
    for (int k = 0; k < 3; k++) {
        if (!copy[k]) continue;
        const size_t n = sizeof(int32_t) * total[k];
        CUDA_TRY(cudaMemcpyAsync(out->weight[k] + base[k], db->fetchW[k].p, n, cudaMemcpyDeviceToHost, cs));
        CUDA_TRY(cudaMemcpyAsync(out->x[k] + base[k], db->fetchX[k].p, n, cudaMemcpyDeviceToHost, cs));
        CUDA_TRY(cudaMemcpyAsync(out->y[k] + base[k], db->fetchY[k].p, n, cudaMemcpyDeviceToHost, cs));
    }
    if (db->copyStream) {
        CUDA_TRY(cudaEventRecord(db->evCopied, cs));
        db->copyPending = true;
    }
    return MP_OK;
}

static mp_status fetchInto(mp_engine *e, mp_device_batch *db, const mp_output *out) {
    const int64_t base[3] = {0, 0, 0};
    int64_t total[3];
    MP_TRY(fetchIssue(e, db, out, 0, base, nullptr, total));
    CUDA_TRY(waitStream(db, db->copyStream ? db->copyStream : db->stream));
    return MP_OK;
}

extern "C" mp_status mp_device_batch_counts(const mp_device_batch *db, int64_t totals[3]) {
    if (!db || !totals) return failf(MP_ERR_ARGUMENT, "mp_device_batch_counts: NULL argument");
    if (!db->ran) return failf(MP_ERR_STATE, "counts before a successful run");
    totals[0] = totals[1] = totals[2] = 0;
    for (const TaskOut &o : db->hostOut)
        for (int k = 0; k < 3; k++) totals[k] += o.count[k];
    return MP_OK;
}

extern "C" mp_status mp_device_batch_fetch_into(mp_engine *e, mp_device_batch *db, const mp_output *out) {
    if (!e || !db || !out) return failf(MP_ERR_ARGUMENT, "mp_device_batch_fetch_into: NULL argument");
    return fetchInto(e, db, out);
}

extern "C" mp_status mp_device_batch_fetch(mp_engine *e, mp_device_batch *db, mp_result **out) {
    if (!e || !db || !out) return failf(MP_ERR_ARGUMENT, "mp_device_batch_fetch: NULL argument");
    *out = nullptr;
    int64_t totals[3];
    MP_TRY(mp_device_batch_counts(db, totals));
    mp_result *r = new mp_result();
    r->nJobs = db->nJobs;
    mp_output o;
    for (int k = 0; k < 3; k++) {
        r->off[k].assign(db->nJobs + 1, 0);
        r->n[k] = totals[k];
        r->w[k].reset(new int32_t[std::max<int64_t>(totals[k], 1)]);  // filled by the copy, not zeroed
        r->x[k].reset(new int32_t[std::max<int64_t>(totals[k], 1)]);
        r->y[k].reset(new int32_t[std::max<int64_t>(totals[k], 1)]);
        o.offsets[k] = r->off[k].data();
        o.weight[k] = r->w[k].get();
        o.x[k] = r->x[k].get();
        o.y[k] = r->y[k].get();
    }
    r->logLik.assign(db->nJobs, 0.0);
    r->cells.assign(db->nJobs, 0);
    o.log_likelihood = r->logLik.data();
    o.cells = r->cells.data();
    // small results come through page-locked staging (one block, lists back to back), then a
    // host copy into the result's arrays
    const size_t tupleBytes = sizeof(int32_t) * 3 * (size_t) (totals[0] + totals[1] + totals[2]);
    const bool staged = tupleBytes <= kStageMax;
    if (staged) {
        mp_status rs = db->stageFetch.reserve(std::max<size_t>(tupleBytes, 16));
        if (rs != MP_OK) {
            delete r;
            return rs;
        }
        int32_t *at = static_cast<int32_t *>(db->stageFetch.p);
        for (int k = 0; k < 3; k++) {
            o.weight[k] = at;
            o.x[k] = at + totals[k];
            o.y[k] = at + 2 * totals[k];
            at += 3 * totals[k];
        }
    }
    mp_status s = fetchInto(e, db, &o);
    if (s != MP_OK) {
        delete r;
        return s;
    }
    if (staged) {
        const int32_t *at = static_cast<const int32_t *>(db->stageFetch.p);
        for (int k = 0; k < 3; k++) {
            const size_t n = sizeof(int32_t) * (size_t) totals[k];
            memcpy(r->w[k].get(), at, n);
            memcpy(r->x[k].get(), at + totals[k], n);
            memcpy(r->y[k].get(), at + 2 * totals[k], n);
            at += 3 * totals[k];
        }
    }
    for (int64_t c : r->cells) r->totalCells += c;
    *out = r;
    return MP_OK;
}

extern "C" void mp_device_batch_destroy(mp_device_batch *db) {
    if (!db) return;
    if (db->device >= 0) cudaSetDevice(db->device);  // the engine may already be gone
    delete db;
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------

// Steady-state throughput (GCUPS of a whole device) of variant v at `warps` warps per block
// on the tasks `subset` (`cells` band cells) of a planned batch: the persistent grid is cut
// to the blocks that get at least six task loads per warp, so that the length-sorted queue
// drains without a tail of idle warps, and the per-block rate is scaled to every SM. Best
// of `reps` launches after one warm-up launch.
static mp_status timeCandidate(mp_device_batch *db, const std::vector<int32_t> &subset, int64_t cells, int v,
                               int warps, int reps, double *gcups) {
    mp_engine *e = db->e;
    cudaStream_t st = db->stream;
    int C = 0, L = 0, K = 0;
    variantShape(v, &C, &L, &K);
    const int loads = ((int) subset.size() + 32 / L - 1) / (32 / L);
    const int blocks = std::max(1, std::min(e->smCount, loads / (6 * warps)));
    db->forceVariant = v;
    db->forceWarps = warps;
    db->forceBlocks = blocks;
    std::vector<int32_t> orderHost;
    mp_status s = buildQueues(db, subset, orderHost);
    if (s == MP_OK)
        s = upload(db->orders, orderHost.data(), sizeof(int32_t) * std::max<size_t>(orderHost.size(), 1), st);
    float best = 0.0f;
    for (int r = 0; s == MP_OK && r <= reps; r++) {
        if (cudaEventRecord(db->ev0, st) != cudaSuccess) s = failf(MP_ERR_CUDA, "event record failed");
        if (s == MP_OK) s = launchQueues(db);
        if (s == MP_OK && cudaEventRecord(db->ev1, st) != cudaSuccess) s = failf(MP_ERR_CUDA, "event record failed");
        if (s == MP_OK && cudaStreamSynchronize(st) != cudaSuccess)
            s = failf(MP_ERR_CUDA, "autotune launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        float ms = 0.0f;
        if (s == MP_OK && cudaEventElapsedTime(&ms, db->ev0, db->ev1) != cudaSuccess)
            s = failf(MP_ERR_CUDA, "event timing failed");
        if (s == MP_OK && r > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    db->forceVariant = -1;
    db->forceWarps = 0;
    db->forceBlocks = 0;
    *gcups = best > 0.0f ? (double) cells / (best * 1e6) * e->smCount / blocks : 0.0;
    return s;
}

extern "C" mp_status mp_engine_autotune_reset(mp_engine *e) {
    if (!e) return failf(MP_ERR_ARGUMENT, "engine is NULL");
    e->tunedBound.clear();
    e->tunedVariant.clear();
    e->tunedWarps.clear();
    return MP_OK;
}

extern "C" mp_status mp_engine_autotune(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *sample,
                                        mp_autotune_report *report) {
    if (!e || !m || !p || !sample) return failf(MP_ERR_ARGUMENT, "mp_engine_autotune: NULL argument");
    CUDA_TRY(cudaSetDevice(e->device));
    // classes: the distinct window capacities of the FP32 variants, ascending
    std::vector<int> bounds;
    for (int v = 0; v < variantCount(); v++)
        if (!variantIsF64(v)) bounds.push_back(variantCapacity(v));
    std::sort(bounds.begin(), bounds.end());
    bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
    if ((int) bounds.size() > MP_AUTOTUNE_MAX_CLASSES) bounds.resize(MP_AUTOTUNE_MAX_CLASSES);
    if (report) {
        memset(report, 0, sizeof(*report));
        report->n_classes = (int32_t) bounds.size();
    }
    // plan and run the sample once with the built-in choice (bands, capacities, hull retries)
    const std::vector<int> keepBound = e->tunedBound, keepVariant = e->tunedVariant, keepWarps = e->tunedWarps;
    MP_TRY(mp_engine_autotune_reset(e));
    mp_device_batch *db = nullptr;
    mp_status s = mp_device_batch_create(e, m, p, sample, &db);
    float ms0 = 0.0f;
    if (s == MP_OK) s = mp_device_batch_run(e, db, &ms0);
    std::vector<int> chosenVariant(bounds.size(), -1);
    std::vector<int> warpsOf(variantCount(), 0);
    const int nTables = m->sharedRepeat ? 1 : 2;
    const int kMinTasks = 2 * e->smCount;  // enough sub-problems for a steady-state measurement
    for (size_t c = 0; s == MP_OK && c < bounds.size(); c++) {
        const int lo = c == 0 ? 0 : bounds[c - 1], hi = bounds[c];
        std::vector<int32_t> subset;
        int64_t cells = 0;
        for (size_t t = 0; t < db->tasks.size(); t++) {
            if (db->f64[t] || db->hull[t] <= lo || db->hull[t] > hi) continue;
            subset.push_back((int32_t) t);
            cells += db->hostOut[t].cells;
        }
        if (report) {
            report->max_hull[c] = hi;
            report->tasks[c] = (int32_t) subset.size();
            report->variant[c] = -1;
        }
        if ((int) subset.size() < kMinTasks || cells <= 0) continue;
        // the built-in choice, for the report
        const int def = pickVariant(0, hi);
        double defRate = 0.0;
        s = timeCandidate(db, subset, cells, def, variantMaxWarps(def, nTables), 2, &defRate);
        double bestRate = 0.0;
        int bestV = -1, bestW = 0, timed = 0;
        for (int v = 0; s == MP_OK && v < variantCount(); v++) {
            if (variantIsF64(v) || variantCapacity(v) < hi) continue;
            const int maxW = variantMaxWarps(v, nTables);
            if (maxW < 1) continue;
            int opts[3] = {maxW, std::max(1, (maxW * 3) / 4), std::max(1, maxW / 2)};
            for (int k = 0; s == MP_OK && k < 3; k++) {
                if (k > 0 && opts[k] == opts[k - 1]) continue;
                double rate = 0.0;
                s = timeCandidate(db, subset, cells, v, opts[k], 2, &rate);
                timed++;
                if (s == MP_OK && rate > bestRate) {
                    bestRate = rate;
                    bestV = v;
                    bestW = opts[k];
                }
            }
        }
        if (s != MP_OK || bestV < 0) break;
        chosenVariant[c] = bestV;
        // one warps setting per variant: the first class that chose it decides
        if (warpsOf[bestV] == 0) warpsOf[bestV] = bestW;
        if (report) {
            int C = 0, L = 0, K = 0;
            variantShape(bestV, &C, &L, &K);
            report->candidates[c] = timed;
            report->variant[c] = bestV;
            report->lanes_per_task[c] = L;
            report->cells_per_lane[c] = C;
            report->checkpoint_stride[c] = K;
            report->warps_per_block[c] = warpsOf[bestV];
            report->gcups[c] = bestRate;
            report->default_gcups[c] = defRate;
        }
    }
    mp_device_batch_destroy(db);
    if (s != MP_OK) {
        e->tunedBound = keepBound;
        e->tunedVariant = keepVariant;
        e->tunedWarps = keepWarps;
        return s;
    }
    e->tunedBound = bounds;
    e->tunedVariant = chosenVariant;
    e->tunedWarps = warpsOf;
    return MP_OK;
}

extern "C" mp_status mp_result_view_get(const mp_result *r, mp_result_view *v) {
    if (!r || !v) return failf(MP_ERR_ARGUMENT, "mp_result_view_get: NULL argument");
    v->n_jobs = r->nJobs;
    for (int k = 0; k < 3; k++) {
        v->offsets[k] = r->off[k].data();
        v->weight[k] = r->w[k].get();
        v->x[k] = r->x[k].get();
        v->y[k] = r->y[k].get();
    }
    v->log_likelihood = r->logLik.data();
    v->cells = r->cells.data();
    v->total_cells = r->totalCells;
    v->device_ms = r->deviceMs;
    return MP_OK;
}

extern "C" void mp_result_destroy(mp_result *r) {
    delete r;
}

// One-shot calls reuse a batch cached in the engine, so repeated calls of similar size
// allocate no device memory after the first.
extern "C" mp_status mp_realign_batch(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                      mp_result **out) {
    if (!out) return failf(MP_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!e || !m || !p || !b) return failf(MP_ERR_ARGUMENT, "mp_realign_batch: NULL argument");
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    if (!e->oneShot) e->oneShot = new mp_device_batch();
    mp_device_batch *db = e->oneShot;
    // the input copies need no wait of their own: the call returns after its last wait
    MP_TRY(batchReset(e, db, m, p, b, false));
    float ms = 0.0f;
    MP_TRY(mp_device_batch_run(e, db, &ms));
    MP_TRY(mp_device_batch_fetch(e, db, out));
    (*out)->deviceMs = ms;
    return MP_OK;
}

// Slices [cut[i], cut[i+1]) of a batch's jobs by work (template + read symbols). With three or
// more slices the first and the last get half the work of the others: the first one's inputs
// are copied before any kernel runs and the last one's tuples after the last kernel, so small
// end slices shorten the pipeline's fill and drain.
static std::vector<int64_t> sliceJobs(const mp_batch *b, int parts) {
    const int64_t n = b->n_jobs;
    std::vector<double> target;  // cumulative work fraction at each inner cut
    const double units = parts >= 3 ? (double) parts - 1.0 : (double) parts;
    double acc = 0.0;
    for (int i = 0; i + 1 < parts; i++) {
        acc += (parts >= 3 && i == 0) ? 0.5 : 1.0;
        target.push_back(acc / units);
    }
    std::vector<int64_t> cut(1, 0);
    int64_t work = 0;
    for (int64_t j = 0; j < n; j++) work += (b->x_end[j] - b->x_begin[j]) + (b->y_offsets[j + 1] - b->y_offsets[j]);
    int64_t sum = 0;
    size_t next = 0;
    for (int64_t j = 0; j + 1 < n && next < target.size(); j++) {
        sum += (b->x_end[j] - b->x_begin[j]) + (b->y_offsets[j + 1] - b->y_offsets[j]);
        if ((double) sum >= target[next] * (double) work) {
            cut.push_back(j + 1);
            next++;
        }
    }
    cut.push_back(n);
    return cut;
}

extern "C" mp_status mp_realign_batch_into(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                           int32_t parts, const mp_output *out, const int64_t cap[3], int64_t need[3]) {
    if (!e || !m || !p || !b || !out || !cap) return failf(MP_ERR_ARGUMENT, "mp_realign_batch_into: NULL argument");
    if (b->n_jobs < 0) return failf(MP_ERR_ARGUMENT, "negative job count");
    if (b->n_jobs > 0 && (!b->x_begin || !b->x_end || !b->y_offsets || !b->anchor_offsets || !b->strand))
        return failf(MP_ERR_ARGUMENT, "batch arrays missing");
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    CUDA_TRY(cudaSetDevice(e->device));
    const int64_t n = b->n_jobs;
    if (parts <= 0) parts = n >= 2048 ? mp_engine::kPipeSlots : 1;
    parts = (int32_t) std::max<int64_t>(1, std::min<int64_t>(parts, std::max<int64_t>(n, 1)));
    const int nSlots = std::min<int>(parts, mp_engine::kPipeSlots);
    if (!e->outStream) CUDA_TRY(cudaStreamCreateWithFlags(&e->outStream, cudaStreamNonBlocking));
    for (int k = 0; k < nSlots; k++) {
        if (e->pipe[k]) continue;
        mp_device_batch *db = new mp_device_batch();
        if (cudaStreamCreateWithFlags(&db->stream, cudaStreamNonBlocking) != cudaSuccess) {
            db->stream = nullptr;
            delete db;
            return failf(MP_ERR_CUDA, "stream creation failed");
        }
        db->ownStream = true;
        int leastPrio = 0, greatestPrio = 0;
        cudaDeviceGetStreamPriorityRange(&leastPrio, &greatestPrio);
        if (cudaStreamCreateWithPriority(&db->copyStream, cudaStreamNonBlocking, greatestPrio) != cudaSuccess ||
            cudaEventCreateWithFlags(&db->evCompacted, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&db->evCopied, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&db->evUploaded, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&db->evKernels, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&db->evStatus, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&db->evReady, cudaEventDisableTiming) != cudaSuccess) {
            delete db;
            return failf(MP_ERR_CUDA, "stream / event creation failed");
        }
        e->pipe[k] = db;
    }
    const std::vector<int64_t> cut = sliceJobs(b, parts);
    const int nSlices = (int) cut.size() - 1;
    int64_t base[3] = {0, 0, 0};
    bool over[3] = {false, false, false};
    for (int k = 0; k < 3; k++)
        if (out->offsets[k]) out->offsets[k][0] = 0;
    // finishes slice i (waits for its run, re-runs what needs it) and queues its tuple copies;
    // slices finish in order, since a slice's output offsets follow the tuples of those before it
    int finished = 0;
    auto finishNext = [&]() -> mp_status {
        mp_device_batch *db = e->pipe[finished % nSlots];
        MP_TRY(runFinish(e, db, nullptr));
        int64_t total[3];
        MP_TRY(fetchIssue(e, db, out, cut[finished], base, cap, total));
        for (int k = 0; k < 3; k++) {
            if (base[k] + total[k] > cap[k]) over[k] = true;
            base[k] += total[k];
        }
        finished++;
        return MP_OK;
    };
    // Every slice is planned, copied in and launched on its own slot as early as the slots allow
    // (all at once when there are no more slices than slots): later slices' kernels fill the SMs
    // that an earlier slice's last tasks leave idle, and each slice's tuples stream out as soon
    // as its kernels end.
    // The slices' input copies run one after another in slice order (each slot's stream waits
    // for the previous slice's copies), so the first slices' inputs arrive at the link's full
    // speed instead of sharing it with every later slice's.
    mp_status st = MP_OK;
    cudaEvent_t prevUploaded = nullptr;
    for (int i = 0; st == MP_OK && i < nSlices; i++) {
        if (i >= nSlots) st = finishNext();  // frees slot i % nSlots
        if (st != MP_OK) break;
        const int64_t j0 = cut[i], j1 = cut[i + 1];
        std::vector<int64_t> yOff(j1 - j0 + 1), aOff(j1 - j0 + 1);
        for (int64_t j = j0; j <= j1; j++) {
            yOff[j - j0] = b->y_offsets[j] - b->y_offsets[j0];
            aOff[j - j0] = b->anchor_offsets[j] - b->anchor_offsets[j0];
        }
        mp_batch sb = *b;
        sb.n_jobs = j1 - j0;
        sb.x_begin = b->x_begin + j0;
        sb.x_end = b->x_end + j0;
        sb.y_offsets = yOff.data();
        sb.y_symbols = b->y_symbols ? b->y_symbols + b->y_offsets[j0] : nullptr;
        sb.anchor_offsets = aOff.data();
        sb.anchors = b->anchors ? b->anchors + 3 * b->anchor_offsets[j0] : nullptr;
        sb.strand = b->strand + j0;
        sb.ragged_left = b->ragged_left ? b->ragged_left + j0 : nullptr;
        sb.ragged_right = b->ragged_right ? b->ragged_right + j0 : nullptr;
        sb.x_shift = b->x_shift ? b->x_shift + j0 : nullptr;
        mp_device_batch *db = e->pipe[i % nSlots];
        db->mode = kModePosterior;
        db->outStream = e->outStream;
        db->scratchBudget = e->scratchBudget / (size_t) nSlots;
        // a reused slot's previous slice has queued its copies on the slot's streams: the new
        // inputs follow them in stream order; the batch's host arrays stay valid until the return
        // the slot's previous slice is compacted and copied out on the copy stream: its buffers
        // are rewritten only after that (a wait on the device, not on the host)
        if (db->copyPending && cudaStreamWaitEvent(db->stream, db->evCopied, 0) != cudaSuccess) {
            st = failf(MP_ERR_CUDA, "stream wait failed");
            break;
        }
        if (prevUploaded && cudaStreamWaitEvent(db->stream, prevUploaded, 0) != cudaSuccess) {
            st = failf(MP_ERR_CUDA, "stream wait failed");
            break;
        }
        st = batchReset(e, db, m, p, &sb, false);
        if (st == MP_OK && cudaEventRecord(db->evUploaded, db->stream) != cudaSuccess)
            st = failf(MP_ERR_CUDA, "event record failed");
        prevUploaded = db->evUploaded;
        if (st == MP_OK) st = runIssue(e, db);
        // slices whose kernels have ended are finished at once (their tuples start to leave)
        // rather than after the last slice is planned
        while (st == MP_OK && finished < i && cudaEventQuery(e->pipe[finished % nSlots]->evStatus) == cudaSuccess)
            st = finishNext();
    }
    while (st == MP_OK && finished < nSlices) st = finishNext();
    for (int k = 0; k < nSlots; k++) {
        cudaError_t ce = cudaStreamSynchronize(e->pipe[k]->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->pipe[k]->copyStream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->outStream);
        e->pipe[k]->copyPending = false;
        if (st == MP_OK && ce != cudaSuccess)
            st = failf(MP_ERR_CUDA, "pipelined pass failed: %s", cudaGetErrorString(ce));
    }
    if (st != MP_OK) return st;
    if (need)
        for (int k = 0; k < 3; k++) need[k] = base[k];
    if (over[0] || over[1] || over[2])
        return failf(MP_ERR_OVERFLOW, "output capacity too small: need %lld / %lld / %lld tuples",
                     (long long) base[0], (long long) base[1], (long long) base[2]);
    return MP_OK;
}

// ---------------------------------------------------------------------------
// forward likelihood (computeForwardProbability) and the adjoint (expected counts)
// ---------------------------------------------------------------------------

// Runs a batch in `mode` on the engine's cached batch of that mode.
static mp_status runMode(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b, int mode,
                         mp_device_batch **slot, mp_device_batch **ran) {
    if (!*slot) *slot = new mp_device_batch();
    mp_device_batch *db = *slot;
    db->mode = mode;
    MP_TRY(batchReset(e, db, m, p, b));
    MP_TRY(mp_device_batch_run(e, db, nullptr));
    *ran = db;
    return MP_OK;
}

extern "C" mp_status mp_forward_batch(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                      double *log_prob) {
    if (!e || !m || !p || !b || (b->n_jobs > 0 && !log_prob))
        return failf(MP_ERR_ARGUMENT, "mp_forward_batch: NULL argument");
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    mp_device_batch *db = nullptr;
    MP_TRY(runMode(e, m, p, b, kModeForward, &e->forwardShot, &db));
    for (int64_t j = 0; j < db->nJobs; j++) {
        double ll = 0.0;
        for (int64_t t = db->jobFirstTask[j]; t < db->jobFirstTask[j + 1]; t++) ll += db->hostOut[t].logLik;
        log_prob[j] = ll;
    }
    return MP_OK;
}

extern "C" mp_status mp_expectations_batch(mp_engine *e, const mp_model *m, const mp_params *p, const mp_batch *b,
                                           mp_expectations *out, double *log_lik) {
    if (!e || !m || !p || !b || !out) return failf(MP_ERR_ARGUMENT, "mp_expectations_batch: NULL argument");
    std::lock_guard<std::mutex> guard(e->oneShotLock);
    mp_device_batch *db = nullptr;
    MP_TRY(runMode(e, m, p, b, kModeAdjoint, &e->adjointShot, &db));
    std::vector<double> small(2 * kExpPerModel, 0.0), rep(2 * kRepTable, 0.0);
    if (!db->tasks.empty()) {
        MP_TRY(db->expect.reserve(sizeof(double) * 2 * kExpPerModel));
        MP_TRY(db->expectRep.reserve(sizeof(double) * 2 * kRepTable));
        CUDA_TRY(cudaMemcpy(small.data(), db->expect.p, sizeof(double) * small.size(), cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(rep.data(), db->expectRep.p, sizeof(double) * rep.size(), cudaMemcpyDeviceToHost));
    }
    memset(out, 0, sizeof(*out));
    for (int md = 0; md < 2; md++) {
        const double *g = small.data() + md * kExpPerModel;
        for (int k = 0; k < 9; k++) out->transitions[md][k] = g[kExpTrans + k] * std::exp(m->logT[md][k]);
        for (int k = 0; k < 25; k++) out->match[md][k] = g[kExpMatch + k];
        for (int k = 0; k < 5; k++) {
            out->gap_x[md][k] = g[kExpGapX + k];
            out->gap_y[md][k] = g[kExpGapY + k];
        }
        for (int k = 0; k < 3; k++) {
            out->start[md][k] = g[kExpStart + k];
            out->end[md][k] = g[kExpEnd + k];
        }
        for (int k = 0; k < kRepTable; k++) out->repeat[md][k] = rep[(size_t) md * kRepTable + k];
    }
    double total = 0.0;
    for (int64_t j = 0; j < db->nJobs; j++) {
        double ll = 0.0;
        for (int64_t t = db->jobFirstTask[j]; t < db->jobFirstTask[j + 1]; t++) ll += db->hostOut[t].logLik;
        if (log_lik) log_lik[j] = ll;
        total += ll;
    }
    out->log_likelihood = total;
    return MP_OK;
}

extern "C" mp_status mp_host_alloc(size_t bytes, void **out) {
    if (!out) return failf(MP_ERR_ARGUMENT, "mp_host_alloc: out is NULL");
    *out = nullptr;
    CUDA_TRY(cudaHostAlloc(out, bytes > 0 ? bytes : 1, cudaHostAllocPortable));
    return MP_OK;
}

extern "C" void mp_host_free(void *p) {
    if (p) cudaFreeHost(p);
}
