// Single-read posterior pass that allocates no memory.
//
// Some callers cannot allocate device memory at all: a host application whose
// framework owns every byte of the GPU through its own pool (so cudaMalloc
// either fails or fights the pool), or code running where allocation is not
// permitted at call time. mp_realign_single_noalloc serves them: every buffer
// the pass needs beyond the caller's host inputs and outputs -- the task
// record, the band records, the forward checkpoints, the output staging and
// the device copies of the symbols and anchors -- lives in one file-scope
// device array of fixed size, g_noallocScratch, that each GPU loading this
// library holds until the process exits.
//
// Limits (checked before any device work, MP_ERR_ARGUMENT beyond them): one
// read, lx + ly <= MP_NOALLOC_MAX_DIAGONALS - 1, a single split rectangle
// (possibly trimmed by a ragged end, as in the batched pass), and a band hull
// of at most 60 window slots (the narrowest slot class).
//
// The first call on a device takes the array's device address with
// cudaGetSymbolAddress while that device is current, so that first call
// should happen before any stream capture. Calls share the array: the pass
// writes every word it later reads (and zeroes its work counter and status
// record itself), and calls serialise on an internal mutex and wait for their
// own completion, on the error paths too; two calls that ran on the GPU at the
// same time would race.
#include "../../include/mpgpu.h"
#include "mp_host.h"
#include "mp_internal.h"

#include <algorithm>
#include <cstring>
#include <mutex>

namespace mp {
cudaError_t launchVariant(int v, const DpArgs &a, int blocks, int warps, cudaStream_t s);
cudaError_t launchBand(const BandArgs &a, cudaStream_t s);
cudaError_t launchCompact(const CompactArgs &a, cudaStream_t s);
}  // namespace mp

using namespace mp;

namespace {

constexpr int64_t kMaxDiag = MP_NOALLOC_MAX_DIAGONALS;  // anti-diagonals 0..N with N < kMaxDiag
constexpr int kVariant = 0;                                // kernel variant used: one task per warp,
constexpr int kC = 2;                                      // 2 slots per lane (window of 64 slots),
constexpr int kK = 8;                                      // checkpoint stride 8
constexpr int64_t kBlocks = kMaxDiag / kK + 2;
constexpr int64_t kCapM = kMaxDiag + kMaxDiag / 8 + 64;
constexpr int64_t kCapG = kMaxDiag * 3 / 4 + 64;

constexpr size_t align256(size_t v) {
    return (v + 255) & ~(size_t) 255;
}

// byte offsets inside the scratch array
constexpr size_t kOffTask = 0;
constexpr size_t kOffTaskOut = align256(kOffTask + sizeof(Task));
constexpr size_t kOffQueue = align256(kOffTaskOut + sizeof(TaskOut));  // queue counter, then order[0]
constexpr size_t kOffXs = align256(kOffQueue + 2 * sizeof(int32_t));
constexpr size_t kOffYs = align256(kOffXs + kMaxDiag * sizeof(uint16_t));
constexpr size_t kOffAnchors = align256(kOffYs + kMaxDiag * sizeof(uint16_t));
constexpr size_t kOffBand = align256(kOffAnchors + (kMaxDiag / 2 + 1) * 3 * sizeof(int32_t));
constexpr size_t kOffChk = align256(kOffBand + (kMaxDiag + 1) * sizeof(int4));
constexpr size_t kOffScal = align256(kOffChk + kBlocks * kC * 32 * sizeof(float4));
constexpr size_t kOffStage = align256(kOffScal + kBlocks * sizeof(int2));
constexpr int64_t kCap[3] = {kCapM, kCapG, kCapG};
constexpr size_t kOffStageList(int k) {  // staged tuples (weight, x, y, 0) of list k
    size_t off = kOffStage;
    for (int i = 0; i < k; i++) off += align256(kCap[i] * sizeof(int4));
    return off;
}
constexpr size_t kOffOut = kOffStageList(2) + align256(kCap[2] * sizeof(int4));
constexpr size_t kOffOutList(int k, int field) {  // compacted lists; field 0 weight, 1 x, 2 y
    size_t off = kOffOut;
    for (int i = 0; i < k; i++) off += 3 * align256(kCap[i] * sizeof(int32_t));
    return off + (size_t) field * align256(kCap[k] * sizeof(int32_t));
}
constexpr size_t kUsed = kOffOutList(2, 2) + align256(kCap[2] * sizeof(int32_t));

}  // namespace

// The scratch of the no-allocation entry point (one per device that loads the library).
static __device__ __align__(256) unsigned char g_noallocScratch[MP_NOALLOC_SCRATCH_BYTES];
static_assert(kUsed <= MP_NOALLOC_SCRATCH_BYTES, "no-allocation scratch layout exceeds the array");

namespace {
std::mutex gNoallocMutex;
constexpr int kMaxDevices = 128;
unsigned char *gNoallocAddr[kMaxDevices] = {nullptr};
}  // namespace

extern "C" mp_status mp_realign_single_noalloc(mp_engine *e, const mp_model *m, const mp_params *p,
                                               const uint16_t *x, int64_t lx, const uint16_t *y, int64_t ly,
                                               const int32_t *anchors, int64_t nAnchors, int strand, int raggedLeft,
                                               int raggedRight, mp_noalloc_output *out) {
    if (!e || !m || !p || !out) return mp_fail(MP_ERR_ARGUMENT, "mp_realign_single_noalloc: NULL argument");
    if (lx < 0 || ly < 0 || nAnchors < 0 || (lx > 0 && !x) || (ly > 0 && !y) || (nAnchors > 0 && !anchors))
        return mp_fail(MP_ERR_ARGUMENT, "mp_realign_single_noalloc: bad sequence or anchor arguments");
    if (lx + ly >= kMaxDiag)
        return mp_fail(MP_ERR_ARGUMENT,
                       "mp_realign_single_noalloc: lx + ly = %lld exceeds the no-allocation limit of %lld",
                       (long long) (lx + ly), (long long) (kMaxDiag - 1));
    for (int k = 0; k < 3; k++) {
        if (out->capacity[k] < 0 ||
            (out->capacity[k] > 0 && (!out->weight[k] || !out->x[k] || !out->y[k])))
            return mp_fail(MP_ERR_ARGUMENT, "mp_realign_single_noalloc: output list %d has no storage", k);
    }
    mp_status st = validateParamsStruct(p);
    if (st != MP_OK) return st;
    const bool dynamic = p->dynamic_anchor_expansion != 0;
    st = validateAnchors(anchors, nAnchors, lx, ly, dynamic, 0);
    if (st != MP_OK) return st;
    // The single split rectangle of the read. With a ragged end the rule may skip the first or
    // last large gap, so the rectangle can be a trimmed part of the matrix: the task then covers
    // exactly that rectangle (origin x1, y1), as the batched planner does.
    std::vector<SplitRectH> rects;
    splitRects(anchors, nAnchors, lx, ly, p->split_matrix_bigger_than_this, raggedLeft != 0, raggedRight != 0, rects);
    if (rects.size() != 1)
        return mp_fail(MP_ERR_ARGUMENT,
                       "mp_realign_single_noalloc: the read needs split rectangles; use mp_realign_batch");
    const SplitRectH r = rects[0];
    const int64_t rlx = r.x2 - r.x1, rly = r.y2 - r.y1;
    const int64_t slots = hullSlotsRect(anchors, nAnchors, r.x1, r.y1, rlx, rly, dynamic, p->diagonal_expansion);
    if (slots > 32 * kC - 2 * kC)
        return mp_fail(MP_ERR_ARGUMENT,
                       "mp_realign_single_noalloc: band hull of %lld slots exceeds the limit of %d; use "
                       "mp_realign_batch",
                       (long long) slots, 32 * kC - 2 * kC);
    if (e->device < 0 || e->device >= kMaxDevices)
        return mp_fail(MP_ERR_ARGUMENT, "mp_realign_single_noalloc: device index %d outside [0, %d)", e->device,
                       kMaxDevices);

    std::lock_guard<std::mutex> lock(gNoallocMutex);
    cudaError_t ce = cudaSetDevice(e->device);
    if (ce != cudaSuccess) return mp_fail(MP_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(ce));
    if (gNoallocAddr[e->device] == nullptr) {
        // set-up, once per device, with that device current
        unsigned char *ptr = nullptr;
        ce = cudaGetSymbolAddress((void **) &ptr, g_noallocScratch);
        if (ce != cudaSuccess || ptr == nullptr)
            return mp_fail(MP_ERR_CUDA, "cudaGetSymbolAddress(no-allocation scratch): %s", cudaGetErrorString(ce));
        gNoallocAddr[e->device] = ptr;
    }
    unsigned char *base = gNoallocAddr[e->device];
    cudaStream_t s = e->stream;
    // Every return after the first queued copy waits for the stream first (declared after the
    // lock, so it runs before the unlock): a failed call never leaves work that writes the shared
    // array running while the next call starts.
    struct StreamDrain {
        cudaStream_t s;
        bool armed = false;
        ~StreamDrain() {
            if (armed) (void) cudaStreamSynchronize(s);
        }
    } drain{s};

    const int32_t N = (int32_t) (rlx + rly);
    Task tk;
    memset(&tk, 0, sizeof(tk));
    tk.lx = (int32_t) rlx;
    tk.ly = (int32_t) rly;
    tk.x1 = (int32_t) r.x1;
    tk.y1 = (int32_t) r.y1;
    tk.nAnchors = (int32_t) nAnchors;
    tk.flags = (raggedLeft ? 1 : 0) | (raggedRight ? 2 : 0) | (strand ? 4 : 0) | (dynamic ? 8 : 0);
    tk.expansion = (int32_t) p->diagonal_expansion;
    const int64_t caps[3] = {N + N / 8 + 64, (int64_t) N * 3 / 4 + 64, (int64_t) N * 3 / 4 + 64};
    for (int k = 0; k < 3; k++) tk.cap[k] = (int32_t) caps[k];
    TaskOut zero;
    memset(&zero, 0, sizeof(zero));
    const int32_t queueAndOrder[2] = {0, 0};

#define NA_TRY(expr)                                                                          \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) return mp_fail(MP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

    drain.armed = true;
    NA_TRY(cudaMemcpyAsync(base + kOffTask, &tk, sizeof(tk), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + kOffTaskOut, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + kOffQueue, queueAndOrder, sizeof(queueAndOrder), cudaMemcpyHostToDevice, s));
    if (rlx > 0)
        NA_TRY(cudaMemcpyAsync(base + kOffXs, x + r.x1, sizeof(uint16_t) * rlx, cudaMemcpyHostToDevice, s));
    if (rly > 0)
        NA_TRY(cudaMemcpyAsync(base + kOffYs, y + r.y1, sizeof(uint16_t) * rly, cudaMemcpyHostToDevice, s));
    if (nAnchors > 0)
        NA_TRY(cudaMemcpyAsync(base + kOffAnchors, anchors, sizeof(int32_t) * 3 * nAnchors, cudaMemcpyHostToDevice, s));

    const Task *dTask = reinterpret_cast<const Task *>(base + kOffTask);
    TaskOut *dOut = reinterpret_cast<TaskOut *>(base + kOffTaskOut);
    BandArgs ba;
    ba.tasks = dTask;
    ba.nTasks = 1;
    ba.anchors = reinterpret_cast<const int32_t *>(base + kOffAnchors);
    ba.band = reinterpret_cast<int2 *>(base + kOffBand);
    ba.out = dOut;
    NA_TRY(launchBand(ba, s));

    DpArgs a;
    memset(&a, 0, sizeof(a));
    a.tasks = dTask;
    a.order = reinterpret_cast<const int32_t *>(base + kOffQueue) + 1;
    a.nTasks = 1;
    a.scratchBlocks = (int32_t) kBlocks;
    a.queue = reinterpret_cast<int32_t *>(base + kOffQueue);
    a.xs = reinterpret_cast<const uint16_t *>(base + kOffXs);
    a.ys = reinterpret_cast<const uint16_t *>(base + kOffYs);
    a.band = reinterpret_cast<const int2 *>(base + kOffBand);
    a.models = m->models.as<DevModel>();
    a.repeatProb = m->repeat.as<float>();
    a.scratch = reinterpret_cast<float4 *>(base + kOffChk);
    a.scratchScalars = reinterpret_cast<int2 *>(base + kOffScal);
    for (int k = 0; k < 3; k++) a.outT[k] = reinterpret_cast<int4 *>(base + kOffStageList(k));
    a.out = dOut;
    a.threshold = (float) p->threshold;
    a.minDiagsBetweenTraceBack = (int32_t) std::min<int64_t>(p->min_diags_between_traceback, 1 << 30);
    a.traceBackDiagonals = (int32_t) p->traceback_diagonals;
    a.diagonalExpansion = (int32_t) std::min<int64_t>(p->diagonal_expansion, 1 << 29);
    a.sharedRepeat = m->sharedRepeat;
    NA_TRY(launchVariant(kVariant, a, 1, 1, s));

    TaskOut res;
    NA_TRY(cudaMemcpyAsync(&res, dOut, sizeof(res), cudaMemcpyDeviceToHost, s));
    NA_TRY(cudaStreamSynchronize(s));
    drain.armed = false;  // nothing of this call is in flight until the compaction below
    if (res.status & kTaskBand) return mp_fail(MP_ERR_ARGUMENT, "invalid band diagonal (anchors inconsistent)");
    if (res.status & kTaskSymbol) return mp_fail(MP_ERR_ARGUMENT, "a symbol's repeat count is >= %d", kMaxRepeat);
    if (res.status & (kTaskWindow | kTaskScratch))
        return mp_fail(MP_ERR_OVERFLOW, "no-allocation pass exceeded its band window or checkpoint area");
    if (res.status & kTaskRange)
        return mp_fail(MP_ERR_OVERFLOW,
                       "the band's probabilities exceed the range of FP32 scaled arithmetic; use mp_realign_batch");
    out->log_likelihood = res.logLik;
    out->cells = res.cells;
    bool tooSmall = false;
    for (int k = 0; k < 3; k++) {
        out->count[k] = res.count[k];
        if (res.count[k] > tk.cap[k])
            return mp_fail(MP_ERR_OVERFLOW, "list %d: %d tuples exceed the no-allocation staging of %d", k,
                           res.count[k], tk.cap[k]);
        if (res.count[k] > out->capacity[k]) tooSmall = true;
    }
    if (tooSmall) return mp_fail(MP_ERR_OVERFLOW, "an output list is smaller than its tuple count (see count)");
    // staged records -> three arrays per list (inside the same static array), then to the host
    CompactArgs ca;
    ca.tasks = dTask;
    ca.out = dOut;
    ca.nTasks = 1;
    for (int k = 0; k < 3; k++) {
        ca.dst[k] = nullptr;
        ca.src[k] = a.outT[k];
        ca.w[k] = reinterpret_cast<int32_t *>(base + kOffOutList(k, 0));
        ca.x[k] = reinterpret_cast<int32_t *>(base + kOffOutList(k, 1));
        ca.y[k] = reinterpret_cast<int32_t *>(base + kOffOutList(k, 2));
    }
    drain.armed = true;
    NA_TRY(launchCompact(ca, s));
    for (int k = 0; k < 3; k++) {
        const int64_t n = res.count[k];
        if (n == 0) continue;
        NA_TRY(cudaMemcpyAsync(out->weight[k], ca.w[k], sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
        NA_TRY(cudaMemcpyAsync(out->x[k], ca.x[k], sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
        NA_TRY(cudaMemcpyAsync(out->y[k], ca.y[k], sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    }
    NA_TRY(cudaStreamSynchronize(s));
    drain.armed = false;
#undef NA_TRY
    return MP_OK;
}
