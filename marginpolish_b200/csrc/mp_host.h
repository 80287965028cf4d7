// Host-side objects shared by the C ABI translation units (internal).
#pragma once

#include "../../include/mpgpu.h"
#include "mp_internal.h"

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <vector>
#include <string>

// Records the thread-local error message of the C ABI and returns s.
mp_status mp_fail(mp_status s, const char *fmt, ...);

// Reference restatements used by the planner (defined in mp_api.cu).
namespace mp {
struct SplitRectH {
    int64_t x1, y1, x2, y2;
};
// Number of split rectangles of one job (getSplitPoints, impl/pairwiseAligner.c:899-926).
int64_t splitCount(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, int64_t maxSize, bool raggedL, bool raggedR);
// The split rectangles themselves (same rule; a single rectangle may be trimmed when a ragged
// end skips the first or last large gap).
void splitRects(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, int64_t maxSize, bool raggedL, bool raggedR,
                std::vector<SplitRectH> &out);
// Upper bound of the 5-diagonal band hull in window slots.
int64_t hullSlots(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, bool dynamic, int64_t fixedExp);
// The same bound for the sub-rectangle with origin (x1, y1) and lengths (lx, ly), whose anchors
// are given in the job's coordinates.
int64_t hullSlotsRect(const int32_t *an, int64_t nA, int64_t x1, int64_t y1, int64_t lx, int64_t ly, bool dynamic,
                      int64_t fixedExp);
// Checks anchor order / range / expansion parity of one job.
mp_status validateAnchors(const int32_t *an, int64_t nA, int64_t lx, int64_t ly, bool dynamic, int64_t job);
mp_status validateParamsStruct(const mp_params *p);
}  // namespace mp

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // Grows to at least n bytes, with headroom of half the need up to 64 MiB: buffers sized by
    // per-call counts (tuples, tasks) then stop growing after a few calls. Growth frees the old
    // buffer, and cudaFree waits for the whole device, which would stall other threads' passes.
    mp_status reserve(size_t n) {
        if (n <= bytes && p) return MP_OK;
        release();
        size_t want = n > 0 ? n + std::min(n / 2, (size_t) 64 << 20) : 16;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            return mp_fail(MP_ERR_MEMORY, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        }
        bytes = want;
        return MP_OK;
    }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

// Grow-only page-locked host buffer (staging for the planner's small uploads, so that their
// copies are asynchronous DMA like the caller's page-locked inputs).
struct PinBuf {
    void *p = nullptr;
    size_t bytes = 0;
    PinBuf() = default;
    PinBuf(const PinBuf &) = delete;
    PinBuf &operator=(const PinBuf &) = delete;
    ~PinBuf() {
        if (p) cudaFreeHost(p);
    }
    mp_status reserve(size_t n) {
        if (n <= bytes && p) return MP_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t want = n + n / 4 + 256;
        if (cudaMallocHost(&p, want) != cudaSuccess) {
            p = nullptr;
            return mp_fail(MP_ERR_MEMORY, "cudaMallocHost(%zu) failed", want);
        }
        bytes = want;
        return MP_OK;
    }
};

// ---------------------------------------------------------------------------
// engine and model
// ---------------------------------------------------------------------------

// Device arrays of mp_forward_pairs (grow only).
struct mp_pair_scratch {
    DevBuf idx, xOff, yOff, xLen, yLen, strand, xs, ys, out, rowOff, rows;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    float kernelMs = 0.0f;  // device time of the last call's launches
    int64_t cells = 0;      // matrix cells of the last call: sum of (lx + 1) (ly + 1)
    int64_t pairs = 0;
    mp_pair_scratch() = default;
    mp_pair_scratch(const mp_pair_scratch &) = delete;
    mp_pair_scratch &operator=(const mp_pair_scratch &) = delete;
    ~mp_pair_scratch() {
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    }
};

struct mp_engine {
    int device = 0;
    int smCount = 0;
    int ccMajor = 0, ccMinor = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Device bytes one batch may hold for forward checkpoints (half the device's memory). A
    // batch whose persistent grid would need more runs on fewer blocks; the pipelined call splits
    // the budget over its slots.
    size_t scratchBudget = 0;
    mp_tuning tuning{};
    bool graphs = false;  // device-batch passes run as captured CUDA graphs
    // autotuned choice (mp_engine_autotune): ascending hull-class bounds with the FP32 kernel
    // variant of each class, and warps per block per variant (0: as many as fit); empty when
    // not tuned
    std::vector<int> tunedBound, tunedVariant, tunedWarps;
    struct mp_device_batch *oneShot = nullptr;  // reused by the one-shot calls (mp_realign_batch*)
    struct mp_device_batch *forwardShot = nullptr;  // reused by mp_forward_batch
    struct mp_device_batch *adjointShot = nullptr;  // reused by mp_expectations_batch
    static constexpr int kPipeSlots = 8;
    struct mp_device_batch *pipe[kPipeSlots] = {};  // the slots of mp_realign_batch_into (own streams)
    cudaStream_t outStream = nullptr;  // tuple copies of mp_realign_batch_into's slots, in slice order
    mp_pair_scratch pairScratch;       // mp_forward_pairs (under oneShotLock)
    struct mp_node_scratch *nodeScratch = nullptr;    // mp_node_update's device arrays
    struct mp_indel_scratch *indelScratch = nullptr;  // the indel candidates' device arrays
    // Page-locked tuple arrays of the POA sets' realignments (w, x, y of each list, grow only),
    // kept by the engine so that later sets do not pin memory again; a realignment holds
    // poaLock while it uses them.
    PinBuf poaTuples[3];
    std::mutex poaLock;
    std::mutex oneShotLock;
};

// Frees the node update's device arrays (mp_nodes.cu).
void mp_node_scratch_free(struct mp_node_scratch *s);
// Frees the indel candidates' device arrays (mp_indels.cu).
void mp_indel_scratch_free(struct mp_indel_scratch *s);

namespace mp {
// Inputs of the complete-indel candidates of many reads (mp_indels.cu): per job its reference's
// and its read's runs in the flat run arrays, and its three tuple lists (matches, gap-x, gap-y)
// with nJobs + 1 offsets each.
struct IndelBatch {
    int64_t nJobs = 0;
    const int64_t *refBase = nullptr, *refRuns = nullptr, *readBase = nullptr, *readRuns = nullptr;
    int64_t nRefRuns = 0, nReadRuns = 0;
    const char *refChars = nullptr;
    const uint32_t *refCounts = nullptr;
    const char *readChars = nullptr;
    const uint32_t *readCounts = nullptr;
    const int64_t *off[3] = {nullptr, nullptr, nullptr};
    const int32_t *w[3] = {nullptr, nullptr, nullptr}, *x[3] = {nullptr, nullptr, nullptr},
                  *y[3] = {nullptr, nullptr, nullptr};
    bool cmpRC = true;
};
// Candidates of every job, inserts first, in poa_augment's order: job j's are
// [candOff[j], candOff[j+1]) of which the first nIns[j] are inserts, whose runs are
// [runOff[j] + at, runOff[j] + at + len) of chars / counts. The per-candidate arrays are
// page-locked buffers of the engine, valid until its next deviceIndelCandidates call.
struct IndelOut {
    std::vector<int64_t> candOff, runOff, nIns;
    const int64_t *pos = nullptr, *len = nullptr, *at = nullptr, *offset = nullptr;
    const uint64_t *nonRle = nullptr;
    const double *weight = nullptr;
    const char *chars = nullptr;
    const uint64_t *counts = nullptr;
};
mp_status deviceIndelCandidates(mp_engine *e, const IndelBatch &b, IndelOut &out);
}  // namespace mp

struct mp_model {
    mp_engine *engine = nullptr;
    int sharedRepeat = 0;  // the two strands' repeat tables are identical
    int noSwitch = 0;      // both strands' switch transitions (gap-x <-> gap-y) are zero
    mp::DevModel host[2];
    double logT[2][9];   // log transitions as given (the adjoint scales its sums by exp(logT))
    DevBuf models;   // DevModel[2]
    DevBuf repeat;   // float [2][kRepTable]
    // FP64 log-space copy for the bubble scorer (mp_forward_pairs)
    mp::DevLogModel logHost[2];
    DevBuf logModels;  // DevLogModel[2]
    DevBuf logRepeat;  // double [2][kRepTable]: repeat_scale * log10 table
};

// Fills the FP64 log-space tables of one strand's model (defined in mp_bubble.cu).
mp_status mp_model_lower_log(const mp_model_desc *d, mp::DevLogModel &m, double *rep);

// Anchor-free alignments whose match posteriors are computed in the reference's own arithmetic
// (getAlignedPairs over the whole matrix, FP64 logs, its approximate log-sum; defined in
// mp_refpost.cu), for the few small alignments whose results decide a choice among near-equal
// weights (the cut of chunk stitching). The model must be without run lengths.
struct RefPair {
    int64_t xOff, yOff;   // into the x and y symbol arrays
    int32_t lx, ly;
    bool raggedLeft, raggedRight, forward;
};
struct RefTuple {
    int32_t weight, x, y;
};
constexpr int64_t kRefMaxCells = (int64_t) 1 << 22;  // per alignment
// out[k]: pair k's match tuples in the reference's list order.
mp_status refMatchPairs(mp_engine *e, const mp_model *m, const mp_params *p, const std::vector<RefPair> &pairs,
                        const std::vector<uint16_t> &xs, const std::vector<uint16_t> &ys,
                        std::vector<std::vector<RefTuple>> &out);
