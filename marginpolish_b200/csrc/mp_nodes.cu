// Device-side node update of the POA graphs: the match part of poa_augment and the run-length
// estimate, computed from the posterior pass's match tuples on the GPU.
//
//   poa_augment, match weights      impl/polisher.c:322-340
//     per match (weight, x, y) of a read: node x+1 gains `weight` in the bin of the read's base
//     at y and in the bin of the read's run length at y (clamped below maxRepeatCount), and an
//     observation (read number, y, weight) is appended to the node's list
//   run-length estimate             impl/polisher.c:1556-1565, :1796-1865
//     per node i >= 1: the observed run lengths' range [lo, hi] (hi clamped below M), then for
//     every underlying length u in it the sum over the node's observations, in list order, of
//     log10 P(observed | u, base, strand) * weight, divided by 10^7; the first maximum wins, and
//     a node without observations (or whose estimate is 0) gets 1
//
// B200 layout, one pass per batch of chunks (every graph of a realignment at once):
//   scatter   one warp per read, lanes over its tuples: FP64 atomics into the base and run-length
//             bins (the weights are integers below 2^24 and their sums stay far below 2^53, so
//             every order of additions gives the same doubles) and an integer count per node;
//   scan      exclusive sum of the counts: each node's segment of the observation list;
//   place     every tuple takes a slot of its node's segment (integer atomic);
//   finish    one thread per node sorts its segment by tuple index -- tuples are numbered in
//             read order, then in the aligner's order within a read, which is the order
//             poa_augment appends observations in -- and runs the estimate over it. Every
//             product and sum is rounded on its own (__dmul_rn / __dadd_rn), as the reference's
//             separate multiply and add are, so the estimates are bit-identical.
// The work is integer and FP64 gather traffic: HBM-bound at a few tens of bytes per tuple.
#include "../../include/mpgpu.h"
#include "mp_host.h"
#include "mp_internal.h"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

namespace {

#define NODE_TRY(expr)              \
    do {                            \
        mp_status _s = (expr);      \
        if (_s != MP_OK) return _s; \
    } while (0)
#define NODE_CUDA(expr)                                                                                   \
    do {                                                                                                  \
        cudaError_t _e = (expr);                                                                          \
        if (_e != cudaSuccess) return mp_fail(MP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e));      \
    } while (0)

// The nucleotide alphabet (impl/stateMachine.c:25-59): A C G T, anything else N (4).
__device__ __forceinline__ int symbolOfDev(char ch) {
    switch (ch) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 4;
    }
}

struct ReadInfo {
    int64_t nodeBase;  // first node of the read's chunk in the batch's node arrays
    int64_t nodeEnd;   // one past its last node
    int64_t runBase;   // first run of the read in the read arrays
    int64_t runs;      // its run count
    int64_t tupBase;   // first match tuple of the read
    int64_t tupEnd;
    int32_t readNo;    // number of the read within its chunk (the observation's read)
    int32_t strand;
};

__global__ void scatterKernel(const ReadInfo *reads, int64_t nReads, const char *readChars, const uint32_t *readCounts,
                              const int32_t *w, const int32_t *x, const int32_t *y, int64_t maxRC, double *bw,
                              double *rcw, int32_t *count, int64_t *tupNode, int32_t *tupRead, int *bad) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nWarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < nReads; r += nWarps) {
        const ReadInfo ri = reads[r];
        for (int64_t t = ri.tupBase + lane; t < ri.tupEnd; t += 32) {
            const int64_t xi = x[t], yi = y[t];
            const int64_t g = ri.nodeBase + xi + 1;
            if (xi < 0 || g >= ri.nodeEnd || yi < 0 || yi >= ri.runs || w[t] < 0) {
                atomicOr(bad, 1);
                tupNode[t] = -1;
                continue;
            }
            const double wt = (double) w[t];
            const int sym = symbolOfDev(readChars[ri.runBase + yi]);
            int64_t rc = (int64_t) readCounts[ri.runBase + yi];
            rc = rc >= maxRC ? maxRC - 1 : rc;
            atomicAdd(bw + g * 5 + sym, wt);
            atomicAdd(rcw + g * maxRC + rc, wt);
            atomicAdd(count + g, 1);
            tupNode[t] = g;
            tupRead[t] = (int32_t) r;
        }
    }
}

__global__ void placeKernel(int64_t nTup, const int64_t *tupNode, const int64_t *start, int32_t *cursor,
                            int64_t *slotTuple) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < nTup; t += (int64_t) gridDim.x * blockDim.x) {
        const int64_t g = tupNode[t];
        if (g < 0) continue;
        const int32_t k = atomicAdd(cursor + g, 1);
        slotTuple[start[g] + k] = t;
    }
}

struct FinishArgs {
    int64_t nNodes;
    const int64_t *start;      // nNodes + 1
    int64_t *slotTuple;        // sorted in place per node
    const uint8_t *nodeSym;    // per node: the symbol of its base
    const uint8_t *nodeFirst;  // per node: 1 for a chunk's 'N' prefix node (no estimate)
    const int32_t *tupRead;
    const int32_t *w, *y;
    const ReadInfo *reads;
    const uint32_t *readCounts;
    const double *log10;       // [4][M][M], NULL: no estimate
    int64_t M;
    uint64_t *repeatCount;     // per node
    int64_t *obsRead, *obsOffset;
    double *obsWeight;
};

__global__ void finishKernel(FinishArgs a) {
    for (int64_t g = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; g < a.nNodes;
         g += (int64_t) gridDim.x * blockDim.x) {
        const int64_t s0 = a.start[g], s1 = a.start[g + 1];
        int64_t *seg = a.slotTuple + s0;
        const int64_t n = s1 - s0;
        // insertion sort by tuple index: the observation order of poa_augment
        for (int64_t i = 1; i < n; i++) {
            const int64_t v = seg[i];
            int64_t j = i - 1;
            while (j >= 0 && seg[j] > v) {
                seg[j + 1] = seg[j];
                j--;
            }
            seg[j + 1] = v;
        }
        if (a.obsRead) {
            for (int64_t i = 0; i < n; i++) {
                const int64_t t = seg[i];
                a.obsRead[s0 + i] = a.reads[a.tupRead[t]].readNo;
                a.obsOffset[s0 + i] = a.y[t];
                a.obsWeight[s0 + i] = (double) a.w[t];
            }
        }
        if (!a.log10 || !a.repeatCount) continue;
        if (a.nodeFirst[g]) {
            a.repeatCount[g] = 0;
            continue;
        }
        // repeatSubMatrix_getMinAndMaxRepeatCountObservations (impl/polisher.c:1813-1834)
        const int64_t M = a.M;
        int64_t lo = M, hi = 0;
        for (int64_t i = 0; i < n; i++) {
            const int64_t t = seg[i];
            const ReadInfo &ri = a.reads[a.tupRead[t]];
            const int64_t c = (int64_t) a.readCounts[ri.runBase + a.y[t]];
            lo = c < lo ? c : lo;
            hi = c > hi ? c : hi;
        }
        if (hi >= M) hi = M - 1;
        uint64_t est = 0;
        if (lo != M) {
            int base = a.nodeSym[g];
            if (base == 4) base = 0;  // 'N' reads the A table
            double best = 0.0;
            int64_t bestAt = 0;
            for (int64_t u = lo; u <= hi; u++) {
                // repeatSubMatrix_getLogProbForGivenRepeatCount (impl/polisher.c:1796-1811)
                double lp = 0.0;
                for (int64_t i = 0; i < n; i++) {
                    const int64_t t = seg[i];
                    const ReadInfo &ri = a.reads[a.tupRead[t]];
                    int64_t c = (int64_t) a.readCounts[ri.runBase + a.y[t]];
                    c = c >= M ? M - 1 : c;
                    const int row = ri.strand ? base : 3 - base;
                    const double l = a.log10[((int64_t) row * M + u) * M + c];
                    lp = __dadd_rn(lp, __dmul_rn(l, (double) a.w[t]));
                }
                lp = lp / (double) mp::kProbOne;
                if (u == lo || lp > best) {  // getMax: the first maximum
                    best = lp;
                    bestAt = u - lo;
                }
            }
            est = (uint64_t) (bestAt + lo);
        }
        a.repeatCount[g] = est == 0 ? 1 : est;  // poa_estimateRepeatCountsUsingBayesianModel
    }
}

}  // namespace

// Device buffers of the node update (grow only), one set per engine.
struct mp_node_scratch {
    DevBuf reads, chars, counts, w, x, y, bw, rcw, count, start, cursor, tupNode, tupRead, slot, nodeSym, nodeFirst,
        log10, rc, obsRead, obsOffset, obsWeight, cubTemp, bad;
    // its own stream: the loop runs the node update beside other GPU work of the same engine
    cudaStream_t stream = nullptr;
    ~mp_node_scratch() {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

std::mutex gNodeLock;  // one node update at a time per process (they share the engine's scratch)

mp_status validate(const mp_node_batch *b) {
    if (!b) return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: NULL batch");
    if (b->n_chunks < 0 || b->max_repeat < 2)
        return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: bad chunk count or max_repeat (%lld)", (long long) b->max_repeat);
    if (b->n_chunks > 0 && (!b->node_offsets || !b->node_bases || !b->chunk_reads || !b->read_offsets ||
                            !b->strand || !b->match_offsets))
        return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: missing input array");
    for (int64_t c = 0; c < b->n_chunks; c++) {
        if (b->node_offsets[c + 1] <= b->node_offsets[c])
            return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: chunk %lld has no nodes", (long long) c);
        if (b->chunk_reads[c + 1] < b->chunk_reads[c])
            return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: chunk %lld: bad read range", (long long) c);
    }
    if (b->n_chunks > 0 && (b->node_offsets[0] != 0 || b->chunk_reads[0] != 0))
        return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: offsets must start at 0");
    const int64_t nReads = b->n_chunks > 0 ? b->chunk_reads[b->n_chunks] : 0;
    for (int64_t r = 0; r < nReads; r++) {
        if (b->read_offsets[r + 1] < b->read_offsets[r] || b->match_offsets[r + 1] < b->match_offsets[r])
            return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: read %lld: bad offsets", (long long) r);
    }
    if (nReads > 0 && (b->read_offsets[0] != 0 || b->match_offsets[0] != 0))
        return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: offsets must start at 0");
    const int64_t nRuns = nReads > 0 ? b->read_offsets[nReads] : 0;
    const int64_t nTup = nReads > 0 ? b->match_offsets[nReads] : 0;
    if ((nRuns > 0 && (!b->read_chars || !b->read_counts)) || (nTup > 0 && (!b->weight || !b->x || !b->y)))
        return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: missing read or tuple array");
    const int64_t nNodes = b->n_chunks > 0 ? b->node_offsets[b->n_chunks] : 0;
    if (nTup >= INT32_MAX || nReads >= INT32_MAX || nNodes >= INT32_MAX)
        return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: 2^31 or more tuples, reads or nodes");
    return MP_OK;
}

template <class T>
mp_status upload(DevBuf &d, const T *h, int64_t n, cudaStream_t s) {
    NODE_TRY(d.reserve(sizeof(T) * (size_t) std::max<int64_t>(n, 1)));
    if (n > 0) NODE_CUDA(cudaMemcpyAsync(d.p, h, sizeof(T) * (size_t) n, cudaMemcpyHostToDevice, s));
    return MP_OK;
}

template <class T>
mp_status download(T *h, const DevBuf &d, int64_t n, cudaStream_t s) {
    if (h && n > 0) NODE_CUDA(cudaMemcpyAsync(h, d.p, sizeof(T) * (size_t) n, cudaMemcpyDeviceToHost, s));
    return MP_OK;
}

int gridFor(int64_t work, int threads, int smCount) {
    const int64_t need = (work + threads - 1) / threads;
    return (int) std::max<int64_t>(1, std::min<int64_t>(need, (int64_t) smCount * 16));
}

}  // namespace

extern "C" mp_status mp_node_update(mp_engine *e, const mp_node_batch *b, const mp_node_result *r) {
    if (!e || !r) return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: NULL argument");
    NODE_TRY(validate(b));
    std::lock_guard<std::mutex> guard(gNodeLock);
    NODE_CUDA(cudaSetDevice(e->device));
    if (!e->nodeScratch) e->nodeScratch = new mp_node_scratch();
    mp_node_scratch &s = *e->nodeScratch;
    if (!s.stream) NODE_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    cudaStream_t st = s.stream;
    const int64_t nC = b->n_chunks;
    const int64_t nNodes = nC > 0 ? b->node_offsets[nC] : 0;
    const int64_t nReads = nC > 0 ? b->chunk_reads[nC] : 0;
    const int64_t nRuns = nReads > 0 ? b->read_offsets[nReads] : 0;
    const int64_t nTup = nReads > 0 ? b->match_offsets[nReads] : 0;
    const int64_t M = b->max_repeat;

    // per-read and per-node descriptors (host, small)
    std::vector<ReadInfo> ri((size_t) nReads);
    std::vector<uint8_t> sym((size_t) nNodes), first((size_t) nNodes, 0);
    for (int64_t c = 0; c < nC; c++) {
        for (int64_t r0 = b->chunk_reads[c]; r0 < b->chunk_reads[c + 1]; r0++) {
            ReadInfo &q = ri[(size_t) r0];
            q.nodeBase = b->node_offsets[c];
            q.nodeEnd = b->node_offsets[c + 1];
            q.runBase = b->read_offsets[r0];
            q.runs = b->read_offsets[r0 + 1] - b->read_offsets[r0];
            q.tupBase = b->match_offsets[r0];
            q.tupEnd = b->match_offsets[r0 + 1];
            q.readNo = (int32_t) (r0 - b->chunk_reads[c]);
            q.strand = b->strand[r0] ? 1 : 0;
        }
        first[(size_t) b->node_offsets[c]] = 1;
    }
    for (int64_t g = 0; g < nNodes; g++) {
        const char ch = b->node_bases[g];
        sym[(size_t) g] = ch == 'A' || ch == 'a' ? 0 : ch == 'C' || ch == 'c' ? 1 : ch == 'G' || ch == 'g' ? 2
                        : ch == 'T' || ch == 't' ? 3 : 4;
    }
    NODE_TRY(upload(s.reads, ri.data(), nReads, st));
    NODE_TRY(upload(s.nodeSym, sym.data(), nNodes, st));
    NODE_TRY(upload(s.nodeFirst, first.data(), nNodes, st));
    NODE_TRY(upload(s.chars, b->read_chars, nRuns, st));
    NODE_TRY(upload(s.counts, b->read_counts, nRuns, st));
    NODE_TRY(upload(s.w, b->weight, nTup, st));
    NODE_TRY(upload(s.x, b->x, nTup, st));
    NODE_TRY(upload(s.y, b->y, nTup, st));
    const bool estimate = b->repeat_log10 != nullptr && r->repeat_counts != nullptr;
    if (estimate) NODE_TRY(upload(s.log10, b->repeat_log10, 4 * M * M, st));
    NODE_TRY(s.bw.reserve(sizeof(double) * 5 * (size_t) std::max<int64_t>(nNodes, 1)));
    NODE_TRY(s.rcw.reserve(sizeof(double) * (size_t) M * (size_t) std::max<int64_t>(nNodes, 1)));
    NODE_TRY(s.count.reserve(sizeof(int32_t) * (size_t) (nNodes + 1)));
    NODE_TRY(s.cursor.reserve(sizeof(int32_t) * (size_t) std::max<int64_t>(nNodes, 1)));
    NODE_TRY(s.start.reserve(sizeof(int64_t) * (size_t) (nNodes + 1)));
    NODE_TRY(s.tupNode.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nTup, 1)));
    NODE_TRY(s.tupRead.reserve(sizeof(int32_t) * (size_t) std::max<int64_t>(nTup, 1)));
    NODE_TRY(s.slot.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nTup, 1)));
    NODE_TRY(s.rc.reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(nNodes, 1)));
    NODE_TRY(s.bad.reserve(sizeof(int)));
    const bool wantObs = r->obs_read || r->obs_offset || r->obs_weight;
    if (wantObs) {
        NODE_TRY(s.obsRead.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nTup, 1)));
        NODE_TRY(s.obsOffset.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nTup, 1)));
        NODE_TRY(s.obsWeight.reserve(sizeof(double) * (size_t) std::max<int64_t>(nTup, 1)));
    }
    NODE_CUDA(cudaMemsetAsync(s.bw.p, 0, sizeof(double) * 5 * (size_t) nNodes, st));
    NODE_CUDA(cudaMemsetAsync(s.rcw.p, 0, sizeof(double) * (size_t) M * (size_t) nNodes, st));
    NODE_CUDA(cudaMemsetAsync(s.count.p, 0, sizeof(int32_t) * (size_t) (nNodes + 1), st));
    NODE_CUDA(cudaMemsetAsync(s.cursor.p, 0, sizeof(int32_t) * (size_t) std::max<int64_t>(nNodes, 1), st));
    NODE_CUDA(cudaMemsetAsync(s.bad.p, 0, sizeof(int), st));

    if (nReads > 0) {
        scatterKernel<<<gridFor(nReads * 32, 256, e->smCount), 256, 0, st>>>(
            s.reads.as<ReadInfo>(), nReads, s.chars.as<char>(), s.counts.as<uint32_t>(), s.w.as<int32_t>(),
            s.x.as<int32_t>(), s.y.as<int32_t>(), M, s.bw.as<double>(), s.rcw.as<double>(), s.count.as<int32_t>(),
            s.tupNode.as<int64_t>(), s.tupRead.as<int32_t>(), s.bad.as<int>());
        NODE_CUDA(cudaGetLastError());
    }
    // segment starts: exclusive sum of the per-node counts (nNodes + 1 entries, the last the total)
    size_t tempBytes = 0;
    NODE_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tempBytes, s.count.as<int32_t>(), s.start.as<int64_t>(),
                                            (int) (nNodes + 1), st));
    NODE_TRY(s.cubTemp.reserve(std::max<size_t>(tempBytes, 16)));
    NODE_CUDA(cub::DeviceScan::ExclusiveSum(s.cubTemp.p, tempBytes, s.count.as<int32_t>(), s.start.as<int64_t>(),
                                            (int) (nNodes + 1), st));
    if (nTup > 0) {
        placeKernel<<<gridFor(nTup, 256, e->smCount), 256, 0, st>>>(nTup, s.tupNode.as<int64_t>(),
                                                                     s.start.as<int64_t>(), s.cursor.as<int32_t>(),
                                                                     s.slot.as<int64_t>());
        NODE_CUDA(cudaGetLastError());
    }
    if (nNodes > 0) {
        FinishArgs fa;
        fa.nNodes = nNodes;
        fa.start = s.start.as<int64_t>();
        fa.slotTuple = s.slot.as<int64_t>();
        fa.nodeSym = s.nodeSym.as<uint8_t>();
        fa.nodeFirst = s.nodeFirst.as<uint8_t>();
        fa.tupRead = s.tupRead.as<int32_t>();
        fa.w = s.w.as<int32_t>();
        fa.y = s.y.as<int32_t>();
        fa.reads = s.reads.as<ReadInfo>();
        fa.readCounts = s.counts.as<uint32_t>();
        fa.log10 = estimate ? s.log10.as<double>() : nullptr;
        fa.M = M;
        fa.repeatCount = s.rc.as<uint64_t>();
        fa.obsRead = wantObs ? s.obsRead.as<int64_t>() : nullptr;
        fa.obsOffset = wantObs ? s.obsOffset.as<int64_t>() : nullptr;
        fa.obsWeight = wantObs ? s.obsWeight.as<double>() : nullptr;
        finishKernel<<<gridFor(nNodes, 128, e->smCount), 128, 0, st>>>(fa);
        NODE_CUDA(cudaGetLastError());
    }
    int bad = 0;
    NODE_CUDA(cudaMemcpyAsync(&bad, s.bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    NODE_TRY(download(r->base_weights, s.bw, 5 * nNodes, st));
    NODE_TRY(download(r->repeat_weights, s.rcw, M * nNodes, st));
    NODE_TRY(download(r->obs_offsets, s.start, nNodes + 1, st));
    if (estimate) NODE_TRY(download(r->repeat_counts, s.rc, nNodes, st));
    if (wantObs) {
        NODE_TRY(download(r->obs_read, s.obsRead, nTup, st));
        NODE_TRY(download(r->obs_offset, s.obsOffset, nTup, st));
        NODE_TRY(download(r->obs_weight, s.obsWeight, nTup, st));
    }
    NODE_CUDA(cudaStreamSynchronize(st));
    if (bad) return mp_fail(MP_ERR_ARGUMENT, "mp_node_update: a match tuple lies outside its graph or read");
    return MP_OK;
}

void mp_node_scratch_free(mp_node_scratch *s) {
    delete s;
}
