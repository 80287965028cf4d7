// Complete-indel candidates of poa_augment on the GPU, for every read of a realignment at once.
//
//   poa_augment, inserts   impl/polisher.c:354-433
//   poa_augment, deletes   impl/polisher.c:435-522
//   helpers                impl/polisher.c:160-314 (hasInternalRepeat, getShift, getMaxCommonSuffix,
//                          rotateString)
//
// A complete insert is a stretch of gap-y tuples with the same x and consecutive y, flanked by
// matches (x, y-1) and (x+1, y+n+1) or by the read's ends; a complete delete is a stretch of gap-x
// tuples with the same y and consecutive x, flanked by matches or by the reference's ends. Each
// candidate gets the smallest weight of its stretch, is shifted left as far as its repeat unit
// allows and then back by its longest common suffix with the reference (inserts rotate by that
// suffix). The candidates of a read depend only on the chunk's reference, the read and the
// read's three tuple lists, so every read is independent; adding them to the graph keeps read
// order and stays on the host.
//
// B200 layout:
//   sort     the three lists of every read sorted by coordinates (segmented radix sorts of packed
//            (x+1, y+1) keys, as gap tuples reach -1; the weights travel as values) -- the order
//            poa_augment sorts them in;
//   index    per read run, its matches' place in the sorted match keys (the flanking-match test
//            is then one or two loads);
//   count    one warp per window of 32 consecutive tuples of a list (every window of every read
//            at once); the lane that holds the first tuple of a stretch counts the stretch's
//            candidates and insert runs;
//   scan     offsets of the windows' candidates and runs, in poa_augment's order (per read its
//            inserts' windows, then its deletes');
//   emit     the same walk writes each candidate (node, length, weight, read offset, its run
//            string for inserts); a warp scan gives every stretch its place in its window.
// The walk is integer work; the sorts move most bytes.
#include "../../include/mpgpu.h"
#include "mp_host.h"
#include "mp_internal.h"

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <vector>

namespace {

#define IND_TRY(expr)               \
    do {                            \
        mp_status _s = (expr);      \
        if (_s != MP_OK) return _s; \
    } while (0)
#define IND_CUDA(expr)                                                                              \
    do {                                                                                            \
        cudaError_t _e = (expr);                                                                    \
        if (_e != cudaSuccess) return mp_fail(MP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

// A run string viewed in place: runs [0, len) at (c, n).
struct View {
    const char *c;
    const uint32_t *n;
    int64_t len;
};

__device__ __forceinline__ bool hasInternalRepeat(View s, int64_t k, bool cmpRC) {
    if (s.len % k != 0) return false;
    for (int64_t i = k; i < s.len; i += k)
        for (int64_t j = 0; j < k; j++)
            if (s.c[j] != s.c[j + i] || (cmpRC && s.n[j] != s.n[j + i])) return false;
    return true;
}

__device__ __forceinline__ bool matchesRef(View ref, int64_t start, View s, int64_t len, bool cmpRC) {
    for (int64_t l = 0; l < len; l++)
        if (ref.c[start + l] != s.c[l] || (cmpRC && ref.n[start + l] != s.n[l])) return false;
    return true;
}

// getShift (impl/polisher.c:269-297): the leftmost start the indel s at refStart moves to.
__device__ int64_t getShift(View ref, int64_t refStart, View s, bool cmpRC) {
    int64_t minRepeat = 0;
    while (minRepeat++ < s.len)
        if (hasInternalRepeat(s, minRepeat, cmpRC)) break;
    for (int64_t k = refStart - minRepeat; k >= 0; k -= minRepeat) {
        if (!matchesRef(ref, k, s, minRepeat, cmpRC)) break;
        refStart = k;
    }
    if (s.len == 1 && cmpRC && refStart > 0 && ref.c[refStart - 1] == s.c[0]) refStart--;
    return refStart;
}

// getMaxCommonSuffix (impl/polisher.c:245-267) of a's first lenA runs and b.
__device__ int64_t maxCommonSuffix(View a, int64_t lenA, View b, bool cmpRC) {
    int64_t i = 0;
    while (lenA - i - 1 >= 0 && b.len - i - 1 >= 0) {
        if (a.c[lenA - 1 - i] != b.c[b.len - 1 - i] || (cmpRC && a.n[lenA - 1 - i] != b.n[b.len - 1 - i])) break;
        i++;
    }
    return i;
}

struct JobIn {
    int64_t refBase, refRuns;    // the job's reference runs in the reference arrays
    int64_t readBase, readRuns;  // its read's runs in the read arrays
};

// One window of the walk: 32 consecutive tuples of one list of one job.
struct Window {
    int32_t job, list;  // list 2: gap-y (inserts), 1: gap-x (deletes)
    int64_t base;       // its first tuple within the job's list
};

struct WalkArgs {
    int64_t nWin;
    const Window *win;
    const JobIn *jobs;
    const char *refC;
    const uint32_t *refN;
    const char *readC;
    const uint32_t *readN;
    const int64_t *off[3];       // per list: nJobs + 1 tuple offsets
    const uint64_t *key[3];      // sorted keys: matches (y, x), gap-x (y, x), gap-y (x, y)
    const int32_t *w[3];         // weights in key order (lists 1 and 2)
    const int32_t *mStart;       // per read run: its first match in the job's sorted matches
    const int32_t *mCount;       // per read run: its matches
    bool cmpRC;
    // count pass: per window
    int64_t *winCand, *winRuns;
    // emit pass
    const int64_t *winCandOff, *winRunOff;  // exclusive sums of the counts (nWin + 1)
    const int64_t *jobRunOff;               // per job: the first run of its inserts
    int64_t *pos, *len, *at, *offset;
    uint64_t *nonRle;
    double *weight;
    char *chars;
    uint64_t *counts;
};

// Sort key of a tuple: its major and minor coordinates, each plus one (gap tuples reach -1: an
// insert before the reference's first run, a delete before the read's first run).
__device__ __forceinline__ uint64_t packKey(int64_t major, int64_t minor) {
    return ((uint64_t) (major + 1) << 32) | (uint64_t) (minor + 1);
}
__device__ __forceinline__ int64_t keyMajor(uint64_t k) {
    return (int64_t) (k >> 32) - 1;
}
__device__ __forceinline__ int64_t keyMinor(uint64_t k) {
    return (int64_t) (k & 0xffffffffu) - 1;
}

// The match (x, y) of the read? Its matches at read run y are a few consecutive entries of its
// (y, x)-sorted match keys, found through the per-run index.
struct MatchIndex {
    const uint64_t *mk;
    const int32_t *start, *count;  // the read's runs
    int64_t runs;
    __device__ __forceinline__ bool has(int64_t x, int64_t y) const {
        if (x < 0 || y < 0 || y >= runs) return false;
        const int32_t s0 = start[y], n = count[y];
        for (int32_t q = s0; q < s0 + n; q++)
            if (keyMinor(mk[q]) == x) return true;
        return false;
    }
};

// Per read run: the first of its matches in the job's sorted match keys and their number.
__global__ void matchIndexKernel(int64_t nJobs, const JobIn *jobs, const int64_t *off0, const uint64_t *mk,
                                 int32_t *mStart, int32_t *mCount) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nWarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
    for (int64_t j = warp; j < nJobs; j += nWarps) {
        const int64_t b = off0[j], n = off0[j + 1] - off0[j];
        const int64_t rb = jobs[j].readBase;
        for (int64_t t = lane; t < n; t += 32) {
            const int64_t y = keyMajor(mk[b + t]);
            if (t == 0 || keyMajor(mk[b + t - 1]) != y) {
                int64_t e = t + 1;
                while (e < n && keyMajor(mk[b + e]) == y) e++;
                mStart[rb + y] = (int32_t) t;
                mCount[rb + y] = (int32_t) (e - t);
            }
        }
    }
}

// Inclusive warp sum.
__device__ __forceinline__ int64_t warpInclusive(int64_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// One window per warp. The list is cut into stretches (a tuple that continues the previous one
// -- the same major coordinate, the minor one more -- joins its stretch); the lane holding a
// stretch's first tuple enumerates the stretch's candidates, whose places follow from the
// window's offset and a warp scan. INS: gap-y tuples sorted by (x, y), complete inserts;
// otherwise gap-x tuples sorted by (y, x), complete deletes.
template <bool EMIT, bool INS>
__device__ void walkWindow(const WalkArgs &a, int64_t w, const Window &wd, int lane) {
    const int64_t j = wd.job;
    const JobIn jb = a.jobs[j];
    const View ref{a.refC + jb.refBase, a.refN + jb.refBase, jb.refRuns};
    const View read{a.readC + jb.readBase, a.readN + jb.readBase, jb.readRuns};
    const MatchIndex mi_{a.key[0] + a.off[0][j], a.mStart + jb.readBase, a.mCount + jb.readBase, jb.readRuns};
    const int L_ = INS ? 2 : 1;
    const uint64_t *key = a.key[L_] + a.off[L_][j];
    const int32_t *wt = a.w[L_] + a.off[L_][j];
    const int64_t n = a.off[L_][j + 1] - a.off[L_][j];
    const int64_t i = wd.base + lane;
    bool start = false;
    int64_t e = i, cnt = 0, runs = 0, ma = 0, mi = 0;
    if (i < n) {
        ma = keyMajor(key[i]);
        mi = keyMinor(key[i]);
        start = i == 0 || keyMajor(key[i - 1]) != ma || keyMinor(key[i - 1]) + 1 != mi;
        if (start) {
            e = i + 1;
            while (e < n && keyMajor(key[e]) == ma && keyMinor(key[e]) == mi + (e - i)) e++;
            for (int64_t k = i; k < e; k++) {
                if (INS) {
                    if (!mi_.has(ma, mi + k - i - 1) && mi + k - i - 1 > -1) continue;
                } else {
                    if (!mi_.has(mi + k - i - 1, ma) && mi + k - i - 1 > -1) continue;
                }
                for (int64_t l = k; l < e; l++) {
                    if (INS) {
                        if (!mi_.has(ma + 1, mi + l - i + 1) && mi + l - i + 1 < read.len) continue;
                        runs += l + 1 - k;
                    } else {
                        if (!mi_.has(mi + l - i + 1, ma + 1) && mi + l - i + 1 < ref.len) continue;
                    }
                    cnt++;
                }
            }
        }
    }
    const int64_t incC = warpInclusive(cnt, lane), incR = warpInclusive(runs, lane);
    if (!EMIT) {
        if (lane == 31) {
            a.winCand[w] = incC;
            a.winRuns[w] = incR;
        }
        return;
    }
    if (!start || cnt == 0) return;
    int64_t q = a.winCandOff[w] + incC - cnt;          // this stretch's first candidate
    int64_t rg = a.winRunOff[w] + incR - runs;         // its first run in the run arrays
    const int64_t r0 = a.jobRunOff[j];                 // the job's first run
    for (int64_t k = i; k < e; k++) {
        if (INS) {
            if (!mi_.has(ma, mi + k - i - 1) && mi + k - i - 1 > -1) continue;
        } else {
            if (!mi_.has(mi + k - i - 1, ma) && mi + k - i - 1 > -1) continue;
        }
        for (int64_t l = k; l < e; l++) {
            double wmin = (double) UINT_MAX;
            if (INS) {
                if (!mi_.has(ma + 1, mi + l - i + 1) && mi + l - i + 1 < read.len) continue;
                const int64_t y0 = mi + k - i, L = l + 1 - k;
                const View ins{read.c + y0, read.n + y0, L};
                for (int64_t m = k; m <= l; m++) wmin = wmin < (double) wt[m] ? wmin : (double) wt[m];
                int64_t p = getShift(ref, ma + 1, ins, a.cmpRC);
                const int64_t suf = maxCommonSuffix(ref, p, ins, a.cmpRC);
                uint64_t nonRle = 0;
                // rotated right by suf: run u of the output is run (u - suf) mod L of ins
                const int64_t sh = suf % L;
                for (int64_t u = 0; u < L; u++) {
                    const int64_t src = (u - sh + L) % L;
                    a.chars[rg + u] = ins.c[src];
                    a.counts[rg + u] = ins.n[src];
                    nonRle += ins.n[src];
                }
                if (suf > 0) p -= suf;
                a.pos[q] = p;
                a.len[q] = L;
                a.at[q] = rg - r0;
                a.nonRle[q] = nonRle;
                a.weight[q] = wmin;
                a.offset[q] = y0;
                rg += L;
            } else {
                if (!mi_.has(mi + l - i + 1, ma + 1) && mi + l - i + 1 < ref.len) continue;
                const int64_t L = l - k + 1;
                for (int64_t m = k; m <= l; m++) wmin = wmin < (double) wt[m] ? wmin : (double) wt[m];
                const int64_t p0 = mi + k - i;
                const View del{ref.c + p0, ref.n + p0, L};
                int64_t p = getShift(ref, p0, del, a.cmpRC);
                p -= maxCommonSuffix(ref, p, del, a.cmpRC);
                a.pos[q] = p;
                a.len[q] = L;
                a.at[q] = -1;
                a.nonRle[q] = 0;
                a.weight[q] = wmin;
                a.offset[q] = ma;
            }
            q++;
        }
    }
}

template <bool EMIT>
__global__ void walkKernel(WalkArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nWarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
    for (int64_t w = warp; w < a.nWin; w += nWarps) {
        const Window wd = a.win[w];
        if (wd.list == 2) walkWindow<EMIT, true>(a, w, wd, lane);
        else walkWindow<EMIT, false>(a, w, wd, lane);
    }
}

// Packed sort keys of one list: matches and gap-x (y, x), gap-y (x, y); a coordinate below -1
// is flagged.
__global__ void keyKernel(int64_t n, const int32_t *x, const int32_t *y, bool xMajor, uint64_t *key, int *bad) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t xi = x[t], yi = y[t];
        if (xi < -1 || yi < -1) {
            atomicOr(bad, 1);
            key[t] = 0;
            continue;
        }
        key[t] = xMajor ? packKey(xi, yi) : packKey(yi, xi);
    }
}

template <class T>
mp_status upload(DevBuf &d, const T *h, int64_t n, cudaStream_t s) {
    IND_TRY(d.reserve(sizeof(T) * (size_t) std::max<int64_t>(n, 1)));
    if (n > 0) IND_CUDA(cudaMemcpyAsync(d.p, h, sizeof(T) * (size_t) n, cudaMemcpyHostToDevice, s));
    return MP_OK;
}

int gridFor(int64_t work, int threads, int smCount) {
    const int64_t need = (work + threads - 1) / threads;
    return (int) std::max<int64_t>(1, std::min<int64_t>(need, (int64_t) smCount * 16));
}

}  // namespace

struct mp_indel_scratch {
    DevBuf jobs, refC, refN, readC, readN, off[3], w[3], x[3], y[3], keyIn[3], keyOut[3], wOut[3], cubTemp, bad;
    DevBuf win, mStart, mCount, winCand, winRuns, winCandOff, winRunOff, jobRunOff, pos, len, at, offset, nonRle,
        weight, chars, counts;
    PinBuf hPos, hLen, hAt, hOffset, hNonRle, hWeight, hChars, hCounts;  // the results, page-locked
    cudaStream_t stream = nullptr;  // its own stream (the node update may run beside it)
    ~mp_indel_scratch() {
        if (stream) cudaStreamDestroy(stream);
    }
};

void mp_indel_scratch_free(mp_indel_scratch *s) {
    delete s;
}

namespace mp {

mp_status deviceIndelCandidates(mp_engine *e, const IndelBatch &b, IndelOut &out) {
    static std::mutex lock;  // one call at a time per process (the engine's scratch is shared)
    std::lock_guard<std::mutex> guard(lock);
    IND_CUDA(cudaSetDevice(e->device));
    if (!e->indelScratch) e->indelScratch = new mp_indel_scratch();
    mp_indel_scratch &s = *e->indelScratch;
    if (!s.stream) IND_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    cudaStream_t st = s.stream;
    const int64_t nJ = b.nJobs;
    for (int k = 0; k < 3; k++)
        if (b.off[k][nJ] >= INT32_MAX || nJ >= INT32_MAX)
            return mp_fail(MP_ERR_ARGUMENT, "indel candidates: 2^31 or more tuples in one list");
    std::vector<JobIn> jobs((size_t) nJ);
    for (int64_t j = 0; j < nJ; j++) jobs[(size_t) j] = JobIn{b.refBase[j], b.refRuns[j], b.readBase[j], b.readRuns[j]};
    IND_TRY(upload(s.jobs, jobs.data(), nJ, st));
    IND_TRY(upload(s.refC, b.refChars, b.nRefRuns, st));
    IND_TRY(upload(s.refN, b.refCounts, b.nRefRuns, st));
    IND_TRY(upload(s.readC, b.readChars, b.nReadRuns, st));
    IND_TRY(upload(s.readN, b.readCounts, b.nReadRuns, st));
    IND_TRY(s.bad.reserve(sizeof(int)));
    IND_CUDA(cudaMemsetAsync(s.bad.p, 0, sizeof(int), st));
    for (int k = 0; k < 3; k++) {
        const int64_t n = b.off[k][nJ];
        IND_TRY(upload(s.off[k], b.off[k], nJ + 1, st));
        IND_TRY(upload(s.x[k], b.x[k], n, st));
        IND_TRY(upload(s.y[k], b.y[k], n, st));
        IND_TRY(s.keyIn[k].reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(n, 1)));
        IND_TRY(s.keyOut[k].reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(n, 1)));
        if (k > 0) {
            IND_TRY(upload(s.w[k], b.w[k], n, st));
            IND_TRY(s.wOut[k].reserve(sizeof(int32_t) * (size_t) std::max<int64_t>(n, 1)));
        }
        if (n > 0) {
            keyKernel<<<gridFor(n, 256, e->smCount), 256, 0, st>>>(n, s.x[k].as<int32_t>(), s.y[k].as<int32_t>(),
                                                                   k == 2, s.keyIn[k].as<uint64_t>(), s.bad.as<int>());
            IND_CUDA(cudaGetLastError());
            // the tuples of every job sorted by key (keys are distinct within a job's list)
            size_t tmp = 0;
            const int64_t *beg = s.off[k].as<int64_t>();
            if (k == 0) {
                IND_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp, s.keyIn[k].as<uint64_t>(),
                                                            s.keyOut[k].as<uint64_t>(), (int) n, (int) nJ, beg,
                                                            beg + 1, st));
                IND_TRY(s.cubTemp.reserve(std::max<size_t>(tmp, 16)));
                IND_CUDA(cub::DeviceSegmentedSort::SortKeys(s.cubTemp.p, tmp, s.keyIn[k].as<uint64_t>(),
                                                            s.keyOut[k].as<uint64_t>(), (int) n, (int) nJ, beg,
                                                            beg + 1, st));
            } else {
                IND_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, tmp, s.keyIn[k].as<uint64_t>(),
                                                             s.keyOut[k].as<uint64_t>(), s.w[k].as<int32_t>(),
                                                             s.wOut[k].as<int32_t>(), (int) n, (int) nJ, beg,
                                                             beg + 1, st));
                IND_TRY(s.cubTemp.reserve(std::max<size_t>(tmp, 16)));
                IND_CUDA(cub::DeviceSegmentedSort::SortPairs(s.cubTemp.p, tmp, s.keyIn[k].as<uint64_t>(),
                                                             s.keyOut[k].as<uint64_t>(), s.w[k].as<int32_t>(),
                                                             s.wOut[k].as<int32_t>(), (int) n, (int) nJ, beg,
                                                             beg + 1, st));
            }
        }
    }
    // windows: per job its inserts' windows, then its deletes' (poa_augment's order)
    std::vector<Window> win;
    std::vector<int64_t> winStart((size_t) nJ + 1, 0), winMid((size_t) std::max<int64_t>(nJ, 1), 0);
    for (int64_t j = 0; j < nJ; j++) {
        winStart[(size_t) j] = (int64_t) win.size();
        for (int k : {2, 1}) {
            if (k == 1) winMid[(size_t) j] = (int64_t) win.size();
            const int64_t n = b.off[k][j + 1] - b.off[k][j];
            for (int64_t base = 0; base < n; base += 32) win.push_back(Window{(int32_t) j, k, base});
        }
    }
    winStart[(size_t) nJ] = (int64_t) win.size();
    const int64_t nW = (int64_t) win.size();
    if (nW + 1 >= INT32_MAX) return mp_fail(MP_ERR_ARGUMENT, "indel candidates: too many tuple windows");
    IND_TRY(upload(s.win, win.data(), nW, st));
    // per read run: its matches in the job's sorted match keys
    IND_TRY(s.mStart.reserve(sizeof(int32_t) * (size_t) std::max<int64_t>(b.nReadRuns, 1)));
    IND_TRY(s.mCount.reserve(sizeof(int32_t) * (size_t) std::max<int64_t>(b.nReadRuns, 1)));
    if (b.nReadRuns > 0) IND_CUDA(cudaMemsetAsync(s.mCount.p, 0, sizeof(int32_t) * (size_t) b.nReadRuns, st));
    if (nJ > 0) {
        matchIndexKernel<<<gridFor(nJ * 32, 128, e->smCount), 128, 0, st>>>(
            nJ, s.jobs.as<JobIn>(), s.off[0].as<int64_t>(), s.keyOut[0].as<uint64_t>(), s.mStart.as<int32_t>(),
            s.mCount.as<int32_t>());
        IND_CUDA(cudaGetLastError());
    }
    WalkArgs a;
    memset(&a, 0, sizeof(a));
    a.nWin = nW;
    a.win = s.win.as<Window>();
    a.jobs = s.jobs.as<JobIn>();
    a.refC = s.refC.as<char>();
    a.refN = s.refN.as<uint32_t>();
    a.readC = s.readC.as<char>();
    a.readN = s.readN.as<uint32_t>();
    for (int k = 0; k < 3; k++) {
        a.off[k] = s.off[k].as<int64_t>();
        a.key[k] = s.keyOut[k].as<uint64_t>();
        a.w[k] = k > 0 ? s.wOut[k].as<int32_t>() : nullptr;
    }
    a.mStart = s.mStart.as<int32_t>();
    a.mCount = s.mCount.as<int32_t>();
    a.cmpRC = b.cmpRC;
    IND_TRY(s.winCand.reserve(sizeof(int64_t) * (size_t) (nW + 1)));
    IND_TRY(s.winRuns.reserve(sizeof(int64_t) * (size_t) (nW + 1)));
    IND_TRY(s.winCandOff.reserve(sizeof(int64_t) * (size_t) (nW + 1)));
    IND_TRY(s.winRunOff.reserve(sizeof(int64_t) * (size_t) (nW + 1)));
    IND_CUDA(cudaMemsetAsync(s.winCand.p, 0, sizeof(int64_t) * (size_t) (nW + 1), st));
    IND_CUDA(cudaMemsetAsync(s.winRuns.p, 0, sizeof(int64_t) * (size_t) (nW + 1), st));
    a.winCand = s.winCand.as<int64_t>();
    a.winRuns = s.winRuns.as<int64_t>();
    const int walkGrid = gridFor(nW * 32, 128, e->smCount);
    if (nW > 0) {
        walkKernel<false><<<walkGrid, 128, 0, st>>>(a);
        IND_CUDA(cudaGetLastError());
    }
    size_t tmp = 0;
    IND_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, s.winCand.as<int64_t>(), s.winCandOff.as<int64_t>(),
                                           (int) (nW + 1), st));
    IND_TRY(s.cubTemp.reserve(std::max<size_t>(tmp, 16)));
    IND_CUDA(cub::DeviceScan::ExclusiveSum(s.cubTemp.p, tmp, s.winCand.as<int64_t>(), s.winCandOff.as<int64_t>(),
                                           (int) (nW + 1), st));
    IND_CUDA(cub::DeviceScan::ExclusiveSum(s.cubTemp.p, tmp, s.winRuns.as<int64_t>(), s.winRunOff.as<int64_t>(),
                                           (int) (nW + 1), st));
    std::vector<int64_t> wc((size_t) nW + 1), wr((size_t) nW + 1);
    int bad = 0;
    IND_CUDA(cudaMemcpyAsync(wc.data(), s.winCandOff.p, sizeof(int64_t) * (size_t) (nW + 1), cudaMemcpyDeviceToHost,
                             st));
    IND_CUDA(cudaMemcpyAsync(wr.data(), s.winRunOff.p, sizeof(int64_t) * (size_t) (nW + 1), cudaMemcpyDeviceToHost,
                             st));
    IND_CUDA(cudaMemcpyAsync(&bad, s.bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    IND_CUDA(cudaStreamSynchronize(st));
    if (bad) return mp_fail(MP_ERR_ARGUMENT, "indel candidates: a tuple has a coordinate below -1");
    // per job: its candidates, its inserts and its runs
    out.candOff.assign((size_t) nJ + 1, 0);
    out.runOff.assign((size_t) nJ + 1, 0);
    out.nIns.assign((size_t) std::max<int64_t>(nJ, 1), 0);
    for (int64_t j = 0; j <= nJ; j++) {
        out.candOff[(size_t) j] = wc[(size_t) winStart[(size_t) j]];
        out.runOff[(size_t) j] = wr[(size_t) winStart[(size_t) j]];
        if (j < nJ) out.nIns[(size_t) j] = wc[(size_t) winMid[(size_t) j]] - wc[(size_t) winStart[(size_t) j]];
    }
    const int64_t nC = out.candOff[(size_t) nJ], nR = out.runOff[(size_t) nJ];
    IND_TRY(upload(s.jobRunOff, out.runOff.data(), nJ + 1, st));
    IND_TRY(s.pos.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.len.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.at.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.offset.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.nonRle.reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.weight.reserve(sizeof(double) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.chars.reserve((size_t) std::max<int64_t>(nR, 1)));
    IND_TRY(s.counts.reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(nR, 1)));
    a.winCandOff = s.winCandOff.as<int64_t>();
    a.winRunOff = s.winRunOff.as<int64_t>();
    a.jobRunOff = s.jobRunOff.as<int64_t>();
    a.pos = s.pos.as<int64_t>();
    a.len = s.len.as<int64_t>();
    a.at = s.at.as<int64_t>();
    a.offset = s.offset.as<int64_t>();
    a.nonRle = s.nonRle.as<uint64_t>();
    a.weight = s.weight.as<double>();
    a.chars = s.chars.as<char>();
    a.counts = s.counts.as<uint64_t>();
    if (nW > 0) {
        walkKernel<true><<<walkGrid, 128, 0, st>>>(a);
        IND_CUDA(cudaGetLastError());
    }
    IND_TRY(s.hPos.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.hLen.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.hAt.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.hOffset.reserve(sizeof(int64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.hNonRle.reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.hWeight.reserve(sizeof(double) * (size_t) std::max<int64_t>(nC, 1)));
    IND_TRY(s.hChars.reserve((size_t) std::max<int64_t>(nR, 1)));
    IND_TRY(s.hCounts.reserve(sizeof(uint64_t) * (size_t) std::max<int64_t>(nR, 1)));
    if (nC > 0) {
        IND_CUDA(cudaMemcpyAsync(s.hPos.p, s.pos.p, sizeof(int64_t) * nC, cudaMemcpyDeviceToHost, st));
        IND_CUDA(cudaMemcpyAsync(s.hLen.p, s.len.p, sizeof(int64_t) * nC, cudaMemcpyDeviceToHost, st));
        IND_CUDA(cudaMemcpyAsync(s.hAt.p, s.at.p, sizeof(int64_t) * nC, cudaMemcpyDeviceToHost, st));
        IND_CUDA(cudaMemcpyAsync(s.hOffset.p, s.offset.p, sizeof(int64_t) * nC, cudaMemcpyDeviceToHost, st));
        IND_CUDA(cudaMemcpyAsync(s.hNonRle.p, s.nonRle.p, sizeof(uint64_t) * nC, cudaMemcpyDeviceToHost, st));
        IND_CUDA(cudaMemcpyAsync(s.hWeight.p, s.weight.p, sizeof(double) * nC, cudaMemcpyDeviceToHost, st));
    }
    if (nR > 0) {
        IND_CUDA(cudaMemcpyAsync(s.hChars.p, s.chars.p, (size_t) nR, cudaMemcpyDeviceToHost, st));
        IND_CUDA(cudaMemcpyAsync(s.hCounts.p, s.counts.p, sizeof(uint64_t) * nR, cudaMemcpyDeviceToHost, st));
    }
    out.pos = static_cast<const int64_t *>(s.hPos.p);
    out.len = static_cast<const int64_t *>(s.hLen.p);
    out.at = static_cast<const int64_t *>(s.hAt.p);
    out.offset = static_cast<const int64_t *>(s.hOffset.p);
    out.nonRle = static_cast<const uint64_t *>(s.hNonRle.p);
    out.weight = static_cast<const double *>(s.hWeight.p);
    out.chars = static_cast<const char *>(s.hChars.p);
    out.counts = static_cast<const uint64_t *>(s.hCounts.p);
    IND_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

}  // namespace mp
