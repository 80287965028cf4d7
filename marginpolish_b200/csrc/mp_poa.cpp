// POA side of the realignment loop: the partial-order graph each chunk's reads are folded
// into, the consensus walk, the anchor alignments for the next iteration, the run-length
// estimate and the iterative driver (MarginPolish impl/polisher.c):
//
//   poa_getReferenceGraph  impl/polisher.c:118-132     Poa::fromReference
//   poa_augment            impl/polisher.c:316-534     augment
//   poa_getAnchorAlignments impl/polisher.c:536-592    anchorAlignments
//   crop + naming          impl/polisher.c:605-654     realignChunks (jobs of one GPU batch)
//   poa_realign            impl/polisher.c:656-703     realignChunks
//   score                  impl/polisher.c:709-758     score
//   poa_getConsensus       impl/polisher.c:1025-1275   consensus
//   repeat-count ML        impl/polisher.c:1556-1565, :1756-1865   estimateRepeatCounts
//   poa_realignIterative   impl/polisher.c:2034-2106   iterate (consensus mode)
//   poa_realignAll         impl/polisher.c:2109-2129   mp_poa_set_realign_all
//
// All chunks advance in lockstep: every realignment of an iteration, over the reads of
// every chunk still iterating, is one batched posterior pass on the GPU; the per-chunk
// graph work runs on host threads, one chunk per thread. Weights are sums of integer
// posteriors held in doubles, so they are exact; observation lists keep the reference's
// order (the posterior tuples arrive in the reference's order).
#include "../../include/mpgpu.h"
#include "mp_host.h"
#include "mp_internal.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#define MP_TRY(expr)                   \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

namespace {

// ---------------------------------------------------------------------------
// run-length strings
// ---------------------------------------------------------------------------

struct Rle {
    std::string c;                // one character per run
    std::vector<uint64_t> n;      // run lengths
    uint64_t nonRle = 0;          // expanded length
    int64_t length() const { return (int64_t) c.size(); }
    void push(char ch, uint64_t k) {
        c.push_back(ch);
        n.push_back(k);
        nonRle += k;
    }
    Rle sub(int64_t start, int64_t len) const {
        Rle r;
        subInto(r, start, len);
        return r;
    }
    // sub() into an existing string, reusing its storage
    void subInto(Rle &r, int64_t start, int64_t len) const {
        r.c.assign(c.begin() + start, c.begin() + start + len);
        r.n.assign(n.begin() + start, n.begin() + start + len);
        r.nonRle = 0;
        for (int64_t i = start; i < start + len; i++) r.nonRle += n[i];
    }
    bool operator==(const Rle &o) const { return nonRle == o.nonRle && c == o.c && n == o.n; }
};

// rleString_construct (impl/polisher.c:1357-1389): runs of equal characters.
Rle rleOf(const std::string &s) {
    Rle r;
    for (size_t i = 0; i < s.size();) {
        size_t j = i + 1;
        while (j < s.size() && s[j] == s[i]) j++;
        r.push(s[i], (uint64_t) (j - i));
        i = j;
    }
    return r;
}

// rleString_construct_no_rle: every character its own run of one.
Rle rleNoRle(const std::string &s) {
    Rle r;
    for (char ch : s) r.push(ch, 1);
    return r;
}

// The nucleotide alphabet (impl/stateMachine.c:25-59): A C G T, anything else N.
int symbolOf(char ch) {
    switch (ch) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 4;
    }
}

char charOf(int s) {
    return "ACGTN"[s < 0 || s > 4 ? 4 : s];
}

// The reference's approximate log-sum (impl/pairwiseAligner.c:279-299): a four-piece cubic
// of the difference (coefficients as the reference writes them, in single precision), the
// smaller term dropped from a difference of 7.5. The consensus walk makes its choices on
// sums of this function, so identical consensus needs the same function.
double lookupCubic(double x) {
    if (x <= 1.00f) return ((-0.009350833524763f * x + 0.130659527668286f) * x + 0.498799810682272f) * x + 0.693203116424741f;
    if (x <= 2.50f) return ((-0.014532321752540f * x + 0.139942324101744f) * x + 0.495635523139337f) * x + 0.692140569840976f;
    if (x <= 4.50f) return ((-0.004605031767994f * x + 0.063427417320019f) * x + 0.695956496475118f) * x + 0.514272634594009f;
    return ((-0.000458661602210f * x + 0.009695946122598f) * x + 0.930734667215156f) * x + 0.168037164329057f;
}

double logAddApprox(double x, double y) {
    const double kZero = -INFINITY, kUnder = 7.5;
    if (x < y) return (x == kZero || y - x >= kUnder) ? y : lookupCubic(y - x) + x;
    return (y == kZero || x - y >= kUnder) ? x : lookupCubic(x - y) + y;
}

// ---------------------------------------------------------------------------
// the graph
// ---------------------------------------------------------------------------

struct Obs {
    int64_t read, offset;
    double weight;
};

struct Insert {
    Rle s;
    double wF = 0.0, wR = 0.0;
    std::vector<Obs> obs;
    double weight() const { return wF + wR; }
};

struct Delete {
    int64_t len = 0;
    double wF = 0.0, wR = 0.0;
    std::vector<Obs> obs;
    double weight() const { return wF + wR; }
};

struct Node {
    char base = 'N';
    uint64_t rc = 1;
    double bw[5] = {0, 0, 0, 0, 0};
    std::vector<Insert> ins;
    std::vector<Delete> del;
};

struct Poa {
    uint64_t maxRC = 2;  // repeat counts are < maxRC
    std::vector<Node> nodes;
    Rle ref;
    // Run-length weights of every node, [node][maxRC], in one array.
    std::vector<double> rcw;
    // Match observations. Folding a read appends them (obsNode: the node of each); groupObs
    // then orders them by node, keeping append order within a node (the reference's
    // observation order), and node i's are obs[obsStart[i] .. obsStart[i+1]).
    std::vector<Obs> obs;
    std::vector<int32_t> obsNode;
    std::vector<int64_t> obsStart;
    // Run-length estimate of nodes 1.. computed on the GPU from the tuples the graph was built
    // from (mp_node_update); empty when the graph was built on the host only.
    std::vector<uint64_t> ml;

    double *rcwOf(int64_t i) { return rcw.data() + i * (int64_t) maxRC; }
    const double *rcwOf(int64_t i) const { return rcw.data() + i * (int64_t) maxRC; }
    const Obs *obsBegin(int64_t i) const { return obs.data() + obsStart[i]; }
    const Obs *obsEnd(int64_t i) const { return obs.data() + obsStart[i + 1]; }
    int64_t obsCount(int64_t i) const { return obsStart[i + 1] - obsStart[i]; }

    void groupObs() {
        const int64_t nN = (int64_t) nodes.size();
        obsStart.assign(nN + 1, 0);
        for (int32_t v : obsNode) obsStart[v + 1]++;
        for (int64_t i = 0; i < nN; i++) obsStart[i + 1] += obsStart[i];
        std::vector<Obs> sorted(obs.size());
        std::vector<int64_t> at(obsStart.begin(), obsStart.end() - 1);
        for (size_t k = 0; k < obs.size(); k++) sorted[(size_t) at[obsNode[k]]++] = obs[k];
        obs.swap(sorted);
        obsNode.clear();
        obsNode.shrink_to_fit();
    }

    // poa_getReferenceGraph: node 0 is an 'N' prefix, then one node per reference run.
    static Poa fromReference(const Rle &reference, uint64_t maxRC) {
        Poa p;
        p.maxRC = maxRC;
        p.ref = reference;
        p.nodes.resize(reference.length() + 1);
        for (int64_t i = 0; i <= reference.length(); i++) {
            Node &n = p.nodes[i];
            char b = i == 0 ? 'N' : (char) toupper((unsigned char) reference.c[i - 1]);
            n.base = charOf(symbolOf(b)) == 'N' ? 'N' : b;  // anything but ACGT becomes N
            n.rc = i == 0 ? 1 : reference.n[i - 1];
        }
        p.rcw.assign((size_t) (reference.length() + 1) * maxRC, 0.0);
        p.obsStart.assign((size_t) reference.length() + 2, 0);
        return p;
    }
};

struct Pair {  // (weight, x, y) of the aligner's lists
    int64_t w, x, y;
};

// ---------------------------------------------------------------------------
// poa_augment (impl/polisher.c:316-534) and its indel helpers (:160-314)
// ---------------------------------------------------------------------------

bool hasInternalRepeat(const Rle &s, int64_t k, bool cmpRC) {
    if (s.length() % k != 0) return false;
    for (int64_t i = k; i < s.length(); i += k)
        for (int64_t j = 0; j < k; j++)
            if (s.c[j] != s.c[j + i] || (cmpRC && s.n[j] != s.n[j + i])) return false;
    return true;
}

bool matchesRef(const Rle &ref, int64_t start, const Rle &s, int64_t len, bool cmpRC) {
    for (int64_t l = 0; l < len; l++)
        if (ref.c[start + l] != s.c[l] || (cmpRC && ref.n[start + l] != s.n[l])) return false;
    return true;
}

// Leftmost position an indel with sequence s at refStart can move to (getShift, :269-297).
int64_t getShift(const Rle &ref, int64_t refStart, const Rle &s, bool cmpRC) {
    int64_t minRepeat = 0;
    while (minRepeat++ < s.length())
        if (hasInternalRepeat(s, minRepeat, cmpRC)) break;
    for (int64_t k = refStart - minRepeat; k >= 0; k -= minRepeat) {
        if (!matchesRef(ref, k, s, minRepeat, cmpRC)) break;
        refStart = k;
    }
    if (s.length() == 1 && cmpRC && refStart > 0 && ref.c[refStart - 1] == s.c[0]) refStart--;
    return refStart;
}

int64_t maxCommonSuffix(const Rle &a, int64_t lenA, const Rle &b, bool cmpRC) {
    int64_t i = 0;
    while (lenA - i - 1 >= 0 && b.length() - i - 1 >= 0) {
        if (a.c[lenA - 1 - i] != b.c[b.length() - 1 - i] ||
            (cmpRC && a.n[lenA - 1 - i] != b.n[b.length() - 1 - i]))
            break;
        i++;
    }
    return i;
}

// Rotates right by k: run i moves to (i + k) mod L (in place).
void rotate(Rle &s, int64_t k) {
    const int64_t L = s.length();
    if (L == 0) return;
    const int64_t m = (L - k % L) % L;
    std::rotate(s.c.begin(), s.c.begin() + m, s.c.end());
    std::rotate(s.n.begin(), s.n.begin() + m, s.n.end());
}

// The match coordinates of one read, indexed by read position: the x values matched to read
// position y are xs[at[y] .. at[y+1]) (a few per position at the posterior threshold).
struct MatchSet {
    std::vector<int32_t> at;
    std::vector<int64_t> xs;
    void build(const std::vector<Pair> &matches, int64_t readLen) {
        at.assign((size_t) readLen + 2, 0);
        for (const Pair &m : matches)
            if (m.y >= 0 && m.y < readLen) at[(size_t) m.y + 1]++;
        for (int64_t y = 0; y <= readLen; y++) at[(size_t) y + 1] += at[(size_t) y];
        xs.resize(matches.size());
        std::vector<int32_t> fill(at.begin(), at.end() - 1);
        for (const Pair &m : matches)
            if (m.y >= 0 && m.y < readLen) xs[(size_t) fill[(size_t) m.y]++] = m.x;
    }
    bool has(int64_t x, int64_t y) const {
        if (y < 0 || y + 1 >= (int64_t) at.size()) return false;
        for (int32_t k = at[(size_t) y]; k < at[(size_t) y + 1]; k++)
            if (xs[(size_t) k] == x) return true;
        return false;
    }
};

// The complete indels of one read against a graph's reference, in the order poa_augment adds
// them to the graph (every insert, then every delete, each in enumeration order). They depend
// only on the reference string, so the candidates of all reads can be found in parallel; adding
// them to the graph (mergeRead) then runs read by read, which keeps the reference's order of
// the graph's insert / delete lists and of their observations.
struct IndelCands {
    std::vector<int64_t> pos;     // node the indel is attached to
    std::vector<int64_t> len;     // runs inserted / deleted
    std::vector<int64_t> at;      // inserts: first run in chars / counts
    std::vector<uint64_t> nonRle; // inserts: expanded length
    std::vector<double> w;
    std::vector<int64_t> offset;  // observation: read position
    std::string chars;
    std::vector<uint64_t> counts;
    int64_t nIns = 0;
    void clear() {
        pos.clear(), len.clear(), at.clear(), nonRle.clear(), w.clear(), offset.clear(), chars.clear(), counts.clear();
        nIns = 0;
    }
};

// The candidates of one read as the merge reads them: arrays owned by an IndelCands (host
// steps) or slices of the GPU pass's page-locked output (device steps).
struct IndelView {
    const int64_t *pos = nullptr, *len = nullptr, *at = nullptr, *offset = nullptr;
    const uint64_t *nonRle = nullptr;
    const double *w = nullptr;
    const char *chars = nullptr;
    const uint64_t *counts = nullptr;
    int64_t n = 0, nIns = 0;
    static IndelView of(const IndelCands &c) {
        IndelView v;
        v.pos = c.pos.data(), v.len = c.len.data(), v.at = c.at.data(), v.offset = c.offset.data();
        v.nonRle = c.nonRle.data(), v.w = c.w.data(), v.chars = c.chars.data(), v.counts = c.counts.data();
        v.n = (int64_t) c.pos.size(), v.nIns = c.nIns;
        return v;
    }
};

void indelCandidates(const Rle &ref, const Rle &read, const std::vector<Pair> &matches, std::vector<Pair> &inserts,
                     std::vector<Pair> &deletes, bool cmpRC, IndelCands &out) {
    // candidate indel sequences, reused across candidates and calls of this thread
    thread_local Rle scratchIns, scratchDel;
    thread_local MatchSet ms;
    out.clear();
    ms.build(matches, read.length());

    // complete inserts: same x, consecutive y, flanked by matches (or the read's ends)
    std::sort(inserts.begin(), inserts.end(), [](const Pair &a, const Pair &b) {
        return a.x != b.x ? a.x < b.x : a.y < b.y;
    });
    const int64_t nI = (int64_t) inserts.size();
    for (int64_t i = 0; i < nI;) {
        const Pair &st = inserts[i];
        int64_t j = i + 1;
        for (; j < nI; j++) {
            if (st.x != inserts[j].x || st.y + j - i != inserts[j].y) break;
        }
        for (int64_t k = i; k < j; k++) {
            if (!ms.has(st.x, st.y + k - i - 1) && st.y + k - i - 1 > -1) continue;
            for (int64_t l = k; l < j; l++) {
                if (!ms.has(st.x + 1, st.y + l - i + 1) && st.y + l - i + 1 < read.length()) continue;
                Rle &ins = scratchIns;
                read.subInto(ins, inserts[k].y, l + 1 - k);
                double w = (double) UINT_MAX;
                for (int64_t m = k; m <= l; m++) w = w < (double) inserts[m].w ? w : (double) inserts[m].w;
                int64_t pos = st.x + 1;
                pos = getShift(ref, pos, ins, cmpRC);
                const int64_t suf = maxCommonSuffix(ref, pos, ins, cmpRC);
                if (suf > 0) {
                    rotate(ins, suf);
                    pos -= suf;
                }
                out.pos.push_back(pos);
                out.len.push_back(ins.length());
                out.at.push_back((int64_t) out.counts.size());
                out.nonRle.push_back(ins.nonRle);
                out.w.push_back(w);
                out.offset.push_back(inserts[k].y);
                out.chars.append(ins.c);
                out.counts.insert(out.counts.end(), ins.n.begin(), ins.n.end());
            }
        }
        i = j;
    }
    out.nIns = (int64_t) out.pos.size();

    // complete deletes: same y, consecutive x, flanked by matches (or the reference's ends)
    std::sort(deletes.begin(), deletes.end(), [](const Pair &a, const Pair &b) {
        return a.y != b.y ? a.y < b.y : a.x < b.x;
    });
    const int64_t nD = (int64_t) deletes.size();
    for (int64_t i = 0; i < nD;) {
        const Pair &st = deletes[i];
        int64_t j = i + 1;
        for (; j < nD; j++) {
            if (st.y != deletes[j].y || st.x + j - i != deletes[j].x) break;
        }
        for (int64_t k = i; k < j; k++) {
            if (!ms.has(st.x + k - i - 1, st.y) && st.x + k - i - 1 > -1) continue;
            for (int64_t l = k; l < j; l++) {
                if (!ms.has(st.x + l - i + 1, st.y + 1) && st.x + l - i + 1 < ref.length()) continue;
                const int64_t len = l - k + 1;
                double w = (double) UINT_MAX;
                for (int64_t m = k; m <= l; m++) w = w < (double) deletes[m].w ? w : (double) deletes[m].w;
                int64_t pos = st.x + k - i;
                Rle &del = scratchDel;
                ref.subInto(del, pos, len);
                pos = getShift(ref, pos, del, cmpRC);
                pos -= maxCommonSuffix(ref, pos, del, cmpRC);
                out.pos.push_back(pos);
                out.len.push_back(len);
                out.at.push_back(-1);
                out.nonRle.push_back(0);
                out.w.push_back(w);
                out.offset.push_back(st.y);
            }
        }
        i = j;
    }
}

// Adds one read to the nodes [lo, hi) of the graph: match weights and observations (tuple
// order; the observations go to obs / obsNode for grouping), then its complete indels, each
// merged into an equal insert / delete of its node or appended as a new one. Every list a node
// holds grows in read order whichever range the node is merged in, so merging disjoint ranges
// on different threads gives the graph of one sequential merge.
void mergeRead(Poa &poa, const Rle &read, bool strand, int64_t readNo, int64_t nMatches, const int32_t *mw,
               const int32_t *mx, const int32_t *my, const IndelView &ic, int64_t lo, int64_t hi,
               std::vector<Obs> &obs, std::vector<int32_t> &obsNode) {
    for (int64_t t = 0; t < nMatches; t++) {
        const int64_t v = mx[t] + 1;
        if (v < lo || v >= hi) continue;
        Node &node = poa.nodes[v];
        const double w = (double) mw[t];
        node.bw[symbolOf(read.c[my[t]])] += w;
        uint64_t rc = read.n[my[t]];
        if (rc >= poa.maxRC) rc = poa.maxRC - 1;
        poa.rcwOf(v)[rc] += w;
        obs.push_back(Obs{readNo, my[t], w});
        obsNode.push_back((int32_t) v);
    }
    const int64_t n = ic.n;
    for (int64_t q = 0; q < n; q++) {
        if (ic.pos[q] < lo || ic.pos[q] >= hi) continue;
        Node &node = poa.nodes[ic.pos[q]];
        const double w = ic.w[q];
        if (q < ic.nIns) {
            const int64_t L = ic.len[q], at = ic.at[q];
            Insert *target = nullptr;
            for (Insert &e : node.ins) {
                if (e.s.nonRle == ic.nonRle[q] && e.s.length() == L &&
                    std::equal(e.s.c.begin(), e.s.c.end(), ic.chars + at) &&
                    std::equal(e.s.n.begin(), e.s.n.end(), ic.counts + at)) {
                    target = &e;
                    break;
                }
            }
            if (!target) {
                Insert e;
                e.s.c.assign(ic.chars + at, ic.chars + at + L);
                e.s.n.assign(ic.counts + at, ic.counts + at + L);
                e.s.nonRle = ic.nonRle[q];
                node.ins.push_back(std::move(e));
                target = &node.ins.back();
            }
            if (strand) target->wF += w; else target->wR += w;
            target->obs.push_back(Obs{readNo, ic.offset[q], w});
        } else {
            const int64_t len = ic.len[q];
            Delete *target = nullptr;
            for (Delete &e : node.del)
                if (e.len == len) {
                    target = &e;
                    break;
                }
            if (!target) {
                node.del.push_back(Delete{len, 0.0, 0.0, {}});
                target = &node.del.back();
            }
            if (strand) target->wF += w; else target->wR += w;
            target->obs.push_back(Obs{readNo, ic.offset[q], w});
        }
    }
}

// poa_augment (impl/polisher.c:316-534) of one read: its candidates, then the merge.
void augment(Poa &poa, const Rle &read, bool strand, int64_t readNo, const std::vector<Pair> &matches,
             std::vector<Pair> &inserts, std::vector<Pair> &deletes, bool cmpRC) {
    thread_local IndelCands ic;
    indelCandidates(poa.ref, read, matches, inserts, deletes, cmpRC, ic);
    std::vector<int32_t> w(matches.size()), x(matches.size()), y(matches.size());
    for (size_t t = 0; t < matches.size(); t++) {
        w[t] = (int32_t) matches[t].w;
        x[t] = (int32_t) matches[t].x;
        y[t] = (int32_t) matches[t].y;
    }
    mergeRead(poa, read, strand, readNo, (int64_t) matches.size(), w.data(), x.data(), y.data(), IndelView::of(ic), 0,
              (int64_t) poa.nodes.size(), poa.obs, poa.obsNode);
}

// ---------------------------------------------------------------------------
// weights and the stop rule (impl/polisher.c:709-758)
// ---------------------------------------------------------------------------

double score(const Poa &poa) {
    double match = 0.0, dis = 0.0, ins = 0.0, del = 0.0;
    for (const Node &n : poa.nodes) match += n.bw[symbolOf(n.base)];
    for (const Node &n : poa.nodes) {
        const int r = symbolOf(n.base);
        for (int j = 0; j < 5; j++)
            if (j != r) dis += n.bw[j];
    }
    for (const Node &n : poa.nodes)
        for (const Insert &e : n.ins) ins += e.weight() * (double) e.s.length();
    for (const Node &n : poa.nodes)
        for (const Delete &e : n.del) del += e.weight() * (double) e.len;
    return match - (del + ins + dis);
}

// ---------------------------------------------------------------------------
// poa_getConsensus (impl/polisher.c:1025-1275)
// ---------------------------------------------------------------------------

int64_t maxWeight(const double *w, int64_t n, int64_t refIndex, double penalty) {
    double best = 0.0;
    int64_t at = -1;
    for (int64_t j = 0; j < n; j++) {
        if (j != refIndex && w[j] >= best) {
            best = w[j];
            at = j;
        }
    }
    return w[refIndex] * penalty > best ? refIndex : at;
}

Rle consensus(const Poa &poa, std::vector<int64_t> &map, double penalty, bool useRle) {
    const int64_t nN = (int64_t) poa.nodes.size();
    const double kZero = -INFINITY;
    std::vector<double> outW(nN, 0.0), fwd(nN + 1, kZero), matchFwd(nN, 0.0);
    fwd[0] = 0.0;
    std::vector<std::vector<const Delete *>> incoming(nN + 1);
    for (int64_t i = 0; i < nN; i++)
        for (const Delete &d : poa.nodes[i].del) incoming[i + d.len + 1].push_back(&d);
    for (int64_t i = 0; i < nN; i++) {
        const Node &node = poa.nodes[i];
        double indel = 0.0;
        for (const Insert &e : node.ins) indel += e.weight();
        for (const Delete &e : node.del) indel += e.weight();
        double mw = 0.0;
        if (i == 0) {
            if (nN == 1) {
                mw = 1.0;
            } else {
                for (int64_t j = 1; j < nN; j++)
                    for (int k = 0; k < 5; k++) mw += poa.nodes[j].bw[k];
                mw /= (double) (nN - 1);
                mw -= indel;
            }
        } else {
            for (int k = 0; k < 5; k++) mw += node.bw[k];
            mw -= indel;
        }
        mw = mw <= 0.0 ? 0.0001 : mw;
        outW[i] = mw + indel;
        for (const Insert &e : node.ins) fwd[i + 1] = logAddApprox(fwd[i + 1], fwd[i] + std::log(e.weight() / outW[i]));
        for (const Delete &e : node.del)
            fwd[i + e.len + 1] = logAddApprox(fwd[i + e.len + 1], fwd[i] + std::log(e.weight() / outW[i]));
        matchFwd[i] = fwd[i] + std::log(mw / outW[i]);
        fwd[i + 1] = logAddApprox(fwd[i + 1], matchFwd[i]);
    }

    map.assign(nN - 1, -1);
    std::vector<std::string> pieces;
    int64_t running = 0;
    char prevBase = '-';
    for (int64_t i = nN; i > 0;) {
        if (i < nN) {
            const Node &node = poa.nodes[i];
            const char base = charOf((int) maxWeight(node.bw, 5, symbolOf(node.base), penalty));
            if (useRle) {
                int64_t rc = maxWeight(poa.rcwOf(i), (int64_t) poa.maxRC, (int64_t) node.rc, penalty);
                rc = rc == 0 ? 1 : rc;
                pieces.push_back(std::string((size_t) rc, base));
                if (prevBase != base) map[i - 1] = running++;
                prevBase = base;
            } else {
                pieces.push_back(std::string(1, base));
                map[i - 1] = running++;
            }
        }
        double maxIns = kZero, totIns = kZero;
        const Insert *bestIns = nullptr;
        const Node &pNode = poa.nodes[i - 1];
        for (const Insert &e : pNode.ins) {
            const double p = std::log(e.weight() / outW[i - 1]) + fwd[i - 1];
            if (p > maxIns) {
                maxIns = p;
                bestIns = &e;
            }
            totIns = logAddApprox(totIns, p);
        }
        double maxDel = kZero, totDel = kZero;
        const Delete *bestDel = nullptr;
        for (const Delete *e : incoming[i]) {
            const double p = std::log(e->weight() / outW[i - e->len - 1]) + fwd[i - e->len - 1];
            if (p > maxDel) {
                maxDel = p;
                bestDel = e;
            }
            totDel = logAddApprox(totDel, p);
        }
        if (matchFwd[i - 1] >= totDel && matchFwd[i - 1] >= totIns) {
            i--;
        } else if (totIns >= totDel) {
            std::string ex;
            for (int64_t r = 0; r < bestIns->s.length(); r++) ex.append((size_t) bestIns->s.n[r], bestIns->s.c[r]);
            pieces.push_back(ex);
            if (useRle) {
                const char last = bestIns->s.c[bestIns->s.length() - 1];
                running += bestIns->s.length() + (last != prevBase ? 0 : -1);
                prevBase = bestIns->s.c[0];
            } else {
                running += (int64_t) bestIns->s.nonRle;
            }
            i--;
        } else {
            i -= bestDel->len + 1;
        }
    }
    std::string expanded;
    for (auto it = pieces.rbegin(); it != pieces.rend(); ++it) expanded += *it;
    Rle out = useRle ? rleOf(expanded) : rleNoRle(expanded);
    for (int64_t i = 0; i < nN - 1; i++)
        if (map[i] != -1) map[i] = out.length() - 1 - map[i];
    return out;
}

// ---------------------------------------------------------------------------
// poa_getAnchorAlignments (impl/polisher.c:536-592)
// ---------------------------------------------------------------------------

struct Anchor {
    int64_t x, y, e;
};

std::vector<std::vector<Anchor>> anchorAlignments(const Poa &poa, const std::vector<int64_t> *map, int64_t nReads,
                                                  const std::vector<double> &probs) {
    std::vector<std::vector<Anchor>> out(nReads);
    for (int64_t i = 1; i < (int64_t) poa.nodes.size(); i++) {
        const int64_t ci = map ? (*map)[i - 1] : i - 1;
        if (ci == -1) continue;
        for (const Obs *op = poa.obsBegin(i); op != poa.obsEnd(i); ++op) {
            const Obs &o = *op;
            const double w = o.weight / (double) mp::kProbOne;
            if (!(w > probs[0])) continue;
            int64_t e = (int64_t) probs[1];
            for (size_t k = 2; k < probs.size(); k += 2) {
                if (w >= probs[k]) e = (int64_t) probs[k + 1];
                else break;
            }
            auto &l = out[o.read];
            if (l.empty() || (l.back().x < ci && l.back().y < o.offset)) l.push_back(Anchor{ci, o.offset, e});
        }
    }
    return out;
}

// ---------------------------------------------------------------------------
// run-length estimate (impl/polisher.c:1556-1565, :1756-1865)
// ---------------------------------------------------------------------------

struct RepeatModel {
    int64_t M = 0;                 // maximumRepeatLength
    std::vector<double> log10;     // [base row][underlying][observed]
    double logProb(int base, bool strand, int64_t observed, int64_t underlying) const {
        if (base == 4) base = 0;   // 'N' reads the A table
        const int64_t idx = (strand ? base : 3 - base) * M * M + underlying * M + observed;
        return log10[idx];
    }
};

uint64_t mlRepeatCount(const Poa &poa, int64_t i, const std::vector<Rle> &reads, const std::vector<uint8_t> &strand,
                       int64_t readBase, const RepeatModel &rm) {
    const Node &node = poa.nodes[i];
    const Obs *ob = poa.obsBegin(i), *oe = poa.obsEnd(i);
    const int base = symbolOf(node.base);
    int64_t lo = rm.M, hi = 0;
    for (const Obs *op = ob; op != oe; ++op) {
        const Obs &o = *op;
        const int64_t c = (int64_t) reads[readBase + o.read].n[o.offset];
        lo = c < lo ? c : lo;
        hi = c > hi ? c : hi;
    }
    if (hi >= rm.M) hi = rm.M - 1;
    if (lo == rm.M) return 0;
    double best = 0.0;
    int64_t bestAt = 0;
    for (int64_t u = lo; u <= hi; u++) {
        double lp = 0.0;
        for (const Obs *op = ob; op != oe; ++op) {
            const Obs &o = *op;
            int64_t c = (int64_t) reads[readBase + o.read].n[o.offset];
            c = c >= rm.M ? rm.M - 1 : c;
            lp += rm.logProb(base, strand[readBase + o.read] != 0, c, u) * o.weight;
        }
        lp /= (double) mp::kProbOne;
        if (u == lo || lp > best) {
            best = lp;
            bestAt = u - lo;
        }
    }
    return (uint64_t) (bestAt + lo);
}

void estimateRepeatCounts(Poa &poa, const std::vector<Rle> &reads, const std::vector<uint8_t> &strand, int64_t readBase,
                          const RepeatModel &rm) {
    poa.ref.nonRle = 0;
    const bool device = poa.ml.size() + 1 == poa.nodes.size();
    for (size_t i = 1; i < poa.nodes.size(); i++) {
        uint64_t rc = device ? poa.ml[i - 1] : mlRepeatCount(poa, (int64_t) i, reads, strand, readBase, rm);
        if (rc == 0) rc = 1;
        poa.ref.n[i - 1] = rc;
        poa.ref.nonRle += rc;
    }
}

// ---------------------------------------------------------------------------
// bubble graph of the polish step (poa_polish, impl/polisher.c:2008-2031, and
// bubbleGraph_constructFromPoa, impl/bubbleGraph.c:415-978)
// ---------------------------------------------------------------------------

struct ReadSub {  // bamChunkRead_getSubstring (impl/bubbleGraph.c:415-438)
    int64_t read;    // read index within the chunk
    int64_t start, length;
    double qual;     // mean quality of the substring's runs, -1 without qualities
};

struct Bubble {
    int64_t refStart, refLength;    // reference allele: runs [refStart, refStart + refLength)
    int64_t alleleFirst, nAlleles;  // into BubbleGraph::alleles
    int64_t readFirst, nReads;      // into BubbleGraph::reads, in the bubble's order
    int64_t supportFirst;           // nAlleles x nReads log-likelihoods, allele-major
};

struct BubbleGraph {
    std::vector<Bubble> bubbles;
    std::vector<Rle> alleles;
    std::vector<ReadSub> reads;
    std::vector<int32_t> scoreFrom;  // per read: the earlier read of the bubble with an equal
                                     // substring whose scores it shares (itself when scored)
    std::vector<float> supports;
    bool scored = false;
};

double totalWeight(const Node &n) {
    double t = 0.0;
    for (int k = 0; k < 5; k++) t += n.bw[k];
    return t;
}

// getCandidateWeights (impl/bubbleGraph.c:583-612): a fraction of the coverage averaged over a
// window of 100 nodes.
std::vector<double> candidateWeights(const Poa &poa, double fraction) {
    const int64_t n = (int64_t) poa.nodes.size(), window = 100;
    std::vector<double> w((size_t) n, 0.0);
    if (window >= n) {
        double avg = 0.0;
        for (int64_t j = 0; j < n; j++) avg += totalWeight(poa.nodes[j]);
        avg /= (double) n;
        std::fill(w.begin(), w.end(), avg * fraction);
        return w;
    }
    double total = 0.0;
    for (int64_t i = 0; i < n; i++) {
        total += totalWeight(poa.nodes[i]);
        if (i >= window) {
            total -= totalWeight(poa.nodes[i - window]);
            w[i - window / 2] = total / (double) window * fraction;
        }
    }
    for (int64_t i = 0; i < window / 2; i++) {
        w[i] = w[window / 2];
        w[n - 1 - i] = w[n - 1 - window / 2];
    }
    return w;
}

// getFilteredAnchorPositions (impl/bubbleGraph.c:614-695): nodes away from every candidate
// variant (a base or run length other than the node's, an insert, or a delete start, with more
// than the candidate weight; repeat counts need twice the weight) by columnAnchorTrim.
std::vector<uint8_t> anchorPositions(const Poa &poa, const std::vector<double> &cw, int64_t trim) {
    const int64_t n = (int64_t) poa.nodes.size();
    std::vector<uint8_t> variant((size_t) n, 0);
    for (int64_t i = 0; i < n; i++) {
        const Node &node = poa.nodes[i];
        const double w = cw[i];
        bool v = false;
        for (int k = 0; k < 5 && !v; k++) {  // hasCandidateSubstitution (:231-244)
            const char base = charOf(k);
            if ((node.bw[k] > w || node.base == base) && base != node.base) v = true;
        }
        const double *rcw = poa.rcwOf(i);
        for (uint64_t rc = 0; rc < poa.maxRC && !v; rc++)  // hasCandidateRepeatCountChange (:246-259)
            if ((rcw[rc] > 2.0 * w || node.rc == rc) && rc != node.rc) v = true;
        for (size_t k = 0; k < node.ins.size() && !v; k++)  // hasCandidateInsert (:274-280)
            if (node.ins[k].weight() > w) v = true;
        if (v) variant[i] = 1;
        // maxCandidateDeleteLength is declared bool (:295), so a candidate delete marks the node
        // and the one after it, whatever its length
        bool del = false;
        for (const Delete &d : node.del)
            if (d.weight() > w && d.len > 0) del = true;
        if (del) {
            variant[i] = 1;
            if (i + 1 < n) variant[i + 1] = 1;
        }
    }
    // expand (:647-664): [i - trim, i + trim) around every variant node
    std::vector<uint8_t> anchor((size_t) n, 1);
    for (int64_t i = 0; i < n; i++)
        if (variant[i])
            for (int64_t j = std::max<int64_t>(i - trim, 0); j < std::min<int64_t>(i + trim, n); j++) anchor[j] = 0;
    return anchor;
}

// sortBaseObservations (:448-468): each node's observations by read, then by descending
// weight. The reference sorts with qsort, a stable merge sort in glibc; the graph keeps the
// new order (the anchor alignments made from it afterwards read it).
void sortObservations(Poa &poa) {
    for (size_t i = 0; i + 1 < poa.obsStart.size(); i++)
        std::stable_sort(poa.obs.begin() + poa.obsStart[i], poa.obs.begin() + poa.obsStart[i + 1],
                         [](const Obs &a, const Obs &b) {
                             if (a.read != b.read) return a.read < b.read;
                             return a.weight > b.weight;
                         });
}

// getReadSubstrings (:508-581) for 0 < from < to < nodes: the runs of every read that has
// observations at both nodes (its first, heaviest one at each), from the one at `from` up to the
// one at `to`; then filterReadSubstrings (:491-506).
void readSubstrings(const Poa &poa, int64_t from, int64_t to, const std::vector<std::vector<uint8_t>> *quals,
                    int64_t readBase, int64_t keepAtLeast, double minQual, std::vector<ReadSub> &out) {
    out.clear();
    const Obs *f = poa.obsBegin(from), *fe = poa.obsEnd(from);
    const Obs *t = poa.obsBegin(to), *te = poa.obsEnd(to);
    auto skip = [](const Obs *p, const Obs *e, int64_t read) {
        while (p != e && p->read == read) ++p;
        return p;
    };
    while (f != fe && t != te) {
        if (f->read == t->read) {
            const int64_t len = t->offset - f->offset;
            if (len > 0) {
                ReadSub rs{f->read, f->offset, len, -1.0};
                if (quals) {
                    const std::vector<uint8_t> &q = (*quals)[readBase + f->read];
                    int64_t sum = 0;
                    for (int64_t k = 0; k < len; k++) sum += (int64_t) q[f->offset + k];
                    rs.qual = (double) sum / (double) len;
                }
                out.push_back(rs);
            }
            const int64_t r = f->read;
            f = skip(f + 1, fe, r);
            t = skip(t + 1, te, t->read);
        } else if (f->read < t->read) {
            f = skip(f + 1, fe, f->read);
        } else {
            t = skip(t + 1, te, t->read);
        }
    }
    std::stable_sort(out.begin(), out.end(), [](const ReadSub &a, const ReadSub &b) { return a.qual > b.qual; });
    while ((int64_t) out.size() > keepAtLeast) {
        const ReadSub &last = out.back();
        if (last.qual >= minQual || last.qual == -1.0) break;
        out.pop_back();
    }
}

bool sameRuns(const Rle &r, int64_t start, int64_t len, const Rle &s, int64_t sStart) {
    return std::equal(r.c.begin() + start, r.c.begin() + start + len, s.c.begin() + sStart) &&
           std::equal(r.n.begin() + start, r.n.begin() + start + len, s.n.begin() + sStart);
}

// bubbleGraph_constructFromPoa (:800-978) without the scores: the bubbles between consecutive
// anchor nodes that have read substrings and more than one allele. The alleles are the distinct
// read substrings (groupRleStrings keys on the run characters and run lengths, :722-742), in
// order of first appearance, with run lengths capped at 255 (getConsensusRleString, :744-765),
// then the reference allele if no read spells it.
BubbleGraph buildBubbles(Poa &poa, const std::vector<Rle> &reads, const std::vector<std::vector<uint8_t>> *quals,
                         int64_t readBase, double candidateFraction, int64_t trim, int64_t keepAtLeast, double minQual) {
    BubbleGraph g;
    const std::vector<double> cw = candidateWeights(poa, candidateFraction);
    sortObservations(poa);
    const std::vector<uint8_t> anchor = anchorPositions(poa, cw, trim);
    const int64_t n = (int64_t) poa.nodes.size();
    std::vector<ReadSub> subs;
    std::vector<int64_t> firstOf;  // per distinct allele: a substring that spells it
    int64_t pAnchor = 0;
    for (int64_t i = 1; i < n; i++) {
        if (!anchor[i]) continue;
        if (i - pAnchor != 1) {
            readSubstrings(poa, pAnchor + 1, i, quals, readBase, keepAtLeast, minQual, subs);
            if (!subs.empty()) {
                // distinct substrings in order of first appearance
                firstOf.clear();
                for (size_t k = 0; k < subs.size(); k++) {
                    const Rle &rk = reads[readBase + subs[k].read];
                    bool seen = false;
                    for (int64_t f : firstOf) {
                        const ReadSub &o = subs[(size_t) f];
                        if (o.length == subs[k].length &&
                            sameRuns(rk, subs[k].start, subs[k].length, reads[readBase + o.read], o.start)) {
                            seen = true;
                            break;
                        }
                    }
                    if (!seen) firstOf.push_back((int64_t) k);
                }
                const int64_t refLen = i - 1 - pAnchor;
                const size_t a0 = g.alleles.size();
                bool seenRef = false;
                for (int64_t f : firstOf) {
                    const ReadSub &o = subs[(size_t) f];
                    const Rle &ro = reads[readBase + o.read];
                    Rle a;
                    for (int64_t k = 0; k < o.length; k++) {
                        const uint64_t c = ro.n[o.start + k];
                        a.push(ro.c[o.start + k], c == 0 ? 1 : (c > 255 ? 255 : c));
                    }
                    if (a.length() == refLen && sameRuns(poa.ref, pAnchor, refLen, a, 0)) seenRef = true;
                    g.alleles.push_back(std::move(a));
                }
                if (!seenRef) g.alleles.push_back(poa.ref.sub(pAnchor, refLen));
                const int64_t nAlleles = (int64_t) (g.alleles.size() - a0);
                if (nAlleles > 1) {
                    Bubble b;
                    b.refStart = pAnchor;
                    b.refLength = refLen;
                    b.alleleFirst = (int64_t) a0;
                    b.nAlleles = nAlleles;
                    b.readFirst = (int64_t) g.reads.size();
                    b.nReads = (int64_t) subs.size();
                    b.supportFirst = 0;
                    // the bubble takes the substrings from the end of the list (stList_pop)
                    for (size_t k = subs.size(); k-- > 0;) g.reads.push_back(subs[k]);
                    // the score cache (:905-951) keys on the substring's runs; the strand is
                    // not part of the key
                    for (int64_t k = 0; k < b.nReads; k++) {
                        const ReadSub &rk = g.reads[(size_t) (b.readFirst + k)];
                        int32_t from = (int32_t) k;
                        for (int64_t q = 0; q < k; q++) {
                            const ReadSub &rq = g.reads[(size_t) (b.readFirst + q)];
                            if (g.scoreFrom[(size_t) (b.readFirst + q)] == (int32_t) q && rq.length == rk.length &&
                                sameRuns(reads[readBase + rk.read], rk.start, rk.length, reads[readBase + rq.read],
                                         rq.start)) {
                                from = (int32_t) q;
                                break;
                            }
                        }
                        g.scoreFrom.push_back(from);
                    }
                    g.bubbles.push_back(b);
                } else {
                    g.alleles.resize(a0);
                }
            }
        }
        pAnchor = i;
    }
    int64_t at = 0;
    for (Bubble &b : g.bubbles) {
        b.supportFirst = at;
        at += b.nAlleles * b.nReads;
    }
    g.supports.assign((size_t) at, 0.0f);
    return g;
}

// bubbleGraph_getConsensusPath (:52-59): per bubble, the allele with the largest summed support
// (reads in the bubble's order; the first of equal sums).
std::vector<int64_t> consensusPath(const BubbleGraph &g) {
    std::vector<int64_t> path(g.bubbles.size(), 0);
    for (size_t i = 0; i < g.bubbles.size(); i++) {
        const Bubble &b = g.bubbles[i];
        double best = 0.0;
        for (int64_t j = 0; j < b.nAlleles; j++) {
            double ll = 0.0;
            for (int64_t k = 0; k < b.nReads; k++) ll += (double) g.supports[(size_t) (b.supportFirst + j * b.nReads + k)];
            if (j == 0 || ll > best) {
                best = ll;
                path[i] = j;
            }
        }
    }
    return path;
}

// bubbleGraph_getConsensusString (:61-177): the reference between bubbles and the chosen allele
// of every bubble, joined and run-length encoded again (runs meeting at a seam merge), and the
// map from reference runs to the new string's runs.
Rle bubbleConsensus(const Poa &poa, const BubbleGraph &g, const std::vector<int64_t> &path, bool useRle,
                    std::vector<int64_t> &map) {
    const Rle &ref = poa.ref;
    const int64_t refLen = ref.length();
    map.assign((size_t) refLen, -1);
    Rle out;
    auto append = [&](const Rle &s, int64_t start, int64_t len) {
        for (int64_t k = start; k < start + len; k++) {
            if (useRle) {
                if (out.length() > 0 && out.c.back() == s.c[k]) {
                    out.n.back() += s.n[k];
                    out.nonRle += s.n[k];
                } else {
                    out.push(s.c[k], s.n[k]);
                }
            } else {
                for (uint64_t r = 0; r < s.n[k]; r++) out.push(s.c[k], 1);
            }
        }
    };
    char previous = '-';
    int64_t j = 0, k = 0;
    for (size_t i = 0; i < g.bubbles.size(); i++) {
        const Bubble &b = g.bubbles[i];
        if (k < b.refStart) {
            append(ref, k, b.refStart - k);
            const char first = ref.c[k], last = ref.c[b.refStart - 1];
            if (useRle && first == previous) k++;
            while (k < b.refStart) map[(size_t) k++] = j++;
            previous = last;
        }
        const Rle &allele = g.alleles[(size_t) (b.alleleFirst + path[i])];
        append(allele, 0, allele.length());
        if (allele.length() == b.refLength && sameRuns(ref, b.refStart, b.refLength, allele, 0)) {  // rleString_eq
            if (useRle && allele.c[0] == previous) k++;
            while (k < b.refStart + b.refLength) map[(size_t) k++] = j++;
        } else {
            k += b.refLength;
            j += allele.length() + ((useRle && allele.c[0] == previous) ? -1 : 0);
        }
        previous = allele.c[allele.length() - 1];
    }
    if (k < refLen) {
        append(ref, k, refLen - k);
        if (useRle && ref.c[k] == previous) k++;
        while (k < refLen) map[(size_t) k++] = j++;
    }
    return out;
}

// Runs f(c) for every chunk index in `chunks` on up to `threads` host threads.
template <class F>
void forChunks(const std::vector<int64_t> &chunks, F f) {
    const unsigned nT = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(),
                                                        (unsigned) std::max<size_t>(chunks.size(), 1)));
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k = next++; k < chunks.size(); k = next++) f(chunks[k]);
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nT; t++) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
}

}  // namespace

// ---------------------------------------------------------------------------
// the chunk set behind the C ABI
// ---------------------------------------------------------------------------

// Steps of the loop whose wall time a set accumulates (mp_poa_set_phase_seconds).
enum {
    kPhaseJobs,        // job arrays of a realignment (crop, symbols, anchors)
    kPhaseDevice,      // the posterior pass on the GPU (upload, kernels, compaction)
    kPhaseFetch,       // tuples into page-locked host arrays
    kPhaseCandidates,  // complete-indel candidates of every read (host threads)
    kPhaseMerge,       // reads folded into the chunks' graphs in read order
    kPhaseConsensus,   // consensus walk and anchor alignments of an iteration
    kPhaseRepeat,      // run-length estimate and score of the new graphs
    kPhaseBubbles,     // bubble graphs and their scores (polish mode)
    kPhaseGroup,       // observation lists grouped by node after the merge
    kPhaseJoin,        // waiting for the GPU's run-length estimate after the merge
    kPhaseCount
};

// Adds the wall time of its scope to one phase counter.
struct PhaseTimer {
    double &acc;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    explicit PhaseTimer(double &a) : acc(a) {}
    ~PhaseTimer() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

struct mp_poa_set {
    mp_engine *e = nullptr;
    const mp_model *m = nullptr;
    mp_params p{};
    double penalty = 0.5;
    bool cmpRC = true, useRle = true;
    std::vector<double> anchorProbs;
    int64_t minIter = 0, maxIter = 0;
    RepeatModel rm;
    int64_t nChunks = 0;
    std::vector<Rle> drafts;                 // per chunk: the draft the set was created with
    std::vector<int64_t> chunkReads;         // n_chunks+1
    std::vector<Rle> reads;
    std::vector<uint8_t> strand;
    std::vector<std::vector<Anchor>> initialAnchors;  // per read (empty list when none given)
    bool haveAnchors = false;
    std::vector<Poa> poas;                   // per chunk (after a realignment)
    std::vector<int64_t> iterations;         // per chunk: iterations run by the last iterate
    // polish mode (poa_polish)
    int64_t minPolish = 0, maxPolish = 0;
    double candidateFraction = 0.18;
    int64_t anchorTrim = 5, keepAtLeast = 15;
    double minQual = 10.0;
    std::vector<std::vector<uint8_t>> quals;  // per read, per run (empty when none given)
    std::vector<BubbleGraph> bubbles;        // per chunk: the last graph mp_poa_set_build_bubbles made
    mp_device_batch *db = nullptr;
    // Wall seconds spent in each step of the loop since the set was created (kPhase*).
    double phase[kPhaseCount] = {};
    // Steps of a realignment that run on the GPU instead of the host threads
    // (mp_poa_set_device_steps; both forms build the same graphs).
    int32_t deviceSteps = MP_POA_DEVICE_RUN_LENGTHS | MP_POA_DEVICE_INDELS;
    // symbols and anchors of the last realignment's jobs (reused between realignments)
    std::vector<uint16_t> jobX, jobY;
    std::vector<int32_t> jobAnchors;
    // every read's runs in one array each (the device-side steps' input)
    std::vector<int64_t> flatReadOff;
    std::string flatReadChars;
    std::vector<uint32_t> flatReadCounts;
    // Graphs the loop has replaced or rejected. The next realignment frees them on a thread of
    // their own while its posterior pass runs on the GPU (the host is idle then; freeing them
    // beside the read merge would contend with its allocations).
    std::vector<Poa> trash;
    std::thread reaper;
    void reapStart() {
        reapJoin();
        if (trash.empty()) return;
        reaper = std::thread([g = std::move(trash)]() mutable { std::vector<Poa>().swap(g); });
        trash.clear();
    }
    void reapJoin() {
        if (reaper.joinable()) reaper.join();
    }
    ~mp_poa_set() {
        reapJoin();
        mp_device_batch_destroy(db);
    }
};

namespace {

// The run-length estimate (impl/polisher.c:1556-1565) of the graphs realignChunks builds for
// `chunks`, on the GPU from the realignment's match tuples (jobs of the listed chunks in order,
// tuples of job j at [off[j], off[j+1])). Every chunk of the set is a graph of the batch; the
// unlisted ones have no tuples. ml receives every node's estimate, chunk c's nodes starting at
// nodeBase[c].
mp_status deviceRepeatCounts(mp_poa_set *s, const std::vector<int64_t> &chunks, const std::vector<Rle> &refs,
                             const std::vector<int64_t> &off, const int32_t *w, const int32_t *x, const int32_t *y,
                             std::vector<uint64_t> &ml, std::vector<int64_t> &nodeBase) {
    const int64_t nC = s->nChunks, nReads = (int64_t) s->reads.size();
    std::vector<uint8_t> listed((size_t) nC, 0);
    for (int64_t c : chunks) listed[(size_t) c] = 1;
    nodeBase.assign((size_t) nC + 1, 0);
    std::string bases;
    for (int64_t c = 0; c < nC; c++) {
        bases.push_back('N');
        if (listed[(size_t) c]) bases.append(refs[c].c);
        nodeBase[(size_t) c + 1] = (int64_t) bases.size();
    }
    // match offsets per read of the set: the listed chunks' jobs are their reads, in order
    std::vector<int64_t> mOff((size_t) nReads + 1, 0);
    int64_t j = 0, at = 0;
    for (int64_t c = 0; c < nC; c++)
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++) {
            if (listed[(size_t) c]) at = off[(size_t) j++ + 1];
            mOff[(size_t) r + 1] = at;
        }
    mp_node_batch b;
    memset(&b, 0, sizeof(b));
    b.n_chunks = nC;
    b.node_offsets = nodeBase.data();
    b.node_bases = bases.data();
    b.chunk_reads = s->chunkReads.data();
    b.read_offsets = s->flatReadOff.data();
    b.read_chars = s->flatReadChars.data();
    b.read_counts = s->flatReadCounts.data();
    b.strand = s->strand.data();
    b.match_offsets = mOff.data();
    b.weight = w;
    b.x = x;
    b.y = y;
    b.max_repeat = s->rm.M;
    b.repeat_log10 = s->rm.log10.data();
    ml.assign(bases.size(), 0);
    mp_node_result r;
    memset(&r, 0, sizeof(r));
    r.repeat_counts = ml.data();
    return mp_node_update(s->e, &b, &r);
}

// poa_realign (impl/polisher.c:656-703) for the given chunks, each against `refs[c]` with
// per-read anchors (NULL: align without anchors): one GPU batch for every read, then each
// chunk's reads are folded into a fresh graph in read order.
mp_status realignChunks(mp_poa_set *s, const std::vector<int64_t> &chunks, const std::vector<Rle> &refs,
                        const std::vector<std::vector<Anchor>> *anchors, std::vector<Poa> &out) {
    if (!s->e || !s->m) return mp_fail(MP_ERR_STATE, "mp_poa: realignment needs an engine and a model");
    // the engine's page-locked tuple arrays are this realignment's until it returns
    std::lock_guard<std::mutex> tuplesGuard(s->e->poaLock);
    // symbol repeat counts are clamped below the repeat table's dimension on the cropping path
    // (impl/polisher.c:634-635) and one lower on the path without anchors (:676-679)
    const uint64_t maxRC = s->useRle ? (uint64_t) s->rm.M : 2;
    const uint32_t maxExcl = (uint32_t) (anchors ? maxRC : maxRC - 1);
    const bool rle = s->m->host[0].runLength != 0;
    auto symbols = [&](const Rle &r, uint16_t *dst) {
        for (int64_t i = 0; i < r.length(); i++) {
            const uint16_t b = (uint16_t) symbolOf(r.c[i]);
            uint64_t cnt = r.n[i];
            cnt = cnt > maxExcl - 1 ? maxExcl - 1 : cnt;
            dst[i] = rle ? (uint16_t) ((cnt << 8) | b) : b;
        }
    };
    // jobs: one per read of the listed chunks, with the reference crop (impl/polisher.c:613-628).
    // Offsets first (chunk order, reads in order), then every chunk's arrays filled in parallel.
    auto tJobs = std::chrono::steady_clock::now();
    std::vector<int64_t> refStart(s->nChunks, 0), firstJobOf(s->nChunks, 0);
    std::vector<int64_t> yo{0}, ao{0};
    int64_t nx = 0;
    for (int64_t c : chunks) {
        refStart[c] = nx;
        nx += refs[c].length();
        firstJobOf[c] = (int64_t) yo.size() - 1;
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++) {
            yo.push_back(yo.back() + s->reads[r].length());
            ao.push_back(ao.back() + (anchors ? (int64_t) (*anchors)[r].size() : 0));
        }
    }
    const int64_t nJobs = (int64_t) yo.size() - 1;
    // the symbol and anchor arrays are the set's, kept between realignments (every entry is
    // written below), so that later realignments reuse memory already mapped
    std::vector<uint16_t> &xs = s->jobX, &ys = s->jobY;
    std::vector<int32_t> &an = s->jobAnchors;
    xs.resize((size_t) nx);
    ys.resize((size_t) yo.back());
    an.resize((size_t) (3 * ao.back()));
    std::vector<int64_t> xb((size_t) nJobs), xe((size_t) nJobs), shift((size_t) nJobs);
    std::vector<uint8_t> st((size_t) nJobs);
    forChunks(chunks, [&](int64_t c) {
        const int64_t L = refs[c].length();
        symbols(refs[c], xs.data() + refStart[c]);
        int64_t j = firstJobOf[c];
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++, j++) {
            const Rle &read = s->reads[r];
            int64_t first = 0, end = L;
            const std::vector<Anchor> *ra = anchors ? &(*anchors)[r] : nullptr;
            if (ra && !ra->empty()) {
                first = ra->front().x - ra->front().y;
                first = first < 0 ? 0 : first;
                end = 1 + ra->back().x + (read.length() - ra->back().y);
                end = end > L ? L : end;
            }
            xb[(size_t) j] = refStart[c] + first;
            xe[(size_t) j] = refStart[c] + end;
            shift[(size_t) j] = first;
            symbols(read, ys.data() + yo[(size_t) j]);
            if (ra) {
                int32_t *dst = an.data() + 3 * ao[(size_t) j];
                for (const Anchor &a : *ra) {
                    *dst++ = (int32_t) (a.x - first);
                    *dst++ = (int32_t) a.y;
                    *dst++ = (int32_t) a.e;
                }
            }
            st[(size_t) j] = s->strand[r];
        }
    });
    std::vector<int64_t> offs[3];
    const int32_t *w[3] = {nullptr, nullptr, nullptr}, *x[3] = {nullptr, nullptr, nullptr},
                  *y[3] = {nullptr, nullptr, nullptr};
    s->phase[kPhaseJobs] += std::chrono::duration<double>(std::chrono::steady_clock::now() - tJobs).count();
    s->reapStart();  // earlier graphs are freed while the GPU works
    if (nJobs > 0) {
        PhaseTimer tDev(s->phase[kPhaseDevice]);
        mp_batch b;
        memset(&b, 0, sizeof(b));
        b.n_jobs = nJobs;
        b.x_begin = xb.data();
        b.x_end = xe.data();
        b.x_symbols_length = (int64_t) xs.size();
        uint16_t dummy = 0;
        int32_t dummyA[3] = {0, 0, 0};
        b.x_symbols = xs.empty() ? &dummy : xs.data();
        b.y_offsets = yo.data();
        b.y_symbols = ys.empty() ? &dummy : ys.data();
        b.anchor_offsets = ao.data();
        b.anchors = an.empty() ? dummyA : an.data();
        b.strand = st.data();
        b.x_shift = shift.data();
        mp_status rc = s->db ? mp_device_batch_reset(s->e, s->db, &s->p, &b)
                             : mp_device_batch_create(s->e, s->m, &s->p, &b, &s->db);
        if (rc != MP_OK) return rc;
        rc = mp_device_batch_run(s->e, s->db, nullptr);
        if (rc != MP_OK) return rc;
    }
    if (nJobs > 0) {
        PhaseTimer tFetch(s->phase[kPhaseFetch]);
        mp_status rc;
        int64_t totals[3];
        rc = mp_device_batch_counts(s->db, totals);
        if (rc != MP_OK) return rc;
        mp_output o;
        memset(&o, 0, sizeof(o));
        for (int k = 0; k < 3; k++) {
            offs[k].assign(nJobs + 1, 0);
            // the list's w, x and y arrays, back to back in the engine's page-locked buffer (the
            // copies run by DMA); the buffer grows by a quarter over the need
            const size_t need = (size_t) std::max<int64_t>(totals[k], 1);
            PinBuf &pb = s->e->poaTuples[k];
            rc = pb.reserve(3 * sizeof(int32_t) * need);
            if (rc != MP_OK) return rc;
            const size_t cap = pb.bytes / (3 * sizeof(int32_t));
            int32_t *base = static_cast<int32_t *>(pb.p);
            w[k] = base;
            x[k] = base + cap;
            y[k] = base + 2 * cap;
            o.offsets[k] = offs[k].data();
            o.weight[k] = base;
            o.x[k] = base + cap;
            o.y[k] = base + 2 * cap;
        }
        rc = mp_device_batch_fetch_into(s->e, s->db, &o);
        if (rc != MP_OK) return rc;
    }
    s->reapJoin();
    // The run-length estimate of the new graphs runs on the GPU (mp_node_update, from the same
    // match tuples) while the host threads fold the reads into the graphs.
    std::vector<uint64_t> ml;
    std::vector<int64_t> nodeBase;
    mp_status mlStatus = MP_OK;
    std::string mlError;  // the worker thread's error message (messages are per thread)
    std::thread mlThread;
    if (s->useRle && nJobs > 0 && (s->deviceSteps & MP_POA_DEVICE_RUN_LENGTHS)) {
        mlThread = std::thread([&]() {
            mlStatus = deviceRepeatCounts(s, chunks, refs, offs[0], w[0], x[0], y[0], ml, nodeBase);
            if (mlStatus != MP_OK) mlError = mp_last_error();
        });
    }
    // fold each chunk's reads into its graph (chunks in parallel, reads in order)
    std::vector<int64_t> firstJob(s->nChunks, 0);
    {
        int64_t j = 0;
        for (int64_t c : chunks) {
            firstJob[c] = j;
            j += s->chunkReads[c + 1] - s->chunkReads[c];
        }
    }
    // Candidates first: every read of every listed chunk in parallel (they depend only on the
    // chunk's reference). Gap-x tuples (consuming the reference) are deletes, gap-y inserts
    // (impl/polisher.c:638-640).
    std::vector<int64_t> jobIdx((size_t) nJobs), jobChunk((size_t) nJobs), jobRead((size_t) nJobs);
    for (int64_t c : chunks)
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++) {
            const int64_t j = firstJob[c] + (r - s->chunkReads[c]);
            jobIdx[(size_t) j] = j;
            jobChunk[(size_t) j] = c;
            jobRead[(size_t) j] = r;
        }
    std::vector<IndelCands> cands(jobIdx.size());
    std::vector<IndelView> views(jobIdx.size());
    mp::IndelOut io;
    if ((s->deviceSteps & MP_POA_DEVICE_INDELS) && nJobs > 0) {
        // on the GPU: every read's candidates at once (mp_indels.cu)
        PhaseTimer tCands(s->phase[kPhaseCandidates]);
        std::vector<int64_t> refBase(s->nChunks, 0), jRefBase((size_t) nJobs), jRefRuns((size_t) nJobs),
            jReadBase((size_t) nJobs), jReadRuns((size_t) nJobs);
        std::string refChars;
        std::vector<uint32_t> refCounts;
        for (int64_t c : chunks) {
            refBase[c] = (int64_t) refChars.size();
            refChars.append(refs[c].c);
            for (uint64_t k : refs[c].n) refCounts.push_back((uint32_t) k);
        }
        for (int64_t j = 0; j < nJobs; j++) {
            const int64_t c = jobChunk[(size_t) j], r = jobRead[(size_t) j];
            jRefBase[(size_t) j] = refBase[c];
            jRefRuns[(size_t) j] = refs[c].length();
            jReadBase[(size_t) j] = s->flatReadOff[(size_t) r];
            jReadRuns[(size_t) j] = s->reads[r].length();
        }
        mp::IndelBatch ib;
        ib.nJobs = nJobs;
        ib.refBase = jRefBase.data();
        ib.refRuns = jRefRuns.data();
        ib.readBase = jReadBase.data();
        ib.readRuns = jReadRuns.data();
        ib.nRefRuns = (int64_t) refChars.size();
        ib.nReadRuns = (int64_t) s->flatReadChars.size();
        ib.refChars = refChars.data();
        ib.refCounts = refCounts.data();
        ib.readChars = s->flatReadChars.data();
        ib.readCounts = s->flatReadCounts.data();
        for (int k = 0; k < 3; k++) {
            ib.off[k] = offs[k].data();
            ib.w[k] = w[k];
            ib.x[k] = x[k];
            ib.y[k] = y[k];
        }
        ib.cmpRC = s->cmpRC;
        mp_status rc = mp::deviceIndelCandidates(s->e, ib, io);
        if (rc != MP_OK) {
            if (mlThread.joinable()) mlThread.join();
            return rc;
        }
        // each read's candidates are a slice of the pass's page-locked output
        for (int64_t j = 0; j < nJobs; j++) {
            IndelView &v = views[(size_t) j];
            const int64_t c0 = io.candOff[(size_t) j], r0 = io.runOff[(size_t) j];
            v.pos = io.pos + c0, v.len = io.len + c0, v.at = io.at + c0, v.offset = io.offset + c0;
            v.nonRle = io.nonRle + c0, v.w = io.weight + c0;
            v.chars = io.chars + r0, v.counts = io.counts + r0;
            v.n = io.candOff[(size_t) j + 1] - c0;
            v.nIns = io.nIns[(size_t) j];
        }
    } else {
        PhaseTimer tCands(s->phase[kPhaseCandidates]);
        forChunks(jobIdx, [&](int64_t j) {
            thread_local std::vector<Pair> lists[3];
            for (int k = 0; k < 3; k++) {
                lists[k].clear();
                for (int64_t t = offs[k][j]; t < offs[k][j + 1]; t++) lists[k].push_back(Pair{w[k][t], x[k][t], y[k][t]});
            }
            indelCandidates(refs[jobChunk[(size_t) j]], s->reads[jobRead[(size_t) j]], lists[0], lists[2], lists[1],
                            s->cmpRC, cands[(size_t) j]);
            views[(size_t) j] = IndelView::of(cands[(size_t) j]);
        });
    }
    // then each chunk's graph, reads in order. With fewer chunks than host threads, a chunk's
    // nodes are split into ranges merged on separate threads (each range takes every read in
    // order, so every node's lists keep the sequential order).
    auto tMerge = std::chrono::steady_clock::now();
    const int64_t nT = std::max(1u, std::thread::hardware_concurrency());
    const int64_t P = std::max<int64_t>(1, std::min<int64_t>(8, (2 * nT + (int64_t) chunks.size() - 1) /
                                                                   std::max<int64_t>(1, (int64_t) chunks.size())));
    forChunks(chunks, [&](int64_t c) { out[c] = Poa::fromReference(refs[c], maxRC); });
    std::vector<int64_t> items;
    for (int64_t c : chunks)
        for (int64_t k = 0; k < P; k++) items.push_back(c * P + k);
    // per range: its observations, then grouped by node (counting sort over the range's nodes,
    // stable: every node's observations stay in read order)
    std::vector<std::vector<Obs>> rangeObs((size_t) (s->nChunks * P));
    std::vector<std::vector<int64_t>> rangeCount((size_t) (s->nChunks * P));
    forChunks(items, [&](int64_t item) {
        const int64_t c = item / P, k = item % P;
        Poa &poa = out[c];
        const int64_t nN = (int64_t) poa.nodes.size();
        const int64_t lo = nN * k / P, hi = nN * (k + 1) / P;
        std::vector<Obs> obs;
        std::vector<int32_t> node;
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++) {
            const int64_t j = firstJob[c] + (r - s->chunkReads[c]);
            const int64_t t0 = offs[0][j];
            mergeRead(poa, s->reads[r], s->strand[r] != 0, r - s->chunkReads[c], offs[0][j + 1] - t0, w[0] + t0,
                      x[0] + t0, y[0] + t0, views[(size_t) j], lo, hi, obs, node);
        }
        std::vector<int64_t> &cnt = rangeCount[(size_t) item];
        cnt.assign((size_t) (hi - lo + 1), 0);
        for (int32_t v : node) cnt[(size_t) (v - lo) + 1]++;
        for (int64_t i = 0; i < hi - lo; i++) cnt[(size_t) i + 1] += cnt[(size_t) i];
        std::vector<Obs> &sorted = rangeObs[(size_t) item];
        sorted.resize(obs.size());
        std::vector<int64_t> at(cnt.begin(), cnt.end() - 1);
        for (size_t q = 0; q < obs.size(); q++) sorted[(size_t) at[(size_t) (node[q] - lo)]++] = obs[q];
    });
    auto tGroup = std::chrono::steady_clock::now();
    s->phase[kPhaseMerge] += std::chrono::duration<double>(tGroup - tMerge).count();
    // the chunk's observation list: the ranges' grouped lists in node order
    forChunks(chunks, [&](int64_t c) {
        Poa &poa = out[c];
        const int64_t nN = (int64_t) poa.nodes.size();
        size_t total = 0;
        for (int64_t k = 0; k < P; k++) total += rangeObs[(size_t) (c * P + k)].size();
        poa.obs.clear();
        poa.obs.reserve(total);
        poa.obsStart.assign((size_t) nN + 1, 0);
        for (int64_t k = 0; k < P; k++) {
            const int64_t lo = nN * k / P, hi = nN * (k + 1) / P;
            const std::vector<int64_t> &cnt = rangeCount[(size_t) (c * P + k)];
            const int64_t base = (int64_t) poa.obs.size();
            for (int64_t i = lo; i < hi; i++) poa.obsStart[(size_t) i + 1] = base + cnt[(size_t) (i - lo) + 1];
            std::vector<Obs> &o = rangeObs[(size_t) (c * P + k)];
            poa.obs.insert(poa.obs.end(), o.begin(), o.end());
            std::vector<Obs>().swap(o);
        }
        poa.obsNode.clear();
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++)
            cands[(size_t) (firstJob[c] + (r - s->chunkReads[c]))] = IndelCands();
    });
    s->phase[kPhaseGroup] += std::chrono::duration<double>(std::chrono::steady_clock::now() - tGroup).count();
    if (mlThread.joinable()) {
        PhaseTimer tJoin(s->phase[kPhaseJoin]);
        mlThread.join();
        if (mlStatus != MP_OK) return mp_fail(mlStatus, "run-length estimate: %s", mlError.c_str());
        for (int64_t c : chunks)
            out[c].ml.assign(ml.begin() + nodeBase[c] + 1, ml.begin() + nodeBase[c] + refs[c].length() + 1);
    }
    return MP_OK;
}

// Scores the bubble graphs of the listed chunks (their `graphs` entries) with one bubble-scoring
// launch: every allele against every distinct read substring of its bubble (the symbol strings
// of rleString_constructSymbolString, run lengths capped below the table), the result stored as
// float like the reference's alleleReadSupports, then copied to the reads that share a substring.
mp_status scoreBubbles(mp_poa_set *s, const std::vector<int64_t> &chunks, std::vector<BubbleGraph> &graphs) {
    if (!s->e || !s->m) return mp_fail(MP_ERR_STATE, "mp_poa: bubble scoring needs an engine and a model");
    const bool rle = s->m->host[0].runLength != 0;
    const uint64_t maxRC = s->useRle ? (uint64_t) s->rm.M : 2;
    auto symbol = [&](char ch, uint64_t cnt) {
        const uint16_t b = (uint16_t) symbolOf(ch);
        cnt = cnt > maxRC - 1 ? maxRC - 1 : cnt;
        return rle ? (uint16_t) ((cnt << 8) | b) : b;
    };
    struct Count {
        int64_t pairs = 0, xs = 0, ys = 0;
    };
    std::vector<Count> cnt(s->nChunks), base(s->nChunks);
    forChunks(chunks, [&](int64_t c) {
        const BubbleGraph &g = graphs[c];
        Count k;
        for (const Bubble &b : g.bubbles) {
            int64_t distinct = 0;
            for (int64_t r = 0; r < b.nReads; r++)
                if (g.scoreFrom[(size_t) (b.readFirst + r)] == (int32_t) r) {
                    distinct++;
                    k.ys += g.reads[(size_t) (b.readFirst + r)].length;
                }
            k.pairs += distinct * b.nAlleles;
            for (int64_t j = 0; j < b.nAlleles; j++) k.xs += g.alleles[(size_t) (b.alleleFirst + j)].length();
        }
        cnt[c] = k;
    });
    Count total;
    for (int64_t c : chunks) {
        base[c] = total;
        total.pairs += cnt[c].pairs;
        total.xs += cnt[c].xs;
        total.ys += cnt[c].ys;
    }
    if (total.pairs == 0) {
        for (int64_t c : chunks) graphs[c].scored = true;
        return MP_OK;
    }
    std::vector<int64_t> xo((size_t) total.pairs), yo((size_t) total.pairs);
    std::vector<int32_t> xl((size_t) total.pairs), yl((size_t) total.pairs);
    std::vector<uint8_t> st((size_t) total.pairs);
    std::vector<uint16_t> xs((size_t) std::max<int64_t>(total.xs, 1)), ys((size_t) std::max<int64_t>(total.ys, 1));
    std::vector<double> ll((size_t) total.pairs);
    forChunks(chunks, [&](int64_t c) {
        const BubbleGraph &g = graphs[c];
        int64_t p = base[c].pairs, x = base[c].xs, y = base[c].ys;
        std::vector<int64_t> alleleAt;
        for (const Bubble &b : g.bubbles) {
            alleleAt.assign((size_t) b.nAlleles, 0);
            for (int64_t j = 0; j < b.nAlleles; j++) {
                const Rle &a = g.alleles[(size_t) (b.alleleFirst + j)];
                alleleAt[(size_t) j] = x;
                for (int64_t k = 0; k < a.length(); k++) xs[(size_t) x++] = symbol(a.c[k], a.n[k]);
            }
            for (int64_t r = 0; r < b.nReads; r++) {
                if (g.scoreFrom[(size_t) (b.readFirst + r)] != (int32_t) r) continue;
                const ReadSub &rs = g.reads[(size_t) (b.readFirst + r)];
                const Rle &read = s->reads[s->chunkReads[c] + rs.read];
                const int64_t yAt = y;
                for (int64_t k = 0; k < rs.length; k++) ys[(size_t) y++] = symbol(read.c[rs.start + k], read.n[rs.start + k]);
                for (int64_t j = 0; j < b.nAlleles; j++) {
                    xo[(size_t) p] = alleleAt[(size_t) j];
                    xl[(size_t) p] = (int32_t) g.alleles[(size_t) (b.alleleFirst + j)].length();
                    yo[(size_t) p] = yAt;
                    yl[(size_t) p] = (int32_t) rs.length;
                    st[(size_t) p] = s->strand[s->chunkReads[c] + rs.read];
                    p++;
                }
            }
        }
    });
    mp_pair_batch pb;
    pb.n_pairs = total.pairs;
    pb.x_offset = xo.data();
    pb.x_length = xl.data();
    pb.y_offset = yo.data();
    pb.y_length = yl.data();
    pb.strand = st.data();
    pb.x_symbols_length = total.xs;
    pb.x_symbols = xs.data();
    pb.y_symbols_length = total.ys;
    pb.y_symbols = ys.data();
    MP_TRY(mp_forward_pairs(s->e, s->m, &pb, ll.data()));
    forChunks(chunks, [&](int64_t c) {
        BubbleGraph &g = graphs[c];
        int64_t p = base[c].pairs;
        for (const Bubble &b : g.bubbles) {
            float *sup = g.supports.data() + b.supportFirst;
            for (int64_t r = 0; r < b.nReads; r++) {
                const int32_t from = g.scoreFrom[(size_t) (b.readFirst + r)];
                if (from == (int32_t) r) {
                    for (int64_t j = 0; j < b.nAlleles; j++) sup[j * b.nReads + r] = (float) ll[(size_t) p++];
                } else {
                    for (int64_t j = 0; j < b.nAlleles; j++) sup[j * b.nReads + r] = sup[j * b.nReads + from];
                }
            }
        }
        g.scored = true;
    });
    return MP_OK;
}

BubbleGraph buildBubblesOf(mp_poa_set *s, int64_t c) {
    return buildBubbles(s->poas[c], s->reads, s->quals.empty() ? nullptr : &s->quals, s->chunkReads[c],
                        s->candidateFraction, s->anchorTrim, s->keepAtLeast, s->minQual);
}

// poa_realignIterative (impl/polisher.c:2034-2106) for every chunk at once, in consensus mode
// (poa_getConsensus) or polish mode (poa_polish: the bubble graphs of all chunks built on host
// threads, scored in one launch, then each chunk's allele choice and new consensus).
mp_status iterate(mp_poa_set *s, bool polishMode) {
    const int64_t nC = s->nChunks;
    const int64_t minIter = polishMode ? s->minPolish : s->minIter;
    const int64_t maxIter = polishMode ? s->maxPolish : s->maxIter;
    std::vector<double> sc(nC);
    std::vector<int64_t> active;
    for (int64_t c = 0; c < nC; c++) {
        sc[c] = score(s->poas[c]);
        s->iterations[c] = 0;
        if (maxIter > 0) active.push_back(c);
    }
    std::vector<Rle> cons(nC);
    std::vector<std::vector<int64_t>> maps(nC);
    std::vector<Poa> next(nC);
    std::vector<BubbleGraph> graphs(polishMode ? nC : 0);
    while (!active.empty()) {
        std::vector<uint8_t> realign(nC, 0);
        if (polishMode) {
            PhaseTimer t(s->phase[kPhaseBubbles]);
            forChunks(active, [&](int64_t c) { graphs[c] = buildBubblesOf(s, c); });
            MP_TRY(scoreBubbles(s, active, graphs));
        }
        std::vector<std::vector<Anchor>> anchors(s->reads.size());
        auto tCons = std::chrono::steady_clock::now();
        forChunks(active, [&](int64_t c) {
            s->iterations[c]++;
            if (polishMode) {
                cons[c] = bubbleConsensus(s->poas[c], graphs[c], consensusPath(graphs[c]), s->useRle, maps[c]);
                graphs[c] = BubbleGraph();
            } else {
                cons[c] = consensus(s->poas[c], maps[c], s->penalty, s->useRle);
            }
            if (cons[c] == s->poas[c].ref) return;  // greedy convergence
            auto a = anchorAlignments(s->poas[c], &maps[c], s->chunkReads[c + 1] - s->chunkReads[c], s->anchorProbs);
            for (int64_t r = 0; r < (int64_t) a.size(); r++) anchors[s->chunkReads[c] + r] = std::move(a[r]);
            realign[c] = 1;
        });
        s->phase[kPhaseConsensus] += std::chrono::duration<double>(std::chrono::steady_clock::now() - tCons).count();
        std::vector<int64_t> go;
        for (int64_t c : active)
            if (realign[c]) go.push_back(c);
        if (go.empty()) break;
        MP_TRY(realignChunks(s, go, cons, &anchors, next));
        std::vector<int64_t> still;
        std::vector<uint8_t> keep(nC, 0);
        PhaseTimer tRep(s->phase[kPhaseRepeat]);
        std::vector<Poa> trash(nC);  // graphs no longer needed: freed during the next realignment
        forChunks(go, [&](int64_t c) {
            if (s->useRle) estimateRepeatCounts(next[c], s->reads, s->strand, s->chunkReads[c], s->rm);
            const double sc2 = score(next[c]);
            if (sc2 <= sc[c] && s->iterations[c] > minIter) {  // greedy stop: keep the old graph
                trash[c] = std::move(next[c]);
                return;
            }
            trash[c] = std::move(s->poas[c]);
            s->poas[c] = std::move(next[c]);
            sc[c] = sc2;
            keep[c] = 1;
        });
        for (Poa &g : trash)
            if (!g.nodes.empty()) s->trash.push_back(std::move(g));
        for (int64_t c : go)
            if (keep[c] && s->iterations[c] < maxIter) still.push_back(c);
        active.swap(still);
    }
    return MP_OK;
}

mp_status chunkCheck(const mp_poa_set *s, int64_t chunk) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa: NULL set");
    if (chunk < 0 || chunk >= s->nChunks) return mp_fail(MP_ERR_ARGUMENT, "mp_poa: chunk %lld out of range",
                                                         (long long) chunk);
    if (s->poas.empty()) return mp_fail(MP_ERR_STATE, "mp_poa: no graph yet (realign first)");
    return MP_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" mp_status mp_poa_set_create(mp_engine *e, const mp_model *m, const mp_params *p, const mp_polish_params *pp,
                                       const mp_polish_batch *b, const double *repeat_log10, mp_poa_set **out) {
    if (!p || !pp || !b || !out) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: NULL argument");
    *out = nullptr;
    if (b->n_chunks < 0 || !b->ref_offsets || !b->chunk_reads || !b->read_offsets || !b->strand)
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: batch arrays missing");
    if (pp->n_anchor_probs < 2 || (pp->n_anchor_probs & 1) || !pp->anchor_probs)
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: anchor probabilities must be (probability, expansion) pairs");
    if (pp->min_iterations < 0 || pp->max_iterations < pp->min_iterations)
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: need 0 <= min_iterations <= max_iterations");
    if (pp->use_run_length && !repeat_log10)
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: run-length polishing needs the repeat-count table");
    if (pp->min_polish_iterations < 0 || pp->max_polish_iterations < pp->min_polish_iterations)
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: need 0 <= min_polish_iterations <= max_polish_iterations");
    if (pp->max_polish_iterations > 0 && !pp->use_read_alleles)
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: polish mode builds its alleles from the reads' substrings "
                       "(use_read_alleles = 1); the enumeration of candidate variants is not built");
    if (pp->column_anchor_trim < 0 || pp->filter_reads_coverage < 0 || std::isnan(pp->candidate_variant_weight) ||
        std::isnan(pp->min_avg_base_quality))
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: polish-mode parameters out of range");
    mp_poa_set *s = new mp_poa_set();
    s->e = e;
    s->m = m;
    s->p = *p;
    s->penalty = pp->reference_base_penalty;
    s->cmpRC = pp->compare_repeat_counts != 0;
    s->useRle = pp->use_run_length != 0;
    s->anchorProbs.assign(pp->anchor_probs, pp->anchor_probs + pp->n_anchor_probs);
    s->minIter = pp->min_iterations;
    s->maxIter = pp->max_iterations;
    s->minPolish = pp->min_polish_iterations;
    s->maxPolish = pp->max_polish_iterations;
    s->candidateFraction = pp->candidate_variant_weight;
    s->anchorTrim = pp->column_anchor_trim;
    s->keepAtLeast = pp->filter_reads_coverage;
    s->minQual = pp->min_avg_base_quality;
    s->rm.M = mp::kMaxRepeat;
    if (repeat_log10) s->rm.log10.assign(repeat_log10, repeat_log10 + 4 * mp::kMaxRepeat * mp::kMaxRepeat);
    s->nChunks = b->n_chunks;
    const int64_t nReads = b->chunk_reads[b->n_chunks] - b->chunk_reads[0];
    if (b->chunk_reads[0] != 0 || nReads < 0) {
        delete s;
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: chunk_reads must start at 0 and not decrease");
    }
    for (int64_t c = 0; c < b->n_chunks; c++) {
        if (b->ref_offsets[c + 1] < b->ref_offsets[c] || b->chunk_reads[c + 1] < b->chunk_reads[c]) {
            delete s;
            return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: offsets of chunk %lld decrease", (long long) c);
        }
        Rle r;
        for (int64_t i = b->ref_offsets[c]; i < b->ref_offsets[c + 1]; i++) r.push(b->ref_chars[i], b->ref_counts[i]);
        s->drafts.push_back(r);
    }
    s->chunkReads.assign(b->chunk_reads, b->chunk_reads + b->n_chunks + 1);
    s->haveAnchors = b->anchor_offsets != nullptr;
    for (int64_t r = 0; r < nReads; r++) {
        Rle rr;
        for (int64_t i = b->read_offsets[r]; i < b->read_offsets[r + 1]; i++) {
            if (b->read_counts[i] == 0) {
                delete s;
                return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_create: read %lld has a zero run length", (long long) r);
            }
            rr.push(b->read_chars[i], b->read_counts[i]);
        }
        s->reads.push_back(rr);
        s->strand.push_back(b->strand[r]);
        s->flatReadChars.append(rr.c);
        for (uint64_t k : rr.n) s->flatReadCounts.push_back((uint32_t) k);
        if (b->read_qualities)
            s->quals.emplace_back(b->read_qualities + b->read_offsets[r], b->read_qualities + b->read_offsets[r + 1]);
        std::vector<Anchor> a;
        if (s->haveAnchors)
            for (int64_t k = b->anchor_offsets[r]; k < b->anchor_offsets[r + 1]; k++)
                a.push_back(Anchor{b->anchors[3 * k], b->anchors[3 * k + 1], b->anchors[3 * k + 2]});
        s->initialAnchors.push_back(a);
    }
    s->iterations.assign(s->nChunks, 0);
    s->flatReadOff.assign((size_t) nReads + 1, 0);
    for (int64_t r = 0; r < nReads; r++) s->flatReadOff[(size_t) r + 1] = s->flatReadOff[(size_t) r] + s->reads[r].length();
    s->bubbles.resize(s->nChunks);
    *out = s;
    return MP_OK;
}

extern "C" void mp_poa_set_destroy(mp_poa_set *s) {
    delete s;
}

extern "C" mp_status mp_poa_set_realign(mp_poa_set *s) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_realign: NULL set");
    std::vector<int64_t> all(s->nChunks);
    for (int64_t c = 0; c < s->nChunks; c++) all[c] = c;
    std::vector<Poa> out(s->nChunks);
    MP_TRY(realignChunks(s, all, s->drafts, s->haveAnchors ? &s->initialAnchors : nullptr, out));
    s->poas = std::move(out);
    return MP_OK;
}

extern "C" mp_status mp_poa_set_realign_pairs(mp_poa_set *s, const int64_t *const pair_offsets[3],
                                              const int64_t *const pairs[3]) {
    if (!s || !pair_offsets || !pairs) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_realign_pairs: NULL argument");
    for (int k = 0; k < 3; k++)
        if (!pair_offsets[k] || (!pairs[k] && pair_offsets[k][s->reads.size()] > 0))
            return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_realign_pairs: list %d missing", k);
    // every pair must name a cell of its chunk's draft and read
    for (int64_t c = 0; c < s->nChunks; c++)
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++)
            for (int k = 0; k < 3; k++)
                for (int64_t t = pair_offsets[k][r]; t < pair_offsets[k][r + 1]; t++) {
                    const int64_t x = pairs[k][3 * t + 1], y = pairs[k][3 * t + 2];
                    const bool okX = k == 2 ? (x >= -1 && x < s->drafts[c].length()) : (x >= 0 && x < s->drafts[c].length());
                    const bool okY = k == 1 ? (y >= -1 && y < s->reads[r].length()) : (y >= 0 && y < s->reads[r].length());
                    if (!okX || !okY || pairs[k][3 * t] < 0)
                        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_realign_pairs: read %lld list %d pair %lld outside the "
                                       "draft / read", (long long) r, k, (long long) (t - pair_offsets[k][r]));
                }
    std::vector<int64_t> all(s->nChunks);
    for (int64_t c = 0; c < s->nChunks; c++) all[c] = c;
    std::vector<Poa> out(s->nChunks);
    const uint64_t maxRC = s->useRle ? (uint64_t) s->rm.M : 2;
    forChunks(all, [&](int64_t c) {
        Poa poa = Poa::fromReference(s->drafts[c], maxRC);
        for (int64_t r = s->chunkReads[c]; r < s->chunkReads[c + 1]; r++) {
            std::vector<Pair> lists[3];
            for (int k = 0; k < 3; k++)
                for (int64_t t = pair_offsets[k][r]; t < pair_offsets[k][r + 1]; t++)
                    lists[k].push_back(Pair{pairs[k][3 * t], pairs[k][3 * t + 1], pairs[k][3 * t + 2]});
            augment(poa, s->reads[r], s->strand[r] != 0, r - s->chunkReads[c], lists[0], lists[2], lists[1], s->cmpRC);
        }
        poa.groupObs();
        out[c] = std::move(poa);
    });
    s->poas = std::move(out);
    return MP_OK;
}

extern "C" mp_status mp_poa_set_iterate(mp_poa_set *s) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_iterate: NULL set");
    if (s->poas.empty()) return mp_fail(MP_ERR_STATE, "mp_poa_set_iterate: realign first");
    return iterate(s, false);
}

extern "C" mp_status mp_poa_set_iterate_polish(mp_poa_set *s) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_iterate_polish: NULL set");
    if (s->poas.empty()) return mp_fail(MP_ERR_STATE, "mp_poa_set_iterate_polish: realign first");
    return iterate(s, true);
}

extern "C" mp_status mp_poa_set_realign_all(mp_poa_set *s) {
    MP_TRY(mp_poa_set_realign(s));
    if (s->maxIter > 0) MP_TRY(iterate(s, false));
    if (s->maxPolish > 0) MP_TRY(iterate(s, true));
    return MP_OK;
}

extern "C" mp_status mp_poa_set_build_bubbles(mp_poa_set *s) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_build_bubbles: NULL set");
    if (s->poas.empty()) return mp_fail(MP_ERR_STATE, "mp_poa_set_build_bubbles: realign first");
    std::vector<int64_t> all(s->nChunks);
    for (int64_t c = 0; c < s->nChunks; c++) all[c] = c;
    forChunks(all, [&](int64_t c) { s->bubbles[c] = buildBubblesOf(s, c); });
    return MP_OK;
}

extern "C" mp_status mp_poa_set_score_bubbles(mp_poa_set *s) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_score_bubbles: NULL set");
    std::vector<int64_t> all(s->nChunks);
    for (int64_t c = 0; c < s->nChunks; c++) all[c] = c;
    return scoreBubbles(s, all, s->bubbles);
}

extern "C" mp_status mp_poa_bubble_sizes(const mp_poa_set *s, int64_t chunk, int64_t sizes[4]) {
    MP_TRY(chunkCheck(s, chunk));
    if (!sizes) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_bubble_sizes: NULL sizes");
    const BubbleGraph &g = s->bubbles[chunk];
    int64_t runs = 0;
    for (const Rle &a : g.alleles) runs += a.length();
    sizes[0] = (int64_t) g.bubbles.size();
    sizes[1] = (int64_t) g.alleles.size();
    sizes[2] = runs;
    sizes[3] = (int64_t) g.reads.size();
    return MP_OK;
}

extern "C" mp_status mp_poa_bubbles(const mp_poa_set *s, int64_t chunk, int64_t *bubbles, int64_t *allele_runs,
                                    char *chars, uint64_t *counts, int64_t *reads, double *quals, float *supports) {
    MP_TRY(chunkCheck(s, chunk));
    const BubbleGraph &g = s->bubbles[chunk];
    for (size_t i = 0; bubbles && i < g.bubbles.size(); i++) {
        const Bubble &b = g.bubbles[i];
        const int64_t v[6] = {b.refStart, b.refLength, b.alleleFirst, b.nAlleles, b.readFirst, b.nReads};
        memcpy(bubbles + 6 * i, v, sizeof(v));
    }
    int64_t at = 0;
    for (size_t j = 0; j < g.alleles.size(); j++) {
        const Rle &a = g.alleles[j];
        if (allele_runs) allele_runs[j] = a.length();
        for (int64_t k = 0; k < a.length(); k++, at++) {
            if (chars) chars[at] = a.c[k];
            if (counts) counts[at] = a.n[k];
        }
    }
    for (size_t k = 0; k < g.reads.size(); k++) {
        if (reads) {
            reads[3 * k] = g.reads[k].read;
            reads[3 * k + 1] = g.reads[k].start;
            reads[3 * k + 2] = g.reads[k].length;
        }
        if (quals) quals[k] = g.reads[k].qual;
    }
    if (supports && !g.supports.empty()) memcpy(supports, g.supports.data(), sizeof(float) * g.supports.size());
    return MP_OK;
}

extern "C" mp_status mp_poa_bubble_consensus(const mp_poa_set *s, int64_t chunk, int64_t *path, char *chars,
                                             uint64_t *counts, int64_t cap, int64_t *n_runs, int64_t *map) {
    MP_TRY(chunkCheck(s, chunk));
    const BubbleGraph &g = s->bubbles[chunk];
    if (!g.scored) return mp_fail(MP_ERR_STATE, "mp_poa_bubble_consensus: score the bubbles first");
    if (!n_runs) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_bubble_consensus: NULL n_runs");
    const std::vector<int64_t> p = consensusPath(g);
    std::vector<int64_t> m;
    const Rle c = bubbleConsensus(s->poas[chunk], g, p, s->useRle, m);
    *n_runs = c.length();
    if (path) std::copy(p.begin(), p.end(), path);
    if (map) std::copy(m.begin(), m.end(), map);
    if (c.length() > cap) return mp_fail(MP_ERR_OVERFLOW, "mp_poa_bubble_consensus: %lld runs, room for %lld",
                                         (long long) c.length(), (long long) cap);
    for (int64_t k = 0; k < c.length(); k++) {
        if (chars) chars[k] = c.c[k];
        if (counts) counts[k] = c.n[k];
    }
    return MP_OK;
}

extern "C" mp_status mp_poa_set_estimate_repeat_counts(mp_poa_set *s) {
    if (!s) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_estimate_repeat_counts: NULL set");
    if (s->poas.empty()) return mp_fail(MP_ERR_STATE, "mp_poa_set_estimate_repeat_counts: realign first");
    if (!s->useRle) return MP_OK;
    std::vector<int64_t> all(s->nChunks);
    for (int64_t c = 0; c < s->nChunks; c++) all[c] = c;
    PhaseTimer t(s->phase[kPhaseRepeat]);
    forChunks(all, [&](int64_t c) { estimateRepeatCounts(s->poas[c], s->reads, s->strand, s->chunkReads[c], s->rm); });
    return MP_OK;
}

extern "C" mp_status mp_poa_set_device_steps(mp_poa_set *s, int32_t steps) {
    if (!s || (steps & ~(MP_POA_DEVICE_RUN_LENGTHS | MP_POA_DEVICE_INDELS)))
        return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_device_steps: NULL set or unknown steps");
    s->deviceSteps = steps;
    return MP_OK;
}

extern "C" mp_status mp_poa_set_phase_seconds(const mp_poa_set *s, double *seconds, int64_t n) {
    if (!s || (!seconds && n > 0) || n < 0) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_set_phase_seconds: bad arguments");
    for (int64_t k = 0; k < n; k++) seconds[k] = k < kPhaseCount ? s->phase[k] : 0.0;
    return MP_OK;
}

extern "C" mp_status mp_poa_info(const mp_poa_set *s, int64_t chunk, mp_poa_chunk_info *info) {
    MP_TRY(chunkCheck(s, chunk));
    if (!info) return mp_fail(MP_ERR_ARGUMENT, "mp_poa_info: NULL info");
    const Poa &poa = s->poas[chunk];
    memset(info, 0, sizeof(*info));
    info->nodes = (int64_t) poa.nodes.size();
    info->max_repeat = (int64_t) poa.maxRC;
    info->reference_runs = poa.ref.length();
    info->observations = (int64_t) poa.obs.size();
    for (const Node &n : poa.nodes) {
        info->inserts += (int64_t) n.ins.size();
        info->deletes += (int64_t) n.del.size();
        for (const Insert &e : n.ins) info->insert_runs += e.s.length();
    }
    info->score = score(poa);
    info->iterations = s->iterations[chunk];
    return MP_OK;
}

extern "C" mp_status mp_poa_nodes(const mp_poa_set *s, int64_t chunk, char *bases, uint64_t *repeat_counts,
                                  double *base_weights, double *repeat_count_weights, int64_t *n_obs, int64_t *n_ins,
                                  int64_t *n_del) {
    MP_TRY(chunkCheck(s, chunk));
    const Poa &poa = s->poas[chunk];
    const int64_t M = (int64_t) poa.maxRC;
    for (size_t i = 0; i < poa.nodes.size(); i++) {
        const Node &n = poa.nodes[i];
        if (bases) bases[i] = n.base;
        if (repeat_counts) repeat_counts[i] = n.rc;
        if (base_weights)
            for (int k = 0; k < 5; k++) base_weights[5 * i + k] = n.bw[k];
        if (repeat_count_weights)
            for (int64_t k = 0; k < M; k++) repeat_count_weights[M * i + k] = poa.rcwOf((int64_t) i)[k];
        if (n_obs) n_obs[i] = poa.obsCount((int64_t) i);
        if (n_ins) n_ins[i] = (int64_t) n.ins.size();
        if (n_del) n_del[i] = (int64_t) n.del.size();
    }
    return MP_OK;
}

extern "C" mp_status mp_poa_observations(const mp_poa_set *s, int64_t chunk, int64_t *read, int64_t *offset,
                                         double *weight) {
    MP_TRY(chunkCheck(s, chunk));
    int64_t k = 0;
    for (const Obs &o : s->poas[chunk].obs) {  // grouped by node, in the reference's order
        read[k] = o.read;
        offset[k] = o.offset;
        weight[k++] = o.weight;
    }
    return MP_OK;
}

extern "C" mp_status mp_poa_inserts(const mp_poa_set *s, int64_t chunk, double *weight_fwd, double *weight_rev,
                                    int64_t *lengths, char *chars, uint64_t *counts, int64_t *n_obs) {
    MP_TRY(chunkCheck(s, chunk));
    int64_t k = 0, runs = 0;
    for (const Node &n : s->poas[chunk].nodes)
        for (const Insert &e : n.ins) {
            weight_fwd[k] = e.wF;
            weight_rev[k] = e.wR;
            lengths[k] = e.s.length();
            n_obs[k] = (int64_t) e.obs.size();
            for (int64_t r = 0; r < e.s.length(); r++) {
                chars[runs + r] = e.s.c[r];
                counts[runs + r] = e.s.n[r];
            }
            runs += e.s.length();
            k++;
        }
    return MP_OK;
}

extern "C" mp_status mp_poa_deletes(const mp_poa_set *s, int64_t chunk, int64_t *lengths, double *weight_fwd,
                                    double *weight_rev, int64_t *n_obs) {
    MP_TRY(chunkCheck(s, chunk));
    int64_t k = 0;
    for (const Node &n : s->poas[chunk].nodes)
        for (const Delete &e : n.del) {
            lengths[k] = e.len;
            weight_fwd[k] = e.wF;
            weight_rev[k] = e.wR;
            n_obs[k++] = (int64_t) e.obs.size();
        }
    return MP_OK;
}

extern "C" mp_status mp_poa_reference(const mp_poa_set *s, int64_t chunk, char *chars, uint64_t *counts) {
    MP_TRY(chunkCheck(s, chunk));
    const Rle &r = s->poas[chunk].ref;
    for (int64_t i = 0; i < r.length(); i++) {
        chars[i] = r.c[i];
        counts[i] = r.n[i];
    }
    return MP_OK;
}

extern "C" mp_status mp_poa_consensus(const mp_poa_set *s, int64_t chunk, char *chars, uint64_t *counts, int64_t cap,
                                      int64_t *n_runs, int64_t *map) {
    MP_TRY(chunkCheck(s, chunk));
    std::vector<int64_t> mp;
    const Rle c = consensus(s->poas[chunk], mp, s->penalty, s->useRle);
    if (n_runs) *n_runs = c.length();
    if (c.length() > cap) return mp_fail(MP_ERR_OVERFLOW, "mp_poa_consensus: %lld runs exceed the capacity %lld",
                                         (long long) c.length(), (long long) cap);
    for (int64_t i = 0; i < c.length(); i++) {
        if (chars) chars[i] = c.c[i];
        if (counts) counts[i] = c.n[i];
    }
    if (map)
        for (size_t i = 0; i < mp.size(); i++) map[i] = mp[i];
    return MP_OK;
}

extern "C" mp_status mp_poa_anchor_alignments(const mp_poa_set *s, int64_t chunk, const int64_t *map,
                                              int64_t *offsets, int64_t *triples, int64_t cap, int64_t *n_anchors) {
    MP_TRY(chunkCheck(s, chunk));
    const int64_t nR = s->chunkReads[chunk + 1] - s->chunkReads[chunk];
    std::vector<int64_t> mv;
    if (map) mv.assign(map, map + (s->poas[chunk].nodes.size() - 1));
    auto a = anchorAlignments(s->poas[chunk], map ? &mv : nullptr, nR, s->anchorProbs);
    int64_t k = 0;
    offsets[0] = 0;
    for (int64_t r = 0; r < nR; r++) {
        for (const Anchor &t : a[r]) {
            if (k < cap) {
                triples[3 * k] = t.x;
                triples[3 * k + 1] = t.y;
                triples[3 * k + 2] = t.e;
            }
            k++;
        }
        offsets[r + 1] = k;
    }
    if (n_anchors) *n_anchors = k;
    if (k > cap) return mp_fail(MP_ERR_OVERFLOW, "mp_poa_anchor_alignments: %lld anchors exceed the capacity",
                                (long long) k);
    return MP_OK;
}
