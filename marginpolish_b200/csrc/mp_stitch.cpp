// Chunk stitching: the polished chunks of a contig joined where neighbouring chunks overlap.
//
//   mergeContigChunks  impl/chunker.c:50-112         mp_merge_contig
//   removeOverlap      impl/polisher.c:1937-2006     the crop of one boundary (cropOf)
//
// For every boundary the reference aligns the last `overlap` characters of the previous chunk
// (as cropped so far) with the first `overlap` characters of the next chunk, without anchors,
// ragged at both ends, and cuts both at the first match pair of the largest posterior weight.
// Here every boundary's alignment is one job of a single GPU launch that computes the match
// posteriors in the reference's own arithmetic (mp_refpost.cu): over an overlap of identical
// sequence the weights form a plateau whose maximum only that arithmetic places where the
// reference does. A boundary's window of the previous chunk is that chunk's last `overlap`
// characters unless the chunk was cropped into them (a chunk shorter than its crop plus the
// overlap, or a spacer that replaced a missing chunk); the walk that applies the crops in order
// re-aligns exactly those boundaries with the strings as they then are.
#include "../../include/mpgpu.h"
#include "mp_host.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#define MP_TRY_POA(expr)               \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

namespace {

// The nucleotide alphabet (impl/stateMachine.c:25-59): A C G T in either case, anything else N.
uint16_t nucleotideSymbol(char ch) {
    switch (ch) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 4;
    }
}

struct Window {
    std::string x, y;  // the previous chunk's tail and the next chunk's head
};

struct Crop {
    int64_t weight = 0;   // integer weight of the chosen match pair, 0 when there is none
    int64_t xEnd = 0;     // exclusive end of the previous chunk in its window: the pair's x (its
                          // base is then taken from the next chunk)
    int64_t yStart = 0;   // first kept character of the next chunk: the pair's y
};

// removeOverlap's windows (impl/polisher.c:1941-1956).
Window windowsOf(const std::string &prefix, const std::string &suffix, int64_t overlap) {
    const int64_t i = std::max<int64_t>((int64_t) prefix.size() - overlap, 0);
    const int64_t j = std::min<int64_t>(overlap, (int64_t) suffix.size());
    return Window{prefix.substr((size_t) i), suffix.substr(0, (size_t) j)};
}

// The match pairs of every window pair (getAlignedPairs with ragged ends,
// impl/pairwiseAligner.c:1132-1139) in one launch, in the reference's arithmetic, then per pair
// the first of the heaviest match pairs (impl/polisher.c:1981-1998). Windows with an empty side
// have no match pairs.
mp_status cropsOf(mp_engine *e, const mp_model *m, const mp_params *p, const std::vector<Window> &w,
                  std::vector<Crop> &out) {
    out.assign(w.size(), Crop());
    std::vector<int64_t> jobOf;
    std::vector<RefPair> pairs;
    std::vector<uint16_t> xs, ys;
    for (size_t k = 0; k < w.size(); k++) {
        out[k].xEnd = (int64_t) w[k].x.size();
        if (w[k].x.empty() || w[k].y.empty()) continue;
        jobOf.push_back((int64_t) k);
        RefPair q{(int64_t) xs.size(), (int64_t) ys.size(), (int32_t) w[k].x.size(), (int32_t) w[k].y.size(), true,
                  true, true};
        for (char ch : w[k].x) xs.push_back(nucleotideSymbol(ch));
        for (char ch : w[k].y) ys.push_back(nucleotideSymbol(ch));
        pairs.push_back(q);
    }
    if (pairs.empty()) return MP_OK;
    std::vector<std::vector<RefTuple>> tuples;
    MP_TRY_POA(refMatchPairs(e, m, p, pairs, xs, ys, tuples));
    for (size_t j = 0; j < pairs.size(); j++) {
        Crop &c = out[(size_t) jobOf[j]];
        bool found = false;
        for (const RefTuple &t : tuples[j]) {
            if (!found || t.weight > c.weight) {  // the first of the heaviest
                found = true;
                c.weight = t.weight;
                c.xEnd = t.x;
                c.yStart = t.y;
            }
        }
    }
    return MP_OK;
}

}  // namespace

extern "C" mp_status mp_merge_contig(mp_engine *e, const mp_model *m, const mp_params *p, int64_t n_chunks,
                                     const int64_t *offsets, const char *chars, int64_t overlap,
                                     int64_t spacer_length, char *out, int64_t cap, int64_t *out_length,
                                     int64_t *report) {
    if (!e || !m || !p || !out_length || (n_chunks > 0 && (!offsets || !chars)) || n_chunks < 0 || overlap < 0 ||
        spacer_length < 0)
        return mp_fail(MP_ERR_ARGUMENT, "mp_merge_contig: bad argument");
    for (int64_t c = 0; c < n_chunks; c++)
        if (offsets[c + 1] < offsets[c]) return mp_fail(MP_ERR_ARGUMENT, "mp_merge_contig: offsets decrease at %lld",
                                                        (long long) c);
    std::vector<std::string> chunk((size_t) n_chunks);
    for (int64_t c = 0; c < n_chunks; c++) chunk[(size_t) c].assign(chars + offsets[c], (size_t) (offsets[c + 1] - offsets[c]));
    // every boundary's windows as if no crop reached into them, aligned in one batch
    std::vector<Window> w;
    for (int64_t c = 1; c < n_chunks; c++) w.push_back(windowsOf(chunk[(size_t) c - 1], chunk[(size_t) c], overlap));
    std::vector<Crop> crops;
    MP_TRY_POA(cropsOf(e, m, p, w, crops));
    // the walk of mergeContigChunks
    const std::string spacer((size_t) spacer_length, 'N');
    std::vector<std::string> pieces;
    for (int64_t c = 0; c < n_chunks; c++) {
        std::string cur = chunk[(size_t) c];
        int64_t kind = 0, weight = 0, trimStart = 0;
        if (!pieces.empty()) {
            std::string &prev = pieces.back();
            Window now = windowsOf(prev, cur, overlap);
            Crop cr = crops[(size_t) c - 1];
            if (now.x != w[(size_t) c - 1].x || now.y != w[(size_t) c - 1].y) {  // cropped into: align again
                std::vector<Crop> one;
                MP_TRY_POA(cropsOf(e, m, p, std::vector<Window>{now}, one));
                cr = one[0];
            }
            weight = cr.weight;
            if (cr.weight > 0) {
                const int64_t i = (int64_t) prev.size() - (int64_t) now.x.size();
                prev.resize((size_t) (cr.xEnd + i));
                cur = cur.substr((size_t) cr.yStart);
                trimStart = cr.yStart;
            } else if (cur.empty()) {
                cur = spacer;  // a missing chunk
                kind = 1;
            } else if (overlap != 0) {
                pieces.push_back("NNNNNNNNNN");  // no overlap found: Ns at the seam
                kind = 2;
            }
        }
        if (report) {
            report[3 * c] = weight;
            report[3 * c + 1] = trimStart;
            report[3 * c + 2] = kind;
        }
        pieces.push_back(cur);
    }
    int64_t total = 0;
    for (const std::string &s : pieces) total += (int64_t) s.size();
    *out_length = total;
    if (total > cap) return mp_fail(MP_ERR_OVERFLOW, "mp_merge_contig: %lld characters, room for %lld",
                                    (long long) total, (long long) cap);
    int64_t at = 0;
    for (const std::string &s : pieces) {
        if (out) memcpy(out + at, s.data(), s.size());
        at += (int64_t) s.size();
    }
    return MP_OK;
}
