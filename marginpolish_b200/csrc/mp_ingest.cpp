// Ingest: a coordinate-sorted BAM file to the chunks, reads and anchors of the polishing loop.
//
//   bamChunker_construct2         impl/htsIntegration.c:149-273   mp_bam_open
//   saveContigChunks              impl/htsIntegration.c:111-140   contigChunks
//   getAlignedReadLength3         impl/htsIntegration.c:23-97     alignedLength
//   convertToReadsAndAlignments   impl/htsIntegration.c:347-661   convertRecord
//   rleString_rleQualities        impl/polisher.c:1692-1714       runQualities
//   runLengthEncodeAlignment      impl/polisher.c:1731-1750       rleAnchors
//
// htslib (a submodule of the reference) is absent, so the file is read here: BGZF blocks
// (gzip members with a BC extra field) inflated with zlib, then the BAM header and records as
// the SAM/BAM specification lays them out. Opening scans the file once: it builds the chunks
// from every contig's aligned extent, as the reference does, and keeps each record's position,
// end and virtual file offset, so that converting a range of chunks later seeks to the first
// record that can overlap them and reads only to their end. Records come in file order, the
// order the reference's region iterator yields them.
#include "../../include/mpgpu.h"
#include "mp_host.h"

#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#define MP_TRY_BAM(expr)               \
    do {                               \
        mp_status _s = (expr);         \
        if (_s != MP_OK) return _s;    \
    } while (0)

namespace {

// ---------------------------------------------------------------------------
// BGZF
// ---------------------------------------------------------------------------

class Bgzf {
public:
    ~Bgzf() {
        if (f_) fclose(f_);
    }
    bool open(const char *path) {
        f_ = fopen(path, "rb");
        return f_ != nullptr;
    }
    // Virtual offset of the next byte: block start << 16 | offset in the block.
    uint64_t tell() const { return (blockStart_ << 16) | (uint64_t) pos_; }
    bool seek(uint64_t voffset) {
        if (fseeko(f_, (off_t) (voffset >> 16), SEEK_SET) != 0) return false;
        nextBlock_ = voffset >> 16;
        buf_.clear();
        pos_ = 0;
        if (!fill()) return false;
        pos_ = (size_t) (voffset & 0xffff);
        return pos_ <= buf_.size();
    }
    // Reads n bytes; false at the end of the file (or on a damaged block: error() tells).
    bool read(void *dst, size_t n) {
        uint8_t *d = static_cast<uint8_t *>(dst);
        while (n > 0) {
            if (pos_ == buf_.size() && !fill()) return false;
            const size_t k = std::min(n, buf_.size() - pos_);
            memcpy(d, buf_.data() + pos_, k);
            pos_ += k;
            d += k;
            n -= k;
        }
        return true;
    }
    const char *error() const { return err_; }

private:
    // Inflates the next non-empty block into buf_.
    bool fill() {
        for (;;) {
            uint8_t h[18];
            blockStart_ = nextBlock_;
            if (fread(h, 1, 12, f_) != 12) return false;  // end of file
            if (h[0] != 31 || h[1] != 139 || h[2] != 8 || !(h[3] & 4)) {
                err_ = "not a BGZF block";
                return false;
            }
            const uint16_t xlen = (uint16_t) (h[10] | (h[11] << 8));
            std::vector<uint8_t> extra(xlen);
            if (fread(extra.data(), 1, xlen, f_) != xlen) {
                err_ = "truncated BGZF header";
                return false;
            }
            int64_t bsize = -1;
            for (size_t i = 0; i + 4 <= extra.size();) {
                const uint16_t slen = (uint16_t) (extra[i + 2] | (extra[i + 3] << 8));
                if (extra[i] == 'B' && extra[i + 1] == 'C' && slen == 2 && i + 6 <= extra.size())
                    bsize = extra[i + 4] | (extra[i + 5] << 8);
                i += 4 + slen;
            }
            if (bsize < 0) {
                err_ = "BGZF block without its size field";
                return false;
            }
            const int64_t cdata = bsize - xlen - 19;
            if (cdata < 0) {
                err_ = "bad BGZF block size";
                return false;
            }
            std::vector<uint8_t> comp((size_t) cdata + 8);
            if (fread(comp.data(), 1, comp.size(), f_) != comp.size()) {
                err_ = "truncated BGZF block";
                return false;
            }
            nextBlock_ = blockStart_ + (uint64_t) bsize + 1;
            const uint32_t isize = comp[cdata + 4] | (comp[cdata + 5] << 8) | (comp[cdata + 6] << 16) |
                                   ((uint32_t) comp[cdata + 7] << 24);
            buf_.assign(isize, 0);
            pos_ = 0;
            if (isize == 0) continue;  // the end-of-file marker, or an empty block
            z_stream zs;
            memset(&zs, 0, sizeof(zs));
            if (inflateInit2(&zs, -15) != Z_OK) {
                err_ = "zlib";
                return false;
            }
            zs.next_in = comp.data();
            zs.avail_in = (uInt) cdata;
            zs.next_out = buf_.data();
            zs.avail_out = isize;
            const int r = inflate(&zs, Z_FINISH);
            inflateEnd(&zs);
            if (r != Z_STREAM_END || zs.avail_out != 0) {
                err_ = "corrupt BGZF block";
                return false;
            }
            return true;
        }
    }

    FILE *f_ = nullptr;
    std::vector<uint8_t> buf_;
    size_t pos_ = 0;
    uint64_t blockStart_ = 0, nextBlock_ = 0;
    const char *err_ = nullptr;
};

// ---------------------------------------------------------------------------
// BAM records
// ---------------------------------------------------------------------------

enum CigarOp { kM = 0, kI = 1, kD = 2, kN = 3, kS = 4, kH = 5, kP = 6, kEq = 7, kX = 8 };

struct Record {
    int32_t tid = -1, pos = 0;
    uint8_t mapq = 0;
    uint16_t flag = 0;
    int32_t lseq = 0;
    std::string name;
    std::vector<uint32_t> cigar;
    std::vector<uint8_t> seq;   // 4-bit codes, two per byte
    std::vector<uint8_t> qual;  // lseq values, 0xff when absent
    int base(int64_t i) const { return (seq[(size_t) (i >> 1)] >> ((~i & 1) << 2)) & 15; }
};

template <class T>
T le(const uint8_t *p) {
    T v;
    memcpy(&v, p, sizeof(T));
    return v;
}

// Reads one record; false at the end of the file.
bool readRecord(Bgzf &z, Record &r, std::vector<uint8_t> &scratch, bool &bad) {
    uint8_t b4[4];
    bad = false;
    if (!z.read(b4, 4)) return false;
    const int32_t size = le<int32_t>(b4);
    if (size < 32) {
        bad = true;
        return false;
    }
    scratch.resize((size_t) size);
    if (!z.read(scratch.data(), (size_t) size)) {
        bad = true;
        return false;
    }
    const uint8_t *p = scratch.data();
    r.tid = le<int32_t>(p);
    r.pos = le<int32_t>(p + 4);
    const uint8_t lname = p[8];
    r.mapq = p[9];
    const uint16_t ncig = le<uint16_t>(p + 12);
    r.flag = le<uint16_t>(p + 14);
    r.lseq = le<int32_t>(p + 16);
    const size_t need = 32 + (size_t) lname + 4 * (size_t) ncig + (size_t) ((r.lseq + 1) / 2) + (size_t) r.lseq;
    if (r.lseq < 0 || need > (size_t) size) {
        bad = true;
        return false;
    }
    const uint8_t *q = p + 32;
    r.name.assign((const char *) q, lname > 0 ? lname - 1 : 0);
    q += lname;
    r.cigar.resize(ncig);
    memcpy(r.cigar.data(), q, 4 * (size_t) ncig);
    q += 4 * (size_t) ncig;
    r.seq.assign(q, q + (r.lseq + 1) / 2);
    q += (r.lseq + 1) / 2;
    r.qual.assign(q, q + r.lseq);
    return true;
}

// getAlignedReadLength3 (impl/htsIntegration.c:23-97): the read length minus its clips, plus
// deletions, minus insertions; with boundaryAtMatch false only soft clips count as clips.
int64_t alignedLength(const Record &r, int64_t &startClip, int64_t &endClip, bool boundaryAtMatch) {
    startClip = endClip = 0;
    const int64_t n = (int64_t) r.cigar.size();
    for (int64_t i = 0; i < n; i++) {
        const int op = r.cigar[i] & 15, num = (int) (r.cigar[i] >> 4);
        if (op == kM || op == kEq || op == kX) break;
        if (op == kD || op == kN) {
            if (!boundaryAtMatch) break;
        } else if (op == kI) {
            if (!boundaryAtMatch) break;
            startClip += num;
        } else if (op == kS) {
            startClip += num;
        }
    }
    for (int64_t i = n - 1; i > 0; i--) {
        const int op = r.cigar[i] & 15, num = (int) (r.cigar[i] >> 4);
        if (op == kM || op == kEq || op == kX) break;
        if (op == kD || op == kN) {
            if (!boundaryAtMatch) break;
        } else if (op == kI) {
            if (!boundaryAtMatch) break;
            endClip += num;
        } else if (op == kS) {
            endClip += num;
        }
    }
    int64_t ins = 0, del = 0;
    for (uint32_t c : r.cigar) {
        if ((c & 15) == kI) ins += c >> 4;
        if ((c & 15) == kD) del += c >> 4;
    }
    return r.lseq - startClip - endClip + del - ins;
}

struct Chunk {
    int32_t tid;
    int64_t boundaryStart, start, end, boundaryEnd;
    uint64_t firstOffset = 0;  // virtual offset of the first record that can overlap it
    bool hasFirst = false;
};

// saveContigChunks (impl/htsIntegration.c:111-140).
void contigChunks(std::vector<Chunk> &out, int32_t tid, int64_t from, int64_t to, int64_t size, int64_t margin) {
    if (size == 0) {
        out.push_back(Chunk{tid, from, from, to, to});
        return;
    }
    for (int64_t i = from; i < to; i += size) {
        const int64_t end = std::min(i + size, to);
        out.push_back(Chunk{tid, std::max(i - margin, from), i, end, std::min(end + margin, to)});
    }
}

// The filters of both scans (impl/htsIntegration.c:200-208, :399-409).
bool keep(const Record &r, const mp_bam_params &p, bool mapq) {
    if (r.lseq <= 0 || r.cigar.empty() || (r.flag & 0x4)) return false;
    if (!p.include_secondary && (r.flag & 0x100)) return false;
    if (!p.include_supplementary && (r.flag & 0x800)) return false;
    if (mapq && r.mapq < p.min_mapq) return false;
    return true;
}

struct ChunkReads {
    std::vector<std::string> names;
    std::vector<std::string> seqs;
    std::vector<std::vector<uint8_t>> quals;   // empty: no qualities
    std::vector<uint8_t> forward;
    std::vector<std::vector<int64_t>> pairs;   // (ref, read, score) triples, chunk / read coordinates
};

// convertToReadsAndAlignments' per-record work (impl/htsIntegration.c:397-646) for one chunk:
// appends the read (trimmed to the chunk, soft clips as configured) and its aligned pairs.
void convertRecord(const Record &r, const Chunk &c, bool includeSoftClip, ChunkReads &out) {
    const int64_t chunkStart = c.boundaryStart, chunkEnd = c.boundaryEnd;
    int64_t sClip = 0, eClip = 0;
    const int64_t alnLen = alignedLength(r, sClip, eClip, false);
    if (alnLen <= 0) return;
    const int64_t alnStart = r.pos, alnEnd = alnStart + alnLen;
    if (alnStart >= chunkEnd || alnEnd <= chunkStart) return;
    std::vector<int64_t> pairs;
    int64_t cigIdx = 0, posInOp = 0, op = -1, num = -1, idxInSeq = 0, idxInRef = alnStart;
    const int64_t refMod = -chunkStart;
    int64_t seqMod, firstIdx;
    if (includeSoftClip) {
        if (alnStart < chunkStart) {
            firstIdx = -1;
            seqMod = 0;
        } else if (alnStart - sClip <= chunkStart) {
            firstIdx = 0;
            seqMod = alnStart - chunkStart;
        } else {
            firstIdx = 0;
            seqMod = sClip;
        }
    } else {
        firstIdx = alnStart < chunkStart ? -1 : 0;
        seqMod = 0;
    }
    int64_t alignedRead = 0;
    const int64_t nCig = (int64_t) r.cigar.size();
    for (int64_t i = 0; i <= alnLen; i++) {
        if (cigIdx == nCig) break;
        if (posInOp == 0) {
            op = r.cigar[(size_t) cigIdx] & 15;
            num = r.cigar[(size_t) cigIdx] >> 4;
        }
        if (op == kM || op == kEq || op == kX) {
            if (idxInRef >= chunkStart && idxInRef < chunkEnd) {
                pairs.push_back(idxInRef + refMod);
                pairs.push_back(idxInSeq + seqMod);
                pairs.push_back(10);  // DEFAULT_ALIGNMENT_SCORE (impl/htsIntegration.c:338)
                alignedRead++;
            }
            idxInSeq++;
            idxInRef++;
        } else if (op == kD || op == kN) {
            idxInRef++;
        } else if (op == kI) {
            idxInSeq++;
            if (idxInRef >= chunkStart && idxInRef < chunkEnd) alignedRead++;
            i--;
        } else if (op == kS || op == kH || op == kP) {
            posInOp = num - 1;
            i--;
        }
        if (firstIdx < 0 && idxInRef >= chunkStart) {
            firstIdx = idxInSeq;
            seqMod = -1 * (firstIdx + seqMod);
        }
        posInOp++;
        if (posInOp == num) {
            cigIdx++;
            posInOp = 0;
        }
    }
    int64_t seqLen = alignedRead;
    int64_t readStart = firstIdx;
    if (firstIdx != 0) {
        readStart += sClip;
    } else if (!includeSoftClip) {
        readStart += sClip;
    } else if (alnStart - sClip <= chunkStart) {
        const int64_t included = alnStart - chunkStart;
        seqLen += included;
        readStart += sClip - included;
    } else {
        seqLen += sClip;
        readStart = 0;
    }
    int64_t readEnd = readStart + seqLen;
    if (alnEnd < chunkEnd && includeSoftClip) {
        if (alnEnd + eClip <= chunkEnd) {
            readEnd += eClip;
            seqLen += eClip;
        } else {
            const int64_t included = chunkEnd - alnEnd;
            seqLen += included;
            readEnd += included;
        }
    }
    static const char kNt16[] = "=ACMGRSVTWYHKDBN";
    std::string seq;
    for (int64_t k = readStart; k < readEnd; k++) seq.push_back(kNt16[r.base(k)]);
    std::vector<uint8_t> qual;
    if (r.lseq > 0 && r.qual[0] != 0xff)
        for (int64_t k = readStart; k < readEnd; k++) qual.push_back(r.qual[(size_t) k]);
    if (pairs.empty() || seq.empty()) return;  // the failure case (:604-611)
    out.names.push_back(r.name);
    out.seqs.push_back(seq);
    out.quals.push_back(qual);
    out.forward.push_back((r.flag & 0x10) ? 0 : 1);
    out.pairs.push_back(pairs);
}

}  // namespace

struct mp_bam {
    std::string path;
    mp_bam_params p{};
    std::string region;            // copy of p.region
    std::vector<std::string> targets;
    std::vector<Chunk> chunks;
    // the last conversion: chunks [first, first + n)
    int64_t convFirst = 0;
    std::vector<ChunkReads> conv;
    std::vector<std::string> convRef;  // the reference pieces given (per chunk, may be empty)
    bool convHasRef = false;
};

namespace {

// Reads the header; leaves z at the first record.
mp_status readHeader(Bgzf &z, std::vector<std::string> &targets) {
    uint8_t m[4];
    if (!z.read(m, 4) || memcmp(m, "BAM\1", 4) != 0) return mp_fail(MP_ERR_ARGUMENT, "mp_bam: not a BAM file");
    uint8_t b4[4];
    if (!z.read(b4, 4)) return mp_fail(MP_ERR_ARGUMENT, "mp_bam: truncated header");
    std::vector<uint8_t> text((size_t) le<int32_t>(b4));
    if (!z.read(text.data(), text.size()) || !z.read(b4, 4)) return mp_fail(MP_ERR_ARGUMENT, "mp_bam: truncated header");
    const int32_t nRef = le<int32_t>(b4);
    for (int32_t i = 0; i < nRef; i++) {
        if (!z.read(b4, 4)) return mp_fail(MP_ERR_ARGUMENT, "mp_bam: truncated header");
        std::vector<char> name((size_t) le<int32_t>(b4));
        if (!z.read(name.data(), name.size()) || !z.read(b4, 4))
            return mp_fail(MP_ERR_ARGUMENT, "mp_bam: truncated header");
        targets.emplace_back(name.data(), name.empty() ? 0 : name.size() - 1);
    }
    return MP_OK;
}

// rleString_rleQualities: each run gets the integer mean of its bases' qualities.
std::vector<uint8_t> runQualities(const std::vector<uint64_t> &counts, const std::vector<uint8_t> &q) {
    std::vector<uint8_t> out;
    size_t at = 0;
    for (uint64_t c : counts) {
        int64_t sum = 0;
        for (uint64_t k = 0; k < c; k++) sum += q[at++];
        out.push_back((uint8_t) (sum / (int64_t) c));
    }
    return out;
}

void runs(const std::string &s, bool rle, std::string &chars, std::vector<uint64_t> &counts) {
    chars.clear();
    counts.clear();
    for (size_t i = 0; i < s.size(); i++) {
        if (rle && !chars.empty() && chars.back() == s[i]) {
            counts.back()++;
        } else {
            chars.push_back(s[i]);
            counts.push_back(1);
        }
    }
}

// runLengthEncodeAlignment: pairs mapped to run coordinates, kept while both strictly increase.
std::vector<int64_t> rleAnchors(const std::vector<int64_t> &pairs, const std::vector<uint64_t> &refCounts,
                                const std::vector<uint64_t> &readCounts) {
    std::vector<int64_t> refMap, readMap;
    for (size_t i = 0; i < refCounts.size(); i++) refMap.insert(refMap.end(), refCounts[i], (int64_t) i);
    for (size_t i = 0; i < readCounts.size(); i++) readMap.insert(readMap.end(), readCounts[i], (int64_t) i);
    std::vector<int64_t> out;
    int64_t x = -1, y = -1;
    for (size_t k = 0; k + 2 < pairs.size(); k += 3) {
        // a reference shorter than the chunk's bounds has no run for the pairs past its end
        if ((size_t) pairs[k] >= refMap.size() || (size_t) pairs[k + 1] >= readMap.size()) continue;
        const int64_t x2 = refMap[(size_t) pairs[k]], y2 = readMap[(size_t) pairs[k + 1]];
        if (x2 > x && y2 > y) {
            out.push_back(x2);
            out.push_back(y2);
            out.push_back(pairs[k + 2]);
            x = x2;
            y = y2;
        }
    }
    return out;
}

}  // namespace

extern "C" mp_status mp_bam_open(const char *path, const mp_bam_params *p, mp_bam **out) {
    if (!path || !p || !out) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_open: NULL argument");
    *out = nullptr;
    if (p->chunk_size < 0 || p->chunk_boundary < 0) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_open: negative chunk size");
    Bgzf z;
    if (!z.open(path)) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_open: cannot open %s", path);
    mp_bam *b = new mp_bam();
    b->path = path;
    b->p = *p;
    mp_status s = readHeader(z, b->targets);
    if (s != MP_OK) {
        delete b;
        return s;
    }
    // region filter (impl/htsIntegration.c:154-165)
    bool byRegion = false;
    std::string regionContig;
    long long regionStart = 0, regionEnd = 0;
    if (p->region) {
        b->region = p->region;
        const size_t colon = b->region.rfind(':');
        if (colon == std::string::npos || colon == 0 ||
            sscanf(b->region.c_str() + colon + 1, "%lld-%lld", &regionStart, &regionEnd) != 2 || regionStart < 0 ||
            regionEnd <= 0 || regionEnd <= regionStart) {
            delete b;
            return mp_fail(MP_ERR_ARGUMENT, "mp_bam_open: region %s is not contig:start-end", p->region);
        }
        regionContig = b->region.substr(0, colon);
        byRegion = true;
    }
    struct Span {
        int32_t tid;
        int64_t pos, end;
        uint64_t voff;
    };
    std::vector<Span> spans;
    Record r;
    std::vector<uint8_t> scratch;
    int32_t curTid = -1;
    int64_t cStart = 0, cEnd = 0;
    for (;;) {
        const uint64_t voff = z.tell();
        bool bad = false;
        if (!readRecord(z, r, scratch, bad)) {
            if (bad || z.error()) {
                delete b;
                return mp_fail(MP_ERR_ARGUMENT, "mp_bam_open: %s: damaged record (%s)", path,
                               z.error() ? z.error() : "bad length");
            }
            break;
        }
        int64_t sc, ec;
        const int64_t len = alignedLength(r, sc, ec, false);
        spans.push_back(Span{r.tid, r.pos, r.pos + std::max<int64_t>(len, 0), voff});
        if (!keep(r, *p, false) || len <= 0 || r.tid < 0 || r.tid >= (int32_t) b->targets.size()) continue;
        const int64_t s0 = r.pos, e0 = r.pos + len;
        if (byRegion && (b->targets[(size_t) r.tid] != regionContig || s0 >= regionEnd || e0 <= regionStart)) continue;
        if (curTid < 0) {
            curTid = r.tid, cStart = s0, cEnd = e0;
        } else if (curTid == r.tid) {
            cStart = std::min(cStart, s0);
            cEnd = std::max(cEnd, e0);
        } else {
            contigChunks(b->chunks, curTid, cStart, cEnd, p->chunk_size, p->chunk_boundary);
            curTid = r.tid, cStart = s0, cEnd = e0;
        }
    }
    if (curTid >= 0) {
        if (byRegion) {
            cStart = std::max<int64_t>(cStart, regionStart);
            cEnd = std::min<int64_t>(cEnd, regionEnd);
        }
        contigChunks(b->chunks, curTid, cStart, cEnd, p->chunk_size, p->chunk_boundary);
    }
    // the first record (in file order) that overlaps each chunk: a contig's chunks are
    // contiguous and ordered, so a record's chunks start at the first whose end lies past it
    std::vector<int64_t> first(b->targets.size() + 1, -1), last(b->targets.size() + 1, -1);
    for (size_t i = 0; i < b->chunks.size(); i++) {
        const int32_t t = b->chunks[i].tid;
        if (first[(size_t) t] < 0) first[(size_t) t] = (int64_t) i;
        last[(size_t) t] = (int64_t) i + 1;
    }
    for (const Span &sp : spans) {
        if (sp.tid < 0 || sp.tid >= (int32_t) b->targets.size() || first[(size_t) sp.tid] < 0) continue;
        auto lo = b->chunks.begin() + first[(size_t) sp.tid], hi = b->chunks.begin() + last[(size_t) sp.tid];
        auto it = std::upper_bound(lo, hi, sp.pos, [](int64_t pos, const Chunk &c) { return pos < c.boundaryEnd; });
        for (; it != hi && it->boundaryStart < sp.end; ++it) {
            if (!it->hasFirst && sp.pos < it->boundaryEnd && sp.end > it->boundaryStart) {
                it->firstOffset = sp.voff;
                it->hasFirst = true;
            }
        }
    }
    *out = b;
    return MP_OK;
}

extern "C" void mp_bam_close(mp_bam *b) {
    delete b;
}

extern "C" mp_status mp_bam_chunk_count(const mp_bam *b, int64_t *n) {
    if (!b || !n) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_chunk_count: NULL argument");
    *n = (int64_t) b->chunks.size();
    return MP_OK;
}

extern "C" mp_status mp_bam_chunk(const mp_bam *b, int64_t i, char *contig, int64_t cap, int64_t bounds[4]) {
    if (!b || !bounds) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_chunk: NULL argument");
    if (i < 0 || i >= (int64_t) b->chunks.size()) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_chunk: no chunk %lld",
                                                                (long long) i);
    const Chunk &c = b->chunks[(size_t) i];
    const std::string &name = b->targets[(size_t) c.tid];
    if (contig) {
        if ((int64_t) name.size() + 1 > cap) return mp_fail(MP_ERR_OVERFLOW, "mp_bam_chunk: contig name too long");
        memcpy(contig, name.c_str(), name.size() + 1);
    }
    bounds[0] = c.boundaryStart;
    bounds[1] = c.start;
    bounds[2] = c.end;
    bounds[3] = c.boundaryEnd;
    return MP_OK;
}

extern "C" mp_status mp_bam_convert(mp_bam *b, int64_t first, int64_t n, const int64_t *ref_offsets,
                                    const char *ref_chars, int64_t max_depth, uint64_t seed) {
    if (!b) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_convert: NULL handle");
    if (first < 0 || n < 0 || first + n > (int64_t) b->chunks.size())
        return mp_fail(MP_ERR_ARGUMENT, "mp_bam_convert: chunks [%lld, %lld) out of range", (long long) first,
                       (long long) (first + n));
    if (ref_offsets && !ref_chars) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_convert: reference offsets without chars");
    b->convFirst = first;
    b->conv.assign((size_t) n, ChunkReads());
    b->convHasRef = ref_offsets != nullptr;
    b->convRef.assign((size_t) n, std::string());
    if (ref_offsets)
        for (int64_t k = 0; k < n; k++) {
            if (ref_offsets[k + 1] < ref_offsets[k]) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_convert: reference offsets decrease");
            b->convRef[(size_t) k].assign(ref_chars + ref_offsets[k], (size_t) (ref_offsets[k + 1] - ref_offsets[k]));
        }
    uint64_t start = UINT64_MAX;
    for (int64_t k = 0; k < n; k++) {
        const Chunk &c = b->chunks[(size_t) (first + k)];
        if (c.hasFirst) start = std::min(start, c.firstOffset);
    }
    if (start != UINT64_MAX) {
        Bgzf z;
        if (!z.open(b->path.c_str()) || !z.seek(start))
            return mp_fail(MP_ERR_ARGUMENT, "mp_bam_convert: cannot read %s", b->path.c_str());
        const Chunk &lastChunk = b->chunks[(size_t) (first + n - 1)];
        Record r;
        std::vector<uint8_t> scratch;
        for (;;) {
            bool bad = false;
            if (!readRecord(z, r, scratch, bad)) {
                if (bad || z.error()) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_convert: damaged record");
                break;
            }
            // sorted by contig, then position (unmapped records last): past the last chunk, nothing
            // more can overlap the range
            if (r.tid < 0 || r.tid > lastChunk.tid || (r.tid == lastChunk.tid && r.pos >= lastChunk.boundaryEnd)) break;
            if (!keep(r, b->p, true)) continue;
            for (int64_t k = 0; k < n; k++) {
                const Chunk &c = b->chunks[(size_t) (first + k)];
                if (c.tid == r.tid) convertRecord(r, c, b->p.include_soft_clip != 0, b->conv[(size_t) k]);
            }
        }
    }
    // poorMansDownsample (impl/htsIntegration.c:663-697): above max_depth, keep each read with
    // probability max_depth / depth. The reference draws from sonLib's generator; this one is a
    // seeded splitmix64, so the kept reads are a different sample of the same rule.
    if (max_depth > 0) {
        uint64_t state = seed;
        auto next = [&state]() {
            uint64_t x = (state += 0x9E3779B97F4A7C15ull);
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
            return (double) ((x ^ (x >> 31)) >> 11) * (1.0 / 9007199254740992.0);
        };
        for (int64_t k = 0; k < n; k++) {
            ChunkReads &cr = b->conv[(size_t) k];
            const Chunk &c = b->chunks[(size_t) (first + k)];
            int64_t total = 0;
            std::string chars;
            std::vector<uint64_t> counts;
            for (const std::string &sq : cr.seqs) {
                runs(sq, b->p.use_run_length != 0, chars, counts);
                total += (int64_t) chars.size();
            }
            const double depth = (double) total / (double) std::max<int64_t>(c.boundaryEnd - c.boundaryStart, 1);
            if (depth < (double) max_depth) continue;
            const double ratio = (double) max_depth / depth;
            ChunkReads kept;
            for (size_t i = 0; i < cr.seqs.size(); i++) {
                if (next() < ratio) {
                    kept.names.push_back(cr.names[i]);
                    kept.seqs.push_back(cr.seqs[i]);
                    kept.quals.push_back(cr.quals[i]);
                    kept.forward.push_back(cr.forward[i]);
                    kept.pairs.push_back(cr.pairs[i]);
                }
            }
            cr = std::move(kept);
        }
    }
    return MP_OK;
}

namespace {

mp_status convCheck(const mp_bam *b, int64_t k) {
    if (!b) return mp_fail(MP_ERR_ARGUMENT, "mp_bam: NULL handle");
    if (k < 0 || k >= (int64_t) b->conv.size())
        return mp_fail(MP_ERR_ARGUMENT, "mp_bam: chunk %lld of the last conversion does not exist", (long long) k);
    return MP_OK;
}

// The k-th converted chunk's reads in the form the loop takes: runs (when run lengths are on),
// per-run qualities, and the anchors in run coordinates (only when the reference was given,
// as in the reference's run-length mode; without run lengths they are the aligned pairs).
struct Converted {
    std::vector<std::string> chars;
    std::vector<std::vector<uint64_t>> counts;
    std::vector<std::vector<uint8_t>> quals;
    std::vector<std::vector<int64_t>> anchors;
};

Converted convertedOf(const mp_bam *b, int64_t k) {
    const ChunkReads &cr = b->conv[(size_t) k];
    const bool rle = b->p.use_run_length != 0;
    Converted c;
    std::string refChars;
    std::vector<uint64_t> refCounts;
    runs(b->convRef[(size_t) k], rle, refChars, refCounts);
    for (size_t i = 0; i < cr.seqs.size(); i++) {
        std::string ch;
        std::vector<uint64_t> cn;
        runs(cr.seqs[i], rle, ch, cn);
        c.quals.push_back(cr.quals[i].empty() ? std::vector<uint8_t>() : runQualities(cn, cr.quals[i]));
        if (rle) c.anchors.push_back(b->convHasRef ? rleAnchors(cr.pairs[i], refCounts, cn) : std::vector<int64_t>());
        else c.anchors.push_back(cr.pairs[i]);
        c.chars.push_back(ch);
        c.counts.push_back(cn);
    }
    return c;
}

}  // namespace

extern "C" mp_status mp_bam_reads_sizes(const mp_bam *b, int64_t k, int64_t sizes[4]) {
    MP_TRY_BAM(convCheck(b, k));
    if (!sizes) return mp_fail(MP_ERR_ARGUMENT, "mp_bam_reads_sizes: NULL sizes");
    const Converted c = convertedOf(b, k);
    int64_t runsTotal = 0, anchorsTotal = 0, nameChars = 0;
    for (size_t i = 0; i < c.chars.size(); i++) {
        runsTotal += (int64_t) c.chars[i].size();
        anchorsTotal += (int64_t) c.anchors[i].size() / 3;
        nameChars += (int64_t) b->conv[(size_t) k].names[i].size();
    }
    sizes[0] = (int64_t) c.chars.size();
    sizes[1] = runsTotal;
    sizes[2] = anchorsTotal;
    sizes[3] = nameChars;
    return MP_OK;
}

extern "C" mp_status mp_bam_reads(const mp_bam *b, int64_t k, int64_t *read_offsets, char *chars, uint32_t *counts,
                                  uint8_t *qualities, uint8_t *has_qualities, uint8_t *strand,
                                  int64_t *anchor_offsets, int32_t *anchors, int64_t *name_offsets, char *names) {
    MP_TRY_BAM(convCheck(b, k));
    const Converted c = convertedOf(b, k);
    const ChunkReads &cr = b->conv[(size_t) k];
    int64_t at = 0, an = 0, nm = 0;
    if (read_offsets) read_offsets[0] = 0;
    if (anchor_offsets) anchor_offsets[0] = 0;
    if (name_offsets) name_offsets[0] = 0;
    for (size_t i = 0; i < c.chars.size(); i++) {
        for (size_t j = 0; j < c.chars[i].size(); j++, at++) {
            if (chars) chars[at] = c.chars[i][j];
            if (counts) counts[at] = (uint32_t) c.counts[i][j];
            if (qualities) qualities[at] = c.quals[i].empty() ? 0 : c.quals[i][j];
        }
        if (read_offsets) read_offsets[i + 1] = at;
        if (has_qualities) has_qualities[i] = c.quals[i].empty() ? 0 : 1;
        if (strand) strand[i] = cr.forward[i];
        for (size_t j = 0; j < c.anchors[i].size(); j++)
            if (anchors) anchors[3 * an + (int64_t) j] = (int32_t) c.anchors[i][j];
        an += (int64_t) c.anchors[i].size() / 3;
        if (anchor_offsets) anchor_offsets[i + 1] = an;
        if (names) memcpy(names + nm, cr.names[i].data(), cr.names[i].size());
        nm += (int64_t) cr.names[i].size();
        if (name_offsets) name_offsets[i + 1] = nm;
    }
    return MP_OK;
}
