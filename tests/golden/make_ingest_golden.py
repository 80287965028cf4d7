"""Generates the ingest fixtures from the reference's own chunking test (tests/chunkingTest.c):

* tests/golden/chunking_test.bam: the test's alignments (tests/data/chunkingTest/
  chunkingTest.sam in the MarginPolish tree: reads with soft and hard clips, insertions and
  deletions placed on chunk boundaries, and quality strings) written as a BAM file by the small
  BGZF / BAM writer below, following the SAM/BAM specification;
* tests/golden/chunking_known_answers.json: the expected reads and aligned pairs of the test's
  four alignment cases (test_readAlignments{With,Without}SoftclippingChunk{Start,End}), read
  from the test source as text: per read the expected sequence and the (reference, read)
  coordinates of every aligned pair.

Usage (where the reference tree exists; a second):
    python tests/golden/make_ingest_golden.py [reference tree]
"""
import json
import os
import re
import struct
import sys
import zlib

HERE = os.path.dirname(os.path.abspath(__file__))
SAM = "tests/data/chunkingTest/chunkingTest.sam"
TEST = "tests/chunkingTest.c"
CASES = ("test_readAlignmentsWithoutSoftclippingChunkStart", "test_readAlignmentsWithSoftclippingChunkStart",
         "test_readAlignmentsWithoutSoftclippingChunkEnd", "test_readAlignmentsWithSoftclippingChunkEnd")


def reg2bin(beg: int, end: int) -> int:
    """The BAI bin of [beg, end) (SAM/BAM specification, section 5.3)."""
    end -= 1
    for shift, offset in ((14, 4681), (17, 585), (20, 73), (23, 9), (26, 1)):
        if beg >> shift == end >> shift:
            return offset + (beg >> shift)
    return 0


def bam_records(lines, tid_of):
    out = []
    for line in lines:
        f = line.rstrip("\n").split("\t")
        qname, flag, rname, pos, mapq, cigar, rnext, pnext, tlen, seq, qual = f[:11]
        tid = tid_of.get(rname, -1)
        pos0 = int(pos) - 1
        ops = [(int(n), "MIDNSHP=X".index(op)) for n, op in re.findall(r"(\d+)([MIDNSHP=X])", cigar)]
        ref_len = sum(n for n, op in ops if op in (0, 2, 3, 7, 8))
        lseq = 0 if seq == "*" else len(seq)
        codes = ["=ACMGRSVTWYHKDBN".index(c) for c in seq.upper()] if lseq else []
        packed = bytes((codes[i] << 4) | (codes[i + 1] if i + 1 < lseq else 0) for i in range(0, lseq, 2))
        quals = bytes([0xff] * lseq) if qual == "*" else bytes(ord(c) - 33 for c in qual)
        ntid = -1 if rnext == "*" else (tid if rnext == "=" else tid_of[rnext])
        name = qname.encode() + b"\0"
        body = struct.pack("<iiBBHHHiiii", tid, pos0, len(name), int(mapq),
                           reg2bin(pos0, pos0 + max(ref_len, 1)), len(ops), int(flag), lseq, ntid, int(pnext) - 1,
                           int(tlen))
        body += name + b"".join(struct.pack("<I", (n << 4) | op) for n, op in ops) + packed + quals
        out.append(struct.pack("<i", len(body)) + body)
    return out


def bgzf(data: bytes) -> bytes:
    """BGZF blocks of at most 64 KB of input each, then the end-of-file block."""
    out = b""
    for at in range(0, len(data), 0xff00):
        raw = data[at:at + 0xff00]
        c = zlib.compressobj(6, zlib.DEFLATED, -15)
        comp = c.compress(raw) + c.flush()
        bsize = len(comp) + 25
        out += struct.pack("<BBBBIBBHBBHH", 31, 139, 8, 4, 0, 0, 255, 6, 66, 67, 2, bsize) + comp
        out += struct.pack("<II", zlib.crc32(raw) & 0xffffffff, len(raw))
    return out + bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")


def write_bam(sam_path: str, out_path: str) -> None:
    header, body, targets = [], [], []
    with open(sam_path) as f:
        for line in f:
            if line.startswith("@"):
                header.append(line)
                if line.startswith("@SQ"):
                    tags = dict(t.split(":", 1) for t in line.rstrip("\n").split("\t")[1:])
                    targets.append((tags["SN"], int(tags["LN"])))
            elif line.strip():
                body.append(line)
    text = "".join(header).encode()
    data = b"BAM\1" + struct.pack("<i", len(text)) + text + struct.pack("<i", len(targets))
    for name, length in targets:
        n = name.encode() + b"\0"
        data += struct.pack("<i", len(n)) + n + struct.pack("<i", length)
    data += b"".join(bam_records(body, {name: i for i, (name, _) in enumerate(targets)}))
    with open(out_path, "wb") as f:
        f.write(bgzf(data))


def known_answers(test_source: str) -> dict:
    """Per alignment test: the expected read count and, per read, the expected sequence and the
    expected (reference, read) coordinates of its aligned pairs."""
    src = open(test_source).read()
    out = {}
    for name in CASES:
        start = src.index(f"static void {name}(")
        end = src.index("static void ", start + 10) if "static void " in src[start + 10:] else len(src)
        body = src[start:end]
        count = int(re.search(r"readCount == (\d+)", body).group(1))
        reads = {}
        for m in re.finditer(r'case (\d+):[^\n]*\n\s*CuAssertTrue\(testCase, stString_eq\("([A-Z]*)", '
                             r'read->rleRead->rleString\)\);\s*assertAlignmentMatching\(testCase, '
                             r'stList_get\(alignments, i\),\s*\(int64_t\[\]\) \{([\d,]*)\},\s*\(int64_t\[\]\) '
                             r'\{([\d,]*)\}, *(\d+)\);', body):
            idx, seq, read_pos, ref_pos, n = m.groups()
            # the test compares the first n entries of each array (one case lists 8 read
            # positions against 7 reference positions)
            rp = ([int(v) for v in read_pos.split(",")] if read_pos else [])[:int(n)]
            fp = ([int(v) for v in ref_pos.split(",")] if ref_pos else [])[:int(n)]
            assert len(rp) == len(fp) == int(n)
            reads[int(idx)] = {"sequence": seq, "pairs": [[a, b] for a, b in zip(fp, rp)]}
        out[name] = {"reads": count, "expected": reads}
    return out


def main() -> None:
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MP_REFERENCE_TREE")
    if not tree or not os.path.exists(os.path.join(tree, SAM)):
        sys.exit("usage: make_ingest_golden.py <reference tree> (or set MP_REFERENCE_TREE)")
    write_bam(os.path.join(tree, SAM), os.path.join(HERE, "chunking_test.bam"))
    ka = known_answers(os.path.join(tree, TEST))
    with open(os.path.join(HERE, "chunking_known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1)
    print({k: (v["reads"], len(v["expected"])) for k, v in ka.items()})


if __name__ == "__main__":
    main()
