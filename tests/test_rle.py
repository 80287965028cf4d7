"""Run-length encoding, symbol strings, run-length anchors and the reference crop (integer-exact)."""
import numpy as np

from marginpolish_b200 import RleString, crop_range, rle_anchors


def _rle_py(s):
    chars, counts = [], []
    for c in s:
        if chars and chars[-1] == c:
            counts[-1] += 1
        else:
            chars.append(c)
            counts.append(1)
    return "".join(chars), counts


def test_rle_roundtrip_and_case_sensitivity():
    rng = np.random.default_rng(0)
    for _ in range(200):
        s = "".join(rng.choice(list("ACGTacgtN"), size=int(rng.integers(0, 60))))
        r = RleString.from_string(s)
        chars, counts = _rle_py(s)
        assert r.chars.decode() == chars
        assert list(r.counts) == counts
        assert r.expand() == s
        assert r.non_rle_length == len(s)


def test_symbols_clamp_repeat_counts():
    r = RleString.from_string("A" * 60 + "c" * 3 + "N" + "g")
    s = r.symbols(True, 51)
    assert list(s) == [(50 << 8) | 0, (3 << 8) | 1, (1 << 8) | 4, (1 << 8) | 2]
    assert list(r.symbols(False)) == [0, 1, 4, 2]
    assert list(r.symbols(True, 50)) == [(49 << 8) | 0, (3 << 8) | 1, (1 << 8) | 4, (1 << 8) | 2]


def test_rle_anchors_keep_strictly_increasing_pairs():
    rng = np.random.default_rng(1)
    for _ in range(50):
        x = RleString.from_string("".join(rng.choice(list("ACGT"), size=80)))
        y = RleString.from_string("".join(rng.choice(list("ACGT"), size=70)))
        xm, ym = x.non_rle_to_rle(), y.non_rle_to_rle()
        n = int(rng.integers(0, 60))
        px = np.sort(rng.choice(80, size=n, replace=False))
        py = np.sort(rng.choice(70, size=n, replace=False))
        pairs = np.stack([px, py, np.full(n, 4)], axis=1)
        got = rle_anchors(pairs, x, y)
        want, lx, ly = [], -1, -1  # runLengthEncodeAlignment (impl/polisher.c:1732-1750)
        for a, b, e in pairs:
            x2, y2 = xm[a], ym[b]
            if x2 > lx and y2 > ly:
                want.append((x2, y2, e))
                lx, ly = x2, y2
        assert [tuple(v) for v in got] == want


def test_crop_range_follows_reference():
    anchors = np.array([[10, 3, 0], [20, 15, 0]], dtype=np.int32)
    # first = max(0, 10-3) = 7; end = min(100, 1 + 20 + (40 - 15)) = 46
    assert crop_range(anchors, 100, 40) == (7, 46)
    assert crop_range(np.zeros((0, 3), np.int32), 100, 40) == (0, 100)
    assert crop_range(np.array([[2, 5, 0]], np.int32), 30, 400) == (0, 30)


def test_generator_restatements_match_the_library():
    """The workload generator's numpy routines (so that generating inputs maps no native library)
    give bit-identical results to the library's run-length encoding, symbols, anchors and crop."""
    from marginpolish_b200 import synth
    rng = np.random.default_rng(3)
    for _ in range(100):
        s = "".join(rng.choice(list("ACGTacgtN"), size=int(rng.integers(0, 200))))
        a, b = synth.rle_encode(s.encode()), RleString.from_string(s)
        assert a.chars == b.chars and np.array_equal(a.counts, b.counts)
        for inc, mx in ((True, 51), (True, 50), (False, 51)):
            assert np.array_equal(synth.rle_symbols(a, inc, mx), b.symbols(inc, mx))
    for _ in range(100):
        x = RleString.from_string("".join(rng.choice(list("ACGT"), size=300, p=[0.4, 0.1, 0.1, 0.4])))
        y = RleString.from_string("".join(rng.choice(list("ACGT"), size=280, p=[0.4, 0.1, 0.1, 0.4])))
        n = int(rng.integers(0, 250))
        px = np.sort(rng.choice(300, size=n, replace=False))
        py = np.sort(rng.choice(280, size=n, replace=False))
        pairs = np.stack([px, py, 2 * rng.integers(0, 30, size=n)], axis=1)
        assert np.array_equal(synth.rle_anchors_monotone(pairs, x, y), rle_anchors(pairs, x, y))
        if n:
            an = rle_anchors(pairs, x, y)
            if an.shape[0]:
                assert synth.crop_range(an, len(x), len(y)) == crop_range(an, len(x), len(y))
