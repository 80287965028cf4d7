"""Run-length encoded strings, symbol strings and run-length anchors.

Thin wrappers over the library's integer-exact host routines:
``RleString`` follows rleString_construct / rleString_expand
(impl/polisher.c:1357-1389, :1496-1506), ``symbols`` follows
rleString_constructSymbolString (impl/stateMachine.c:133-146) and
``rle_anchors`` follows runLengthEncodeAlignment (impl/polisher.c:1732-1750).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import c_char, c_int32, c_int64, c_uint16, c_uint32


@dataclass
class RleString:
    chars: bytes             # one character per run
    counts: np.ndarray       # uint32 run lengths

    @classmethod
    def from_string(cls, s) -> "RleString":
        if isinstance(s, str):
            s = s.encode()
        n = len(s)
        chars = (c_char * max(n, 1))()
        counts = np.zeros(max(n, 1), dtype=np.uint32)
        nr = c_int64(0)
        _lib.check(_lib.load().mp_rle_encode(s, n, chars, _lib.ptr(counts, c_uint32), nr))
        return cls(bytes(chars[:nr.value]), counts[:nr.value].copy())

    def __len__(self) -> int:
        return len(self.chars)

    @property
    def non_rle_length(self) -> int:
        return int(self.counts.sum())

    def expand(self) -> str:
        return "".join(chr(c) * int(k) for c, k in zip(self.chars, self.counts))

    def symbols(self, include_counts: bool = True, max_repeat_exclusive: int = _lib.MP_MAX_REPEAT,
                start: int = 0, length: int | None = None) -> np.ndarray:
        """uint16 symbols of runs [start, start+length)."""
        if length is None:
            length = len(self) - start
        if start < 0 or length < 0 or start + length > len(self):
            raise ValueError("symbol range outside the run-length string")
        out = np.zeros(max(length, 1), dtype=np.uint16)
        chars = (c_char * max(length, 1)).from_buffer_copy(self.chars[start:start + length] or b"\0")
        cnt = np.ascontiguousarray(self.counts[start:start + length])
        if cnt.size == 0:
            cnt = np.zeros(1, dtype=np.uint32)
        _lib.check(_lib.load().mp_rle_symbols(chars, _lib.ptr(cnt, c_uint32), length, 1 if include_counts else 0,
                                              max_repeat_exclusive, _lib.ptr(out, c_uint16)))
        return out[:length]

    def non_rle_to_rle(self) -> np.ndarray:
        """rleString_getNonRleToRleCoordinateMap (impl/polisher.c:1718-1730)."""
        return np.repeat(np.arange(len(self), dtype=np.int64), self.counts.astype(np.int64))


def rle_anchors(pairs: np.ndarray, x: RleString, y: RleString) -> np.ndarray:
    """Base-level aligned pairs (n, 3: x, y, expansion) -> strictly increasing RLE anchors (m, 3) int32."""
    pairs = np.ascontiguousarray(pairs, dtype=np.int64).reshape(-1, 3)
    n = pairs.shape[0]
    out = np.zeros((max(n, 1), 3), dtype=np.int32)
    m = c_int64(0)
    xc = np.ascontiguousarray(x.counts, dtype=np.uint32)
    yc = np.ascontiguousarray(y.counts, dtype=np.uint32)
    _lib.check(_lib.load().mp_rle_anchors(_lib.ptr(pairs, c_int64), n, _lib.ptr(xc, c_uint32), len(x),
                                          _lib.ptr(yc, c_uint32), len(y), _lib.ptr(out, c_int32), m))
    return out[:m.value].copy()


def crop_range(anchors: np.ndarray, template_length: int, read_length: int) -> tuple[int, int]:
    """Template crop of getAlignedPairsWithIndelsCroppingReference (impl/polisher.c:613-628)."""
    a = np.ascontiguousarray(anchors, dtype=np.int32).reshape(-1, 3)
    s, e = c_int64(0), c_int64(0)
    _lib.check(_lib.load().mp_crop_range(_lib.ptr(a, c_int32) if a.size else None, a.shape[0], template_length,
                                         read_length, s, e))
    return s.value, e.value
