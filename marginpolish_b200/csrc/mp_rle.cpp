// Host-side run-length encoding, symbol strings and run-length anchors
// (inputs of the realignment pass; integer logic, bit-exact with the reference).
#include "../../include/mpgpu.h"

#include <cstdint>
#include <string>
#include <vector>

extern "C" mp_status mp_rle_encode(const char *s, int64_t n, char *runChars, uint32_t *runCounts, int64_t *nRuns) {
    if ((!s && n > 0) || n < 0 || !nRuns) return MP_ERR_ARGUMENT;
    int64_t r = 0;
    uint32_t k = 1;
    for (int64_t i = 0; i < n; i++) {
        // a run ends at the last character or where the next character differs (case-sensitive)
        if (i + 1 == n || s[i] != s[i + 1]) {
            runChars[r] = s[i];
            runCounts[r] = k;
            r++;
            k = 1;
        } else {
            k++;
        }
    }
    *nRuns = r;
    return MP_OK;
}

static inline uint16_t baseSymbol(char c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 4;
    }
}

extern "C" mp_status mp_rle_symbols(const char *runChars, const uint32_t *runCounts, int64_t n, int includeCounts,
                                    uint32_t maxExclusive, uint16_t *out) {
    if (n < 0 || (n > 0 && (!runChars || !out || (includeCounts && !runCounts)))) return MP_ERR_ARGUMENT;
    if (includeCounts && (maxExclusive < 1 || maxExclusive > 256)) return MP_ERR_ARGUMENT;
    for (int64_t i = 0; i < n; i++) {
        uint16_t b = baseSymbol(runChars[i]);
        if (includeCounts) {
            uint64_t rl = runCounts[i];
            if (rl >= maxExclusive) rl = maxExclusive - 1;
            out[i] = (uint16_t) ((rl << 8) | b);
        } else {
            out[i] = b;
        }
    }
    return MP_OK;
}

extern "C" mp_status mp_rle_anchors(const int64_t *pairs, int64_t n, const uint32_t *xCounts, int64_t xRuns,
                                    const uint32_t *yCounts, int64_t yRuns, int32_t *out, int64_t *nOut) {
    if (n < 0 || !nOut || (n > 0 && (!pairs || !out || !xCounts || !yCounts))) return MP_ERR_ARGUMENT;
    std::vector<int64_t> xMap, yMap;
    for (int64_t i = 0; i < xRuns; i++) xMap.insert(xMap.end(), xCounts[i], i);
    for (int64_t i = 0; i < yRuns; i++) yMap.insert(yMap.end(), yCounts[i], i);
    int64_t x = -1, y = -1, k = 0;
    for (int64_t i = 0; i < n; i++) {
        int64_t px = pairs[3 * i], py = pairs[3 * i + 1];
        if (px < 0 || py < 0 || px >= (int64_t) xMap.size() || py >= (int64_t) yMap.size()) return MP_ERR_ARGUMENT;
        int64_t x2 = xMap[px], y2 = yMap[py];
        if (x2 > x && y2 > y) {
            out[3 * k] = (int32_t) x2;
            out[3 * k + 1] = (int32_t) y2;
            out[3 * k + 2] = (int32_t) pairs[3 * i + 2];
            k++;
            x = x2;
            y = y2;
        }
    }
    *nOut = k;
    return MP_OK;
}
