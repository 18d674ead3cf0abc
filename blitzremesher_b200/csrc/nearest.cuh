// Nearest covered sample in a packed coverage mask: the distance search of
// the incremental audit (the directed Hausdorff term of evaluate.cpp:196-209
// restricted to the changed samples). Host and device: the same code is
// compiled into the audit kernels and into the CPU tests that check it
// against brute force. `M` provides `size` (samples per row) and
// `chunk(row, c)`: bits [32c, 32c + 32) of a row, bit i = sample 32c + i.
#pragma once
#include "common.cuh"

#if defined(__CUDACC__)
#define NEAREST_HD __host__ __device__
// the mask types of the kernels are device-only; the host instantiations use
// host masks
#define NEAREST_HD_PRAGMA _Pragma("nv_exec_check_disable")
#else
#define NEAREST_HD
#define NEAREST_HD_PRAGMA
#endif

namespace b200 {

NEAREST_HD inline uint32_t bit_clz(uint32_t v) {
#if defined(__CUDA_ARCH__)
    return uint32_t(__clz(v));
#else
    return v ? uint32_t(__builtin_clz(v)) : 32u;
#endif
}
NEAREST_HD inline uint32_t bit_ffs(uint32_t v) {
#if defined(__CUDA_ARCH__)
    return uint32_t(__ffs(v));
#else
    return uint32_t(__builtin_ffs(int(v)));
#endif
}

// Smallest |dx| <= maxdx with a covered sample at (x+dx, row); kNone if none.
// The two sides are scanned one chunk each per step, outward, so the scan
// ends near the nearest covered sample instead of at a row end.
NEAREST_HD_PRAGMA
template <class M> NEAREST_HD inline uint32_t nearest_in_row(const M& mask, uint32_t row, uint32_t x, uint32_t maxdx) {
    const uint32_t cx = x >> 5, bx = x & 31;
    uint32_t best = kNone;
    const uint32_t w = mask.chunk(row, cx);
    const uint32_t left = w & (bx == 31 ? 0xffffffffu : ((2u << bx) - 1u));
    const uint32_t right = w & (0xffffffffu << bx);
    if (left) best = bx - (31 - bit_clz(left));
    if (right) {
        const uint32_t d = (bit_ffs(right) - 1) - bx;
        best = d < best ? d : best;
    }
    if (best == 0) return 0;
    const uint32_t chunks = (mask.size + 31) >> 5;
    bool go_left = cx > 0, go_right = cx + 1 < chunks;
    for (uint32_t k = 1; go_left || go_right; ++k) {
        if (go_left) {
            const uint32_t c = cx - k;
            const uint32_t nearest = x - (c * 32 + 31);
            if (nearest > maxdx || nearest >= best) {
                go_left = false;
            } else {
                const uint32_t v = mask.chunk(row, c);
                if (v) {
                    const uint32_t d = x - (c * 32 + (31 - bit_clz(v)));
                    best = d < best ? d : best;
                    go_left = false;
                } else if (c == 0) {
                    go_left = false;
                }
            }
        }
        if (go_right) {
            const uint32_t c = cx + k;
            const uint32_t nearest = c * 32 - x;
            if (nearest > maxdx || nearest >= best) {
                go_right = false;
            } else {
                const uint32_t v = mask.chunk(row, c);
                if (v) {
                    const uint32_t d = c * 32 + (bit_ffs(v) - 1) - x;
                    best = d < best ? d : best;
                    go_right = false;
                } else if (c + 1 >= chunks) {
                    go_right = false;
                }
            }
        }
    }
    return best <= maxdx ? best : kNone;
}

// Exact squared Euclidean distance from (x, y) to the nearest covered sample
// (kNone: none), or any value <= `enough` once a covered sample that close is
// found (the caller only needs distances above `enough`: the running
// maximum), or cap + 1 when no covered sample lies within squared distance
// `cap` (the caller only needs to know that it is farther; cap = UINT32_MAX:
// no cap). The search runs in boxes of half-width R = 32, 128, ...: rows are
// scanned up to R columns until a covered sample is found, and then within
// its distance; a result <= R^2 (or <= enough) is final, since every sample
// left out of the box is farther than R. With a cap the last box reaches
// floor(sqrt(cap)) + 1, beyond which every sample is farther than the cap.
NEAREST_HD_PRAGMA
template <class M>
NEAREST_HD inline uint32_t nearest_d2(const M& mask, uint32_t x, uint32_t y, uint32_t enough = 0,
                                      uint32_t cap = 0xffffffffu) {
    const uint32_t size = mask.size;
    const bool capped = cap != 0xffffffffu;
    uint32_t reach = size;
    if (capped) {
        uint64_t r = uint64_t(sqrt(double(cap)));
        while (r * r > cap) --r;
        while ((r + 1) * (r + 1) <= cap) ++r;
        reach = r + 1 < size ? uint32_t(r + 1) : size;
    }
    for (uint32_t R = 32;; R *= 4) {
        const bool last = R >= reach;
        const uint32_t box = last ? reach : R;
        uint32_t best = kNone;
        for (uint32_t dy = 0;; ++dy) {
            const uint64_t dy2 = uint64_t(dy) * dy;
            if (best != kNone && (dy2 >= best || best <= enough)) break;
            if (dy > box && (best == kNone || last)) break;
            bool any = false;
            for (int side = 0; side < (dy ? 2 : 1); ++side) {
                const int64_t row = side ? int64_t(y) + dy : int64_t(y) - dy;
                if (row < 0 || row >= int64_t(size)) continue;
                any = true;
                uint32_t maxdx = best == kNone ? box : uint32_t(sqrtf(float(best - dy2))) + 1;
                if (last && maxdx > box) maxdx = box;
                const uint32_t dx = nearest_in_row(mask, uint32_t(row), x, maxdx);
                if (dx != kNone) {
                    const uint64_t d = uint64_t(dx) * dx + dy2;
                    if (d < best) best = uint32_t(d);
                }
            }
            if (!any) break;
        }
        if (last) return capped && (best == kNone || best > cap) ? cap + 1 : best;
        if (best != kNone && (best <= enough || uint64_t(best) <= uint64_t(R) * R)) return best;
    }
}

} // namespace b200
