// CPU check of the distance field values the audit reports: below 2^24 the
// exact integer squared distance equals the reference's float field (as the
// oracle computes it, evaluate.cpp:33-70); from 2^24 up, cpu_field_value
// (csrc/common.cuh) reproduces the float field's roundings. On a 4160 x 4160
// raster with covered samples in one corner, so that the far corner is
// beyond 2^24. Prints "field <samples> <exact-regime mismatches> <rounded-
// regime mismatches> <rounded-regime samples>"; exit 0 only without
// mismatches.
#include "../blitzremesher_b200/csrc/common.cuh"
#include "../oracle/blitz_oracle.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

using namespace b200;

int main() {
    const uint32_t W = 4160, H = 4160;
    std::mt19937_64 rng(99);
    std::vector<std::pair<uint32_t, uint32_t>> pts; // covered samples (x, y)
    for (int i = 0; i < 40; ++i) pts.push_back({uint32_t(rng() % 300), uint32_t(rng() % 300)});
    for (int i = 0; i < 6; ++i) pts.push_back({uint32_t(rng() % 1500), uint32_t(rng() % 200)});
    std::vector<uint64_t> words((size_t(W) * H + 63) / 64, 0);
    std::vector<std::vector<uint32_t>> row_x(H);
    for (auto [x, y] : pts) {
        const size_t i = size_t(y) * W + x;
        words[i / 64] |= uint64_t(1) << (i % 64);
        row_x[y].push_back(x);
    }
    std::vector<float> field(size_t(W) * H);
    if (bo_distance_field(words.data(), W, H, field.data()) != 0) return 2;
    uint64_t n = 0, bad_exact = 0, bad_round = 0, rounded = 0;
    std::vector<uint32_t> g(size_t(H) * W, kNone); // filled per queried column
    for (int t = 0; t < 3000; ++t) {
        const uint32_t x = t % 2 ? W - 1 - uint32_t(rng() % 1200) : uint32_t(rng() % W);
        const uint32_t y = t % 2 ? H - 1 - uint32_t(rng() % 1200) : uint32_t(rng() % H);
        uint64_t exact = ~0ull;
        for (auto [px, py] : pts) {
            const int64_t dx = int64_t(px) - x, dy = int64_t(py) - y;
            exact = std::min<uint64_t>(exact, uint64_t(dx * dx + dy * dy));
        }
        const float want = field[size_t(y) * W + x];
        ++n;
        if (exact < kExactLimit) {
            const float got = float(exact);
            bad_exact += std::memcmp(&got, &want, 4) != 0;
        } else {
            for (uint32_t q = 0; q < H; ++q) {
                uint32_t best = kNone;
                for (uint32_t px : row_x[q]) best = std::min<uint32_t>(best, px > x ? px - x : x - px);
                g[size_t(q) * W + x] = best;
            }
            const float got = cpu_field_value(g.data(), W, H, x, y);
            ++rounded;
            bad_round += std::memcmp(&got, &want, 4) != 0;
        }
    }
    printf("field %llu %llu %llu %llu\n", (unsigned long long)n, (unsigned long long)bad_exact,
           (unsigned long long)bad_round, (unsigned long long)rounded);
    return bad_exact || bad_round ? 1 : 0;
}
