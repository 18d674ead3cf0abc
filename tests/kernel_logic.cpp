// CPU check of two pieces of the audit kernels' exact logic, compiled from
// the same headers the CUDA library uses (csrc/common.cuh, csrc/nearest.cuh):
//  1. face_interval: per row, the binary searches over the FP64 edge terms
//     return exactly the samples face_covers accepts (one interval or none);
//  2. nearest_d2: the outward, boxed row search returns the brute-force
//     squared distance to the nearest covered sample (or, with `enough`, a
//     value <= enough whenever the true distance is <= enough).
// Prints "intervals <rows checked> <mismatches>" and "nearest <queries>
// <mismatches>"; exit status 0 only without mismatches.
#include "../blitzremesher_b200/csrc/nearest.cuh"

#include <cstdio>
#include <random>
#include <vector>

using namespace b200;

struct HostMask {
    std::vector<uint8_t> bit;
    uint32_t size;
    uint32_t chunk(uint32_t row, uint32_t c) const {
        uint32_t v = 0;
        for (uint32_t i = 0; i < 32; ++i) {
            const uint32_t x = c * 32 + i;
            if (x < size && bit[size_t(row) * size + x]) v |= 1u << i;
        }
        return v;
    }
};

static uint64_t brute_nearest(const HostMask& m, uint32_t x, uint32_t y) {
    uint64_t best = kNone;
    for (uint32_t yy = 0; yy < m.size; ++yy)
        for (uint32_t xx = 0; xx < m.size; ++xx)
            if (m.bit[size_t(yy) * m.size + xx]) {
                const int64_t dx = int64_t(xx) - x, dy = int64_t(yy) - y;
                const uint64_t d = uint64_t(dx * dx + dy * dy);
                if (d < best) best = d;
            }
    return best;
}

int main() {
    std::mt19937_64 rng(20261203);
    auto uni = [&](double lo, double hi) { return lo + (hi - lo) * double(rng() >> 11) * (1.0 / 9007199254740992.0); };
    // 1. intervals
    uint64_t rows = 0, bad_rows = 0;
    for (int t = 0; t < 6000; ++t) {
        const uint32_t size = t % 3 == 0 ? 4160 : (t % 3 == 1 ? 256 : 64);
        const double span = t % 4 == 0 ? size * 0.9 : (t % 4 == 1 ? 40.0 : (t % 4 == 2 ? 3.0 : 0.7));
        const double cx = uni(span, size - span > span ? size - span : span + 1);
        const double cy = uni(span, size - span > span ? size - span : span + 1);
        Proj p[3];
        for (auto& q : p) q = Proj{cx + uni(-span, span), cy + uni(-span, span), 1.0};
        if (t % 7 == 0) p[2] = Proj{p[0].x + (p[1].x - p[0].x) * 0.5, p[0].y + (p[1].y - p[0].y) * 0.5 + 1e-7, 1.0};
        // edges through sample centres (ties of the edge test), horizontal and
        // vertical edges
        if (t % 11 == 1)
            for (auto& q : p) q.x = std::floor(q.x) + .5, q.y = std::floor(q.y) + .5;
        if (t % 13 == 2) p[1].y = p[0].y;
        if (t % 17 == 3) p[2].x = p[1].x;
        const FaceSetup s = setup_face(p[0], p[1], p[2], false, t % 2 == 0, size);
        if (s.status != kFaceOk) continue;
        const int step = s.y1 - s.y0 > 400 ? 37 : 1;
        for (int y = s.y0; y <= s.y1; y += step) {
            int lo, hi;
            face_interval(s, double(y) + .5, lo, hi);
            bool ok = true;
            for (int x = s.x0; x <= s.x1 && ok; ++x) ok = face_covers(s, x, y) == (x >= lo && x <= hi);
            // the interval searched from the edges' guessed crossings, and
            // from arbitrary guesses, is the same set
            int glo, ghi;
            face_interval_guess(s, double(y) + .5, glo, ghi);
            const bool empty = lo > hi;
            ok = ok && (empty ? glo > ghi : (glo == lo && ghi == hi));
            int guess[3];
            const int span_x = s.x1 - s.x0 + 3;
            for (int e = 0; e < 3; ++e)
                guess[e] = t % 3 == 0 ? int(rng() % 20000) - 10000 : s.x0 - 1 + int(rng() % uint64_t(span_x));
            face_interval_at(s, double(y) + .5, guess, glo, ghi);
            ok = ok && (empty ? glo > ghi : (glo == lo && ghi == hi));
            ++rows;
            bad_rows += !ok;
        }
    }
    printf("intervals %llu %llu\n", (unsigned long long)rows, (unsigned long long)bad_rows);
    // 2. nearest covered sample
    uint64_t queries = 0, bad_queries = 0;
    for (int t = 0; t < 240; ++t) {
        HostMask m;
        m.size = 16 + uint32_t(rng() % 200);
        if (t % 40 == 0) m.size = 700;
        m.bit.assign(size_t(m.size) * m.size, 0);
        const int kind = t % 4;
        if (kind == 0) {
            for (auto& b : m.bit) b = rng() % 1000 < 3;
        } else if (kind == 1) {
            const double cx = uni(0, m.size), cy = uni(0, m.size), r = uni(0, m.size * 0.6);
            for (uint32_t y = 0; y < m.size; ++y)
                for (uint32_t x = 0; x < m.size; ++x)
                    m.bit[size_t(y) * m.size + x] = (x - cx) * (x - cx) + (y - cy) * (y - cy) <= r * r;
        } else if (kind == 3) {
            m.bit[size_t(rng() % m.size) * m.size + rng() % m.size] = 1;
        }
        for (int q = 0; q < 50; ++q) {
            const uint32_t x = uint32_t(rng() % m.size), y = uint32_t(rng() % m.size);
            const uint32_t enough = q % 3 == 0 ? uint32_t(rng() % 60) : 0;
            const uint64_t want = brute_nearest(m, x, y);
            const uint32_t got = nearest_d2(m, x, y, enough);
            bool ok;
            if (want == kNone) ok = got == kNone;
            else if (enough && want <= enough) ok = got >= want && got <= enough;
            else ok = got == want;
            // with a cap: the same answer when the nearest is within it, else
            // cap + 1 (also for an empty mask)
            const uint32_t cap = q % 2 ? uint32_t(rng() % (4ull * m.size * m.size)) : uint32_t(rng() % 50);
            const uint32_t capped = nearest_d2(m, x, y, enough, cap);
            if (want == kNone || want > cap) ok = ok && capped == cap + 1;
            else if (enough && want <= enough) ok = ok && capped >= want && capped <= enough;
            else ok = ok && capped == want;
            ++queries;
            bad_queries += !ok;
        }
    }
    printf("nearest %llu %llu\n", (unsigned long long)queries, (unsigned long long)bad_queries);
    return bad_rows || bad_queries ? 1 : 0;
}
