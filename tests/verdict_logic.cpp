// CPU check of the per-view measurement the verdict kernel computes
// (finish_view and bounded_refinement of csrc/common.cuh, host and device)
// against the oracle's restatements (bo_finish_view, bo_bounded_refinement,
// pinned to the reference's evaluate goldens): field by field, bit for bit.
// Prints "finish_view <cases> <mismatches>" and "refinement <cases>
// <mismatches>"; exit 0 only without mismatches.
#include "../blitzremesher_b200/csrc/common.cuh"
#include "../oracle/blitz_oracle.h"

#include <cstdio>
#include <cstring>
#include <random>

using namespace b200;

static bool same_bits(double a, double b) { return std::memcmp(&a, &b, 8) == 0; }

int main() {
    std::mt19937_64 rng(4242);
    uint64_t cases = 0, bad = 0;
    const uint32_t sss[] = {1, 2, 4, 8, 16, 32};
    for (int t = 0; t < 200000; ++t) {
        ViewRecord r{};
        r.total = uint32_t(rng() % 5000000);
        r.changed = t % 7 == 0 ? 0 : (r.total ? uint32_t(rng() % (r.total + 1)) : 0);
        r.ca = uint8_t(rng() % 8 != 0), r.cb = uint8_t(rng() % 8 != 0);
        const uint64_t k = rng() % 4;
        r.max_d2 = k == 0 ? uint32_t(rng() % 64) : (k == 1 ? uint32_t(rng() % 100000) : uint32_t(rng() % (1u << 24)));
        r.flags = uint8_t((rng() % 10 == 0 ? kRecClippedRef : 0) | (rng() % 10 == 0 ? kRecClippedCand : 0));
        GateSettings g{};
        g.limit = (rng() % 1000) / 250.0;
        g.max_changed_area = (rng() % 1001) / 1000.0;
        g.conservative_screen = uint8_t(rng() % 4 == 0);
        const uint32_t ss = sss[rng() % 6];
        Measurement m = default_measurement();
        finish_view(m, r, g, ss, double(r.max_d2));
        bo_view_record o{};
        o.max_d2 = double(r.max_d2), o.changed = r.changed, o.total = r.total, o.ca = r.ca, o.cb = r.cb;
        o.same = r.changed == 0;
        o.clipped_ref = (r.flags & kRecClippedRef) != 0, o.clipped_cand = (r.flags & kRecClippedCand) != 0;
        bo_eval_settings s{};
        s.limit = g.limit, s.max_changed_area = g.max_changed_area, s.conservative_screen = g.conservative_screen;
        s.supersample = s.max_supersample = uint8_t(ss);
        bo_measurement w{};
        bo_finish_view(&o, &s, uint8_t(ss), &w);
        ++cases;
        bad += !(same_bits(m.error, w.error) && same_bits(m.coverage, w.coverage) &&
                 same_bits(m.coverage_upper, w.coverage_upper) && same_bits(m.changed_area, w.changed_area) &&
                 m.supersample == w.supersample && m.passed == w.passed);
    }
    printf("finish_view %llu %llu\n", (unsigned long long)cases, (unsigned long long)bad);
    uint64_t rc = 0, rbad = 0;
    for (int t = 0; t < 20000; ++t) {
        const double screen = t % 5 == 0 ? double(rng() % 16385) : (rng() % 1000000) / 97.0;
        const uint32_t ss = sss[rng() % 6], mx = sss[rng() % 6];
        if (mx < ss) continue;
        ++rc;
        rbad += bounded_refinement(screen, ss, mx) != bo_bounded_refinement(screen, uint8_t(ss), uint8_t(mx));
    }
    printf("refinement %llu %llu\n", (unsigned long long)rc, (unsigned long long)rbad);
    return bad || rbad ? 1 : 0;
}
