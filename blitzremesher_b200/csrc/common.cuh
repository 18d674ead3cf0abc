// Shared host/device definitions for the B200 candidate-audit engine.
//
// Everything here compiles both under nvcc (device + host) and under a plain
// C++ compiler (for CPU unit checks of the index and FP64 logic). FP64
// expressions are written in the reference's evaluation order; the library is
// built with --fmad=false / -ffp-contract=off so no product is fused.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define BH __host__ __device__ __forceinline__
#else
#define BH inline
#endif

namespace b200 {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint64_t kMaxSamples = 64000000ull; // evaluate.cpp:129
constexpr uint32_t kExactLimit = 1u << 24;    // squared distances exact in the CPU float field

struct Camera {
    float right[3], up[3], forward[3];
    double distance, focal, scale;
    uint32_t perspective;
    uint32_t pad;
};

struct Proj {
    double x, y, z;
};

// evaluate.cpp:137-141 — FP64 projection into sample space.
BH Proj project(float px, float py, float pz, const float* center, const Camera& c, uint32_t ss,
                uint32_t size) {
    double x = double(px) - double(center[0]), y = double(py) - double(center[1]),
           z0 = double(pz) - double(center[2]);
    double df = x * double(c.forward[0]) + y * double(c.forward[1]) + z0 * double(c.forward[2]);
    double dr = x * double(c.right[0]) + y * double(c.right[1]) + z0 * double(c.right[2]);
    double du = x * double(c.up[0]) + y * double(c.up[1]) + z0 * double(c.up[2]);
    double z = c.distance - df, sc = c.perspective ? c.focal / z : c.scale;
    Proj p;
    p.x = dr * sc * double(ss) + double(size) * .5;
    p.y = du * sc * double(ss) + double(size) * .5;
    p.z = z;
    return p;
}

BH double edge_fn(double ax, double ay, double bx, double by, double x, double y) {
    return (bx - ax) * (y - ay) - (by - ay) * (x - ax);
}

enum FaceStatus : int32_t { kFaceOk = 0, kFaceCulled = 1, kFaceClipZ = 2, kFaceClipBox = 3 };

// Triangle setup of evaluate.cpp:146-165: cull, orient, bbox, L1 slacks.
struct FaceSetup {
    double ax, ay, dx, dy, ex, ey, r0, r1, r2;
    int32_t x0, x1, y0, y1;
    int32_t status;
    int32_t pad;
};

BH double fmin3(double a, double b, double c) { return a < b ? (a < c ? a : c) : (b < c ? b : c); }
BH double fmax3(double a, double b, double c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }

BH FaceSetup setup_face(Proj a, Proj d, Proj e, bool perspective, bool two, uint32_t size) {
    FaceSetup s;
    s.x0 = s.y0 = 1;
    s.x1 = s.y1 = 0;
    s.ax = s.ay = s.dx = s.dy = s.ex = s.ey = s.r0 = s.r1 = s.r2 = 0;
    s.pad = 0;
    if (perspective && (a.z <= 0 || d.z <= 0 || e.z <= 0)) {
        s.status = kFaceClipZ;
        return s;
    }
    double area = edge_fn(a.x, a.y, d.x, d.y, e.x, e.y);
    if (std::fabs(area) < 1e-16) {
        s.status = kFaceCulled;
        return s;
    }
    bool back = area < 0;
    if (back && !two) {
        s.status = kFaceCulled;
        return s;
    }
    if (back) {
        Proj t = d;
        d = e;
        e = t;
    }
    // std::min/max over three doubles (evaluate.cpp:157-158): NaN ordering is
    // irrelevant because a nonfinite bound is rejected below.
    double minx = fmin3(a.x, d.x, e.x), maxx = fmax3(a.x, d.x, e.x);
    double miny = fmin3(a.y, d.y, e.y), maxy = fmax3(a.y, d.y, e.y);
    if (!std::isfinite(minx) || !std::isfinite(maxx) || !std::isfinite(miny) || !std::isfinite(maxy) ||
        minx < 0 || miny < 0 || maxx > double(size) || maxy > double(size)) {
        s.status = kFaceClipBox;
        return s;
    }
    int fx0 = int(std::floor(minx)), fx1 = int(std::floor(maxx));
    int fy0 = int(std::floor(miny)), fy1 = int(std::floor(maxy));
    s.x0 = fx0 > 0 ? fx0 : 0;
    s.x1 = fx1 < int(size) - 1 ? fx1 : int(size) - 1;
    s.y0 = fy0 > 0 ? fy0 : 0;
    s.y1 = fy1 < int(size) - 1 ? fy1 : int(size) - 1;
    s.ax = a.x, s.ay = a.y, s.dx = d.x, s.dy = d.y, s.ex = e.x, s.ey = e.y;
    s.r0 = .5 * (std::fabs(e.x - d.x) + std::fabs(e.y - d.y));
    s.r1 = .5 * (std::fabs(a.x - e.x) + std::fabs(a.y - e.y));
    s.r2 = .5 * (std::fabs(d.x - a.x) + std::fabs(d.y - a.y));
    s.status = kFaceOk;
    return s;
}

// Conservative coverage test at a sample centre (evaluate.cpp:166-168).
BH bool face_covers(const FaceSetup& s, int x, int y) {
    double px = double(x) + .5, py = double(y) + .5;
    double u = edge_fn(s.dx, s.dy, s.ex, s.ey, px, py);
    if (u + s.r0 < 0) return false;
    double v = edge_fn(s.ex, s.ey, s.ax, s.ay, px, py);
    if (v + s.r1 < 0) return false;
    double w = edge_fn(s.ax, s.ay, s.dx, s.dy, px, py);
    return !(w + s.r2 < 0);
}

// Covered samples [lo, hi] of row py - .5 of face s (lo > hi: none), from
// s's bbox columns: each edge term of face_covers is monotone in x, so a
// binary search per edge finds the interval's ends with the same FP64
// expressions.
BH void face_interval(const FaceSetup& s, double py, int& lo, int& hi) {
    lo = s.x0, hi = s.x1;
    // edge (d, e), edge (e, a), edge (a, d) of face_covers
    const double ax3[3] = {s.dx, s.ex, s.ax}, ay3[3] = {s.dy, s.ey, s.ay};
    const double bx3[3] = {s.ex, s.ax, s.dx}, by3[3] = {s.ey, s.ay, s.dy};
    const double r3[3] = {s.r0, s.r1, s.r2};
    for (int e = 0; e < 3 && lo <= hi; ++e) {
        const double ax = ax3[e], ay = ay3[e], r = r3[e];
        const double t1 = (bx3[e] - ax) * (py - ay), c = by3[e] - ay;
        // covered(x) = !((t1 - c * (x + .5 - ax)) + r < 0)
        auto ok = [&](int x) { return !((t1 - c * ((double(x) + .5) - ax)) + r < 0); };
        if (c > 0) { // true then false: last covered x
            if (!ok(lo)) {
                hi = lo - 1;
                break;
            }
            int a = lo, b = hi;
            while (a < b) {
                const int m = a + (b - a + 1) / 2;
                if (ok(m)) a = m;
                else b = m - 1;
            }
            hi = a;
        } else if (c < 0) { // false then true: first covered x
            if (!ok(hi)) {
                hi = lo - 1;
                break;
            }
            int a = lo, b = hi;
            while (a < b) {
                const int m = a + (b - a) / 2;
                if (ok(m)) b = m;
                else a = m + 1;
            }
            lo = a;
        } else if (!ok(lo)) {
            hi = lo - 1;
        }
    }
}

// The same interval from guessed edge boundaries: per edge of face_covers
// the covered samples of a row are a prefix (c >= 0: up to the last covered
// x, x0 - 1 when none) or a suffix (c < 0: from the first covered x, x1 + 1
// when none) of the face's bbox columns. From any guess, an exponential
// search brackets the boundary and a binary search over the same FP64 edge
// expressions settles it exactly, so [max of suffix starts, min of prefix
// ends] equals face_interval's interval (lo > hi: none) whatever `guess`
// holds; a good guess takes one or two tests per edge.
BH void face_interval_at(const FaceSetup& s, double py, const int guess[3], int& lo, int& hi) {
    const double ax3[3] = {s.dx, s.ex, s.ax}, ay3[3] = {s.dy, s.ey, s.ay};
    const double bx3[3] = {s.ex, s.ax, s.dx}, by3[3] = {s.ey, s.ay, s.dy};
    const double r3[3] = {s.r0, s.r1, s.r2};
    double t1[3], c[3];
    bool prefix[3];
    int last[3]; // per edge the last column whose test equals `prefix`: the boundary
    bool settled[3];
    // One column's test, the out-of-range columns as sentinels: left of the
    // bbox a prefix is covered and a suffix is not, right of it the other
    // way round.
    // (px = double(x) + 1/2, exact, as evaluate.cpp's sample centre)
    auto ok_at = [&](int e, int x, double px) {
        const bool covered = !((t1[e] - c[e] * (px - ax3[e])) + r3[e] < 0);
        return x < s.x0 ? prefix[e] : (x > s.x1 ? !prefix[e] : covered);
    };
    auto ok = [&](int e, int x) { return ok_at(e, x, double(x) + .5); };
    // The three columns around each guess, for all edges at once (no
    // branches: independent tests); most boundaries are settled there.
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        t1[e] = (bx3[e] - ax3[e]) * (py - ay3[e]);
        c[e] = by3[e] - ay3[e];
        prefix[e] = c[e] >= 0; // c == 0: every column or none
        const int g = guess[e] < s.x0 - 1 ? s.x0 - 1 : (guess[e] > s.x1 + 1 ? s.x1 + 1 : guess[e]);
        const double pg = double(g) + .5; // g - 1 and g + 1 are pg -/+ 1, exactly
        const bool before = ok_at(e, g - 1, pg - 1.0) == prefix[e], at = ok_at(e, g, pg) == prefix[e],
                   after = ok_at(e, g + 1, pg + 1.0) == prefix[e];
        settled[e] = (at && !after) || (!at && before);
        last[e] = at ? g : g - 1;
    }
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        if (settled[e]) continue;
        const int g = guess[e] < s.x0 - 1 ? s.x0 - 1 : (guess[e] > s.x1 + 1 ? s.x1 + 1 : guess[e]);
        // Bracket [a, b] with ok(a) == prefix and ok(b) != prefix, then bisect.
        int a, b;
        if (ok(e, g) == prefix[e]) {
            a = g;
            for (int step = 1;; step *= 2) {
                b = a + step;
                if (b >= s.x1 + 1) {
                    b = s.x1 + 1;
                    break;
                }
                if (ok(e, b) != prefix[e]) break;
                a = b;
            }
        } else {
            b = g;
            for (int step = 1;; step *= 2) {
                a = b - step;
                if (a <= s.x0 - 1) {
                    a = s.x0 - 1;
                    break;
                }
                if (ok(e, a) == prefix[e]) break;
                b = a;
            }
        }
        while (b - a > 1) {
            const int m = a + (b - a) / 2;
            if (ok(e, m) == prefix[e]) a = m;
            else b = m;
        }
        last[e] = a;
    }
    lo = s.x0, hi = s.x1;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        if (prefix[e]) hi = last[e] < hi ? last[e] : hi; // last covered
        else lo = last[e] + 1 > lo ? last[e] + 1 : lo;   // first covered
    }
}

// face_interval_at with each edge's boundary guessed from its crossing
// x* = (t1 + r) / c + ax - 1/2 in single precision (within a small fraction
// of a sample of the exact one; the searches settle it).
BH void face_interval_guess(const FaceSetup& s, double py, int& lo, int& hi) {
    const double ax3[3] = {s.dx, s.ex, s.ax}, ay3[3] = {s.dy, s.ey, s.ay};
    const double bx3[3] = {s.ex, s.ax, s.dx}, by3[3] = {s.ey, s.ay, s.dy};
    const double r3[3] = {s.r0, s.r1, s.r2};
    int guess[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const double c = by3[e] - ay3[e];
        const float num = float((bx3[e] - ax3[e]) * (py - ay3[e]) + r3[e]), den = float(c);
#ifdef __CUDA_ARCH__
        float xs = __fdividef(num, den) + float(ax3[e]) - .5f;
#else
        float xs = num / den + float(ax3[e]) - .5f;
#endif
        // NaN, infinities and far crossings clamp to the sentinels
        xs = fmaxf(xs, float(s.x0 - 1));
        xs = fminf(xs, float(s.x1 + 1));
        guess[e] = c == 0 ? s.x0 : (c > 0 ? int(floorf(xs)) : int(ceilf(xs)));
    }
    face_interval_at(s, py, guess, lo, hi);
}

// CPU float value of the field where the exact distance reaches 2^24: the
// row pass rounds g^2 to float, the column pass rounds (dy^2 + f) to float;
// the lower envelope of the reference picks the smallest such value. `g`:
// per row the distance to its nearest covered sample in column x (kNone:
// none), row stride `width`.
BH float cpu_field_value(const uint32_t* g, uint32_t width, uint32_t height, uint32_t x, uint32_t y) {
    float best = INFINITY;
    for (uint32_t q = 0; q < height; ++q) {
        uint32_t gq = g[size_t(q) * width + x];
        if (gq == kNone) continue;
#if defined(__CUDA_ARCH__)
        float f = __uint2float_rn(gq * gq);
#else
        float f = float(gq * gq);
#endif
        double dy = double(y) - double(q);
#if defined(__CUDA_ARCH__)
        float val = __double2float_rn(dy * dy + double(f));
#else
        float val = float(dy * dy + double(f));
#endif
        best = val < best ? val : best;
    }
    return best;
}

// Raw per-(candidate, view) audit record consumed by finish_view.
struct ViewRecord {
    uint32_t max_d2;  // max squared distance over XOR samples (exact integer)
    uint32_t changed; // popcount(reference ^ candidate)
    uint32_t total;   // popcount(reference | candidate)
    uint8_t ca, cb;   // reference / candidate cover anything
    uint8_t flags;    // kRecClippedRef | kRecClippedCand | kRecFallback | kRecLarge
    uint8_t pad;
};
constexpr uint8_t kRecClippedRef = 1, kRecClippedCand = 2, kRecFallback = 4, kRecLarge = 8;

struct Measurement {
    double error, coverage, coverage_upper, changed_area, normal_degrees;
    uint32_t worst_view, changed_area_worst_view, views_evaluated;
    uint8_t supersample, complete, passed, resource_limited, cancelled;
    uint8_t reserved[3];
};

struct GateSettings {
    double screen_size, limit, max_changed_area;
    uint32_t views; // number of cameras
    uint8_t supersample, max_supersample, conservative_screen, pad;
};

BH Measurement default_measurement() {
    Measurement m{};
    m.error = m.coverage = m.coverage_upper = m.changed_area = m.normal_degrees = 0;
    m.worst_view = m.changed_area_worst_view = m.views_evaluated = 0;
    m.supersample = 0;
    m.complete = 1;
    m.passed = 1;
    m.resource_limited = 0;
    m.cancelled = 0;
    m.reserved[0] = m.reserved[1] = m.reserved[2] = 0;
    return m;
}

BH double coverage_value(const ViewRecord& r, uint32_t ss, double max_d2) {
    if (r.changed == 0) return 0;                     // same masks (evaluate.cpp:202)
    if (r.ca != r.cb) return INFINITY;                // one side empty
    return std::sqrt(max_d2) / double(ss);
}

// finish_view, coverage profile (evaluate.cpp:271-298). `max_d2` is the CPU
// float field maximum promoted to double.
BH void finish_view(Measurement& cur, const ViewRecord& r, const GateSettings& s, uint32_t ss,
                    double max_d2) {
    cur.supersample = uint8_t(ss);
    cur.coverage = coverage_value(r, ss, max_d2);
    cur.coverage_upper = cur.coverage + 2 * std::sqrt(2.0) / double(ss) + 1e-6;
    bool clipped = (r.flags & (kRecClippedRef | kRecClippedCand)) != 0;
    if (clipped) cur.coverage_upper = INFINITY;
    cur.error = cur.coverage_upper;
    cur.changed_area = r.total ? double(r.changed) / double(r.total) : 0;
    cur.passed = cur.error <= s.limit && cur.changed_area <= s.max_changed_area;
    if (s.conservative_screen) {
        double lower = cur.coverage - 2 * std::sqrt(2.0) / double(ss) - 1e-6;
        cur.error = clipped ? 0 : (lower > 0.0 ? lower : 0.0);
        cur.passed = cur.error <= s.limit;
    }
}

// Refinement stop rule of evaluate.cpp:336-337.
BH bool refinement_done(const Measurement& cur, const GateSettings& s, uint32_t ss) {
    return s.conservative_screen || cur.passed || ss >= s.max_supersample ||
           cur.coverage - 2 * std::sqrt(2.0) / double(ss) > s.limit || !std::isfinite(cur.error) ||
           cur.coverage_upper <= s.limit;
}

// Aggregation of one finished view into the result (evaluate.cpp:340-349).
// Returns false when the audit stops at this view.
BH bool aggregate_view(Measurement& result, const Measurement& cur, uint32_t v) {
    ++result.views_evaluated;
    if (cur.error > result.error) {
        result.worst_view = v;
        result.error = cur.error;
        result.supersample = cur.supersample;
    }
    if (cur.coverage > result.coverage) result.coverage = cur.coverage;
    if (cur.coverage_upper > result.coverage_upper) result.coverage_upper = cur.coverage_upper;
    if (cur.changed_area > result.changed_area) {
        result.changed_area = cur.changed_area;
        result.changed_area_worst_view = v;
    }
    if (cur.normal_degrees > result.normal_degrees) result.normal_degrees = cur.normal_degrees;
    if (!cur.passed) {
        result.passed = 0;
        result.complete = 0;
        return false;
    }
    return true;
}

// audit_measurement.hpp:8-17
BH bool measurement_accepted(const Measurement& m) {
    bool nonfinite = std::isnan(m.error) || std::isnan(m.coverage) || std::isnan(m.coverage_upper) ||
                     !std::isfinite(m.changed_area) || !std::isfinite(m.normal_degrees) ||
                     (m.passed && (!std::isfinite(m.error) || !std::isfinite(m.coverage) ||
                                   !std::isfinite(m.coverage_upper)));
    return m.complete && m.passed && !m.cancelled && !m.resource_limited && !nonfinite;
}

// graph.cpp:5-18
BH uint32_t bounded_refinement(double screen, uint32_t ss, uint32_t max_ss) {
    uint64_t side = uint64_t(std::ceil(screen + 8));
    while (ss < max_ss) {
        uint32_t next = ss * 2 < max_ss ? ss * 2 : max_ss;
        if (side * side * next * next > kMaxSamples) break;
        ss = next;
    }
    return ss;
}

BH uint32_t raster_size(double screen, uint32_t ss) { return uint32_t(std::ceil(screen + 8)) * ss; }

// Position key with zero signs folded (action.cpp:8-12).
BH uint32_t position_bits(float f) {
    float g = f == 0.f ? 0.f : f;
    uint32_t u;
    std::memcpy(&u, &g, 4);
    return u;
}
BH uint32_t hash_position(uint32_t bx, uint32_t by, uint32_t bz) {
    uint32_t h = bx * 0x9e3779b9u;
    h = (h ^ by) * 0x85ebca6bu;
    h = (h ^ bz) * 0xc2b2ae35u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}

} // namespace b200
