// CPU oracle for the candidate-audit path — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement, in this project's own code, of BlitzRemesher's audit path.
// Only tests, the smoke check and the CPU-baseline leg of the benchmark use it,
// always as the checker; the CUDA product never links or calls it. Every
// function names the reference file:line it restates. Arithmetic follows the
// reference operation by operation (double vs float, evaluation order, no
// contraction: build with -ffp-contract=off -fno-fast-math), because parity is
// bit-exact.
#include "blitz_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <unordered_map>
#include <vector>

namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr uint32_t kNone = UINT32_MAX;
constexpr uint64_t kMaxSamples = 64000000; // evaluate.cpp:129, internal.hpp:11

struct V3 {
    float x, y, z;
};
V3 load3(const float* p, size_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
// mesh.hpp:23 — each component rounded to float after a double multiply.
V3 scale3(V3 a, double s) { return {float(a.x * s), float(a.y * s), float(a.z * s)}; }
// mesh.hpp:24 — products and sums in double from float inputs.
double dot(V3 a, V3 b) { return double(a.x) * b.x + double(a.y) * b.y + double(a.z) * b.z; }
// mesh.hpp:25 — float cross product.
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double length(V3 a) { return std::sqrt(dot(a, a)); }
V3 normalized(V3 a) {
    double l = length(a);
    return l > 0 ? scale3(a, 1 / l) : V3{0, 0, 0};
}
bool finite3(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

struct Mesh {
    const bo_mesh* m;
    uint32_t faces() const { return m->face_count; }
    V3 pos(uint32_t i) const { return load3(m->positions, i); }
    uint16_t material(uint32_t f) const { return m->materials ? m->materials[f] : 0; }
    // mesh.hpp:50 — two-sided iff the face's material flags it.
    bool two_sided(uint32_t f) const {
        auto mat = material(f);
        return mat < m->double_sided_count && m->double_sided && m->double_sided[mat];
    }
};

// evaluate.cpp:16-20
V3 rotate(V3 v, uint32_t seed) {
    double a = (seed % 65521) * .000731, b = ((seed >> 8) % 32749) * .000913;
    double x = v.x * std::cos(a) - v.y * std::sin(a), y = v.x * std::sin(a) + v.y * std::cos(a);
    return {float(x), float(y * std::cos(b) - v.z * std::sin(b)),
            float(y * std::sin(b) + v.z * std::cos(b))};
}
// evaluate.cpp:21
double edge_fn(double ax, double ay, double bx, double by, double x, double y) {
    return (bx - ax) * (y - ay) - (by - ay) * (x - ax);
}

struct Raster {
    uint32_t width = 0, height = 0;
    std::vector<uint64_t> words;
    bool clipped = false;
    bool covered(size_t i) const { return (words[i / 64] >> (i % 64)) & 1; }
};

bo_camera camera_of(V3 right, V3 up, V3 forward, double distance, double focal, double scale,
                    bool perspective) {
    bo_camera c{};
    c.right[0] = right.x, c.right[1] = right.y, c.right[2] = right.z;
    c.up[0] = up.x, c.up[1] = up.y, c.up[2] = up.z;
    c.forward[0] = forward.x, c.forward[1] = forward.y, c.forward[2] = forward.z;
    c.distance = distance, c.focal = focal, c.scale = scale, c.perspective = perspective;
    return c;
}

// evaluate.cpp:108-124 — Fibonacci-sphere directions, orthographic first.
std::vector<bo_camera> make_cameras(const bo_bounds& b, double screen, uint16_t ortho,
                                    uint16_t persp, uint32_t seed) {
    std::vector<bo_camera> out;
    for (int projection = 0; projection < 2; ++projection) {
        unsigned count = projection ? persp : ortho;
        for (unsigned i = 0; i < count; ++i) {
            double z = 1 - 2 * (i + .5) / count, r = std::sqrt(std::max(0.0, 1 - z * z)),
                   angle = i * kPi * (3 - std::sqrt(5.0));
            V3 forward = normalized(rotate({float(r * std::cos(angle)), float(z), float(r * std::sin(angle))},
                                           seed + projection * 104729u));
            V3 hint = std::abs(forward.y) > .99 ? V3{1, 0, 0} : V3{0, 1, 0};
            V3 right = normalized(cross(hint, forward)), up = normalized(cross(forward, right));
            double height = std::max(1024.0, 2 * screen), focal = height / (2 * std::tan(kPi / 6));
            double distance = b.radius * std::sqrt(1 + std::pow(2 * focal / screen, 2));
            out.push_back(camera_of(right, up, forward, distance, focal, screen / (b.radius * 2),
                                    bool(projection)));
        }
    }
    return out;
}

uint32_t raster_size(double screen, uint8_t ss) { return uint32_t(std::ceil(screen + 8)) * ss; }

// evaluate.cpp:125-189, packed CoverageRaster variant.
Raster rasterize(const Mesh& m, const bo_bounds& b, const bo_camera& c, double screen, uint8_t ss,
                 bool force_two) {
    if (!ss || !std::isfinite(screen) || screen <= 0 || screen > 16384)
        throw std::invalid_argument("invalid raster extent");
    uint32_t size = raster_size(screen, ss);
    if (uint64_t(size) * size > kMaxSamples)
        throw std::length_error("raster exceeds per-view memory budget");
    Raster out;
    out.width = out.height = size;
    out.words.assign((size_t(size) * size + 63) / 64, 0);
    struct P {
        double x, y, z;
    };
    std::vector<P> projected(m.m->vertex_count);
    for (uint32_t i = 0; i < m.m->vertex_count; ++i) {
        V3 a = m.pos(i);
        double x = double(a.x) - b.center[0], y = double(a.y) - b.center[1],
               z0 = double(a.z) - b.center[2];
        auto dp = [&](const float* axis) { return x * axis[0] + y * axis[1] + z0 * axis[2]; };
        double z = c.distance - dp(c.forward), sc = c.perspective ? c.focal / z : c.scale;
        auto& p = projected[i];
        p.x = dp(c.right) * sc * ss + size * .5;
        p.y = dp(c.up) * sc * ss + size * .5;
        p.z = z;
    }
    for (uint32_t f = 0; f < m.faces(); ++f) {
        uint32_t ia = m.m->indices[3 * f], ib = m.m->indices[3 * f + 1], ic = m.m->indices[3 * f + 2];
        P a = projected[ia], d = projected[ib], e = projected[ic];
        if (c.perspective && (a.z <= 0 || d.z <= 0 || e.z <= 0)) {
            out.clipped = true;
            continue;
        }
        double area = edge_fn(a.x, a.y, d.x, d.y, e.x, e.y);
        if (std::abs(area) < 1e-16) continue;
        bool back = area < 0, two = force_two || m.two_sided(f);
        if (back && !two) continue;
        if (back) std::swap(d, e);
        double minx = std::min({a.x, d.x, e.x}), maxx = std::max({a.x, d.x, e.x});
        double miny = std::min({a.y, d.y, e.y}), maxy = std::max({a.y, d.y, e.y});
        if (!std::isfinite(minx) || !std::isfinite(maxx) || !std::isfinite(miny) ||
            !std::isfinite(maxy) || minx < 0 || miny < 0 || maxx > size || maxy > size) {
            out.clipped = true;
            return out;
        }
        int x0 = std::max(0, int(std::floor(minx))), x1 = std::min(int(size) - 1, int(std::floor(maxx)));
        int y0 = std::max(0, int(std::floor(miny))), y1 = std::min(int(size) - 1, int(std::floor(maxy)));
        double r0 = .5 * (std::abs(e.x - d.x) + std::abs(e.y - d.y));
        double r1 = .5 * (std::abs(a.x - e.x) + std::abs(a.y - e.y));
        double r2 = .5 * (std::abs(d.x - a.x) + std::abs(d.y - a.y));
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                double u = edge_fn(d.x, d.y, e.x, e.y, x + .5, y + .5),
                       v = edge_fn(e.x, e.y, a.x, a.y, x + .5, y + .5),
                       w = edge_fn(a.x, a.y, d.x, d.y, x + .5, y + .5);
                if (u + r0 < 0 || v + r1 < 0 || w + r2 < 0) continue;
                size_t index = size_t(y) * size + x;
                out.words[index / 64] |= uint64_t(1) << (index % 64);
            }
    }
    return out;
}

// Felzenszwalb–Huttenlocher lower envelope of sampled parabolas, with the
// reference's double intersections and float outputs (evaluate.cpp:33-53).
void envelope_1d(const float* f, float* out, int n, std::vector<int>& v, std::vector<double>& z) {
    int k = 0;
    v[0] = 0;
    z[0] = -kInf;
    z[1] = kInf;
    for (int q = 1; q < n; ++q) {
        double s;
        for (;;) {
            int p = v[k];
            s = ((double(f[q]) + double(q) * q) - (double(f[p]) + double(p) * p)) / (2 * (q - p));
            if (s > z[k] || k == 0) break;
            --k;
        }
        ++k;
        v[k] = q;
        z[k] = s;
        z[k + 1] = kInf;
    }
    k = 0;
    for (int x = 0; x < n; ++x) {
        while (z[k + 1] < x) ++k;
        double d = x - v[k];
        out[x] = float(d * d + f[v[k]]);
    }
}

// evaluate.cpp:58-70 — separable squared EDT to the nearest covered sample.
std::vector<float> distance_field(const Raster& r) {
    size_t n = size_t(r.width) * r.height;
    std::vector<float> a(n), b(n);
    for (size_t i = 0; i < n; ++i) a[i] = r.covered(i) ? 0.f : 1e15f;
    size_t len = std::max(r.width, r.height);
    std::vector<int> v(len);
    std::vector<double> z(len + 1);
    std::vector<float> f(len), d(len);
    for (uint32_t y = 0; y < r.height; ++y)
        envelope_1d(a.data() + size_t(y) * r.width, b.data() + size_t(y) * r.width, int(r.width), v, z);
    for (uint32_t x = 0; x < r.width; ++x) {
        for (uint32_t y = 0; y < r.height; ++y) f[y] = b[size_t(y) * r.width + x];
        envelope_1d(f.data(), d.data(), int(r.height), v, z);
        for (uint32_t y = 0; y < r.height; ++y) a[size_t(y) * r.width + x] = d[y];
    }
    return a;
}

// evaluate.cpp:196-209 plus the popcounts of evaluate.cpp:276-279.
bo_view_record record_of(const Raster& a, const Raster& c) {
    if (a.width != c.width || a.height != c.height) throw std::invalid_argument("raster shapes differ");
    bo_view_record r{};
    bool ca = false, cb = false, same = true;
    for (size_t i = 0; i < a.words.size(); ++i) {
        ca |= a.words[i] != 0;
        cb |= c.words[i] != 0;
        same &= a.words[i] == c.words[i];
        r.changed += __builtin_popcountll(a.words[i] ^ c.words[i]);
        r.total += __builtin_popcountll(a.words[i] | c.words[i]);
    }
    r.ca = ca, r.cb = cb, r.same = same;
    r.clipped_ref = a.clipped, r.clipped_cand = c.clipped;
    r.max_d2 = 0;
    if (!same && ca == cb) {
        double maximum = 0;
        auto directed = [&](const Raster& from, const Raster& to) {
            auto values = distance_field(to);
            for (size_t i = 0; i < values.size(); ++i)
                if (from.covered(i)) maximum = std::max(maximum, double(values[i]));
        };
        directed(a, c);
        directed(c, a);
        r.max_d2 = maximum;
    }
    return r;
}

double coverage_of(const bo_view_record& r, uint8_t ss) {
    if (r.same) return 0;
    if (r.ca != r.cb) return kInf;
    return std::sqrt(r.max_d2) / ss;
}

// evaluate.cpp:271-298, coverage profile.
void finish_view(bo_measurement& cur, const bo_view_record& r, const bo_eval_settings& s, uint8_t ss) {
    cur.supersample = ss;
    cur.coverage = coverage_of(r, ss);
    cur.coverage_upper = cur.coverage + 2 * std::sqrt(2.0) / ss + 1e-6;
    if (r.clipped_cand || r.clipped_ref) cur.coverage_upper = kInf;
    cur.error = cur.coverage_upper;
    cur.changed_area = r.total ? double(r.changed) / double(r.total) : 0;
    cur.passed = cur.error <= s.limit && cur.changed_area <= s.max_changed_area;
    if (s.conservative_screen) {
        cur.error = (r.clipped_ref || r.clipped_cand)
                        ? 0
                        : std::max(0.0, cur.coverage - 2 * std::sqrt(2.0) / ss - 1e-6);
        cur.passed = cur.error <= s.limit;
    }
}

bo_measurement default_measurement() {
    bo_measurement m{};
    m.complete = 1;
    m.passed = 1;
    return m;
}

// evaluation_settings.hpp:10-23 (coverage-profile fields only).
void validate_settings(const bo_bounds& b, const bo_eval_settings& s) {
    bool center_ok = std::isfinite(b.center[0]) && std::isfinite(b.center[1]) && std::isfinite(b.center[2]);
    if (!(s.screen_size > 0) || !std::isfinite(s.screen_size) || s.screen_size > 16384 ||
        !(b.radius > 0) || !std::isfinite(b.radius) || !center_ok || s.profile > 2 ||
        !(s.limit >= 0) || !std::isfinite(s.limit) || !s.supersample ||
        s.max_supersample < s.supersample || s.max_supersample > 32 ||
        !std::isfinite(s.max_changed_area) || s.max_changed_area < 0 || s.max_changed_area > 1)
        throw std::invalid_argument("invalid evaluation settings");
    if (!s.views_orthographic && !s.views_perspective)
        throw std::invalid_argument("at least one camera required");
}

template <class T> bool same_array(const T* a, const T* b, size_t n) {
    if (!n || a == b) return true;
    if (!a || !b) return false;
    return std::memcmp(a, b, n * sizeof(T)) == 0;
}
// evaluate.cpp:71-82 — positions, indices, materials and double-sided flags.
bool identical(const bo_mesh& a, const bo_mesh& b) {
    if (a.vertex_count != b.vertex_count || a.face_count != b.face_count) return false;
    if (!same_array(a.positions, b.positions, size_t(a.vertex_count) * 3)) return false;
    if (!same_array(a.indices, b.indices, size_t(a.face_count) * 3)) return false;
    if (bool(a.materials) != bool(b.materials) ||
        !same_array(a.materials, b.materials, a.materials ? a.face_count : 0))
        return false;
    uint32_t na = a.double_sided ? a.double_sided_count : 0, nb = b.double_sided ? b.double_sided_count : 0;
    return na == nb && same_array(a.double_sided, b.double_sided, na);
}

// evaluate.cpp:312-352 (no coverage cache, coverage profile).
bo_measurement evaluate(const bo_mesh& reference, const bo_mesh& candidate, const bo_bounds& b,
                        const bo_eval_settings& s) {
    bo_measurement result = default_measurement();
    result.supersample = s.supersample;
    validate_settings(b, s);
    auto views = make_cameras(b, s.screen_size, s.views_orthographic, s.views_perspective, s.views_seed);
    if (identical(reference, candidate)) return result;
    Mesh ref{&reference}, cand{&candidate};
    for (uint32_t v = 0; v < views.size(); ++v) {
        bo_measurement current = default_measurement();
        current.worst_view = v;
        for (unsigned ss = s.supersample;; ss = std::min<unsigned>(s.max_supersample, ss * 2)) {
            try {
                Raster a = rasterize(ref, b, views[v], s.screen_size, uint8_t(ss), s.force_two_sided);
                Raster c = rasterize(cand, b, views[v], s.screen_size, uint8_t(ss), s.force_two_sided);
                finish_view(current, record_of(a, c), s, uint8_t(ss));
            } catch (const std::length_error&) {
                result.complete = 0;
                result.passed = 0;
                result.resource_limited = 1;
                result.error = kInf;
                return result;
            }
            if (s.conservative_screen || current.passed || ss >= s.max_supersample ||
                current.coverage - 2 * std::sqrt(2.0) / ss > s.limit || !std::isfinite(current.error) ||
                current.coverage_upper <= s.limit)
                break;
        }
        ++result.views_evaluated;
        if (current.error > result.error) {
            result.worst_view = v;
            result.error = current.error;
            result.supersample = current.supersample;
        }
        result.coverage = std::max(result.coverage, current.coverage);
        result.coverage_upper = std::max(result.coverage_upper, current.coverage_upper);
        if (current.changed_area > result.changed_area) {
            result.changed_area = current.changed_area;
            result.changed_area_worst_view = v;
        }
        result.normal_degrees = std::max(result.normal_degrees, current.normal_degrees);
        if (!current.passed) {
            result.passed = 0;
            result.complete = 0;
            return result;
        }
    }
    return result;
}

// audit_measurement.hpp:8-17
bool measurement_passed(const bo_measurement& m) {
    bool nonfinite = std::isnan(m.error) || std::isnan(m.coverage) || std::isnan(m.coverage_upper) ||
                     !std::isfinite(m.changed_area) || !std::isfinite(m.normal_degrees) ||
                     (m.passed && (!std::isfinite(m.error) || !std::isfinite(m.coverage) ||
                                   !std::isfinite(m.coverage_upper)));
    return m.complete && m.passed && !m.cancelled && !m.resource_limited && !nonfinite;
}

// ---------------------------------------------------------------------------
// Collapse topology (action.cpp:27-145; action_gpu.cu:178-344).
uint32_t position_bits(float f) {
    float g = f == 0 ? 0.f : f;
    uint32_t u;
    std::memcpy(&u, &g, 4);
    return u;
}
std::array<uint32_t, 3> position_key(V3 p) { return {position_bits(p.x), position_bits(p.y), position_bits(p.z)}; }

struct Topology {
    uint32_t n = 0;
    std::vector<uint32_t> geometry, canonical;
    std::vector<uint32_t> offsets, neighbors, face_offsets, faces;
    std::vector<std::pair<uint64_t, uint32_t>> edges; // (a<<32|b, count) sorted
    std::vector<uint8_t> boundary, invalid;
};

// action.cpp:8-12, 33-46 — each slot maps to the smallest slot index at the same
// position (zero signs folded). With attributes, uv must also match (the
// canonical welding of action_gpu.cu:178-211 for a mesh with only uv).
std::vector<uint32_t> weld(const bo_mesh& m, bool with_uv) {
    std::vector<uint32_t> order(m.vertex_count);
    std::iota(order.begin(), order.end(), 0);
    auto key = [&](uint32_t i) {
        auto k = position_key(load3(m.positions, i));
        std::array<uint32_t, 5> out{k[0], k[1], k[2], 0, 0};
        if (with_uv && m.uv) {
            std::memcpy(&out[3], &m.uv[2 * i], 4);
            std::memcpy(&out[4], &m.uv[2 * i + 1], 4);
        }
        return out;
    };
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        auto ka = key(a), kb = key(b);
        return ka != kb ? ka < kb : a < b;
    });
    std::vector<uint32_t> root(m.vertex_count);
    uint32_t r = order.empty() ? 0 : order[0];
    for (auto i : order) {
        if (key(i) != key(r)) r = i;
        root[i] = r;
    }
    return root;
}

// action.cpp:49-145 on the given class ids. The executor keeps the classes of
// the episode's initial mesh across commits (action_gpu.cu:1520-1527 welds once
// at construction); pass them in `classes`.
Topology build_topology(const bo_mesh& m, bool preserve_uv, const Topology* classes = nullptr) {
    Topology t;
    t.n = m.vertex_count;
    t.geometry = classes ? classes->geometry : weld(m, false);
    t.canonical = classes ? classes->canonical : weld(m, preserve_uv);
    const uint32_t n = t.n;
    t.offsets.assign(n + 1, 0);
    t.face_offsets.assign(n + 1, 0);
    t.boundary.assign(n, 0);
    t.invalid.assign(n, 0);
    std::vector<uint64_t> pairs;
    for (uint32_t f = 0; f < m.face_count; ++f) {
        uint32_t v[3];
        for (int j = 0; j < 3; ++j) v[j] = t.geometry[m.indices[3 * f + j]];
        for (int j = 0; j < 3; ++j) {
            uint32_t a = v[j], b = v[(j + 1) % 3];
            ++t.face_offsets[a + 1];
            if (a == b) {
                for (auto i : v) t.invalid[i] = 1;
                continue;
            }
            if (a > b) std::swap(a, b);
            pairs.push_back(uint64_t(a) << 32 | b);
        }
    }
    std::sort(pairs.begin(), pairs.end());
    for (size_t i = 0; i < pairs.size();) {
        size_t end = i + 1;
        while (end < pairs.size() && pairs[end] == pairs[i]) ++end;
        uint32_t a = uint32_t(pairs[i] >> 32), b = uint32_t(pairs[i]);
        size_t count = end - i;
        if (count == 1) t.boundary[a] = t.boundary[b] = 1;
        if (count > 2) t.invalid[a] = t.invalid[b] = 1;
        t.edges.push_back({pairs[i], uint32_t(std::min<size_t>(3, count))});
        ++t.offsets[a + 1];
        ++t.offsets[b + 1];
        i = end;
    }
    std::partial_sum(t.offsets.begin(), t.offsets.end(), t.offsets.begin());
    std::partial_sum(t.face_offsets.begin(), t.face_offsets.end(), t.face_offsets.begin());
    t.neighbors.resize(t.edges.size() * 2);
    t.faces.resize(size_t(m.face_count) * 3);
    auto next = t.offsets, face_next = t.face_offsets;
    for (auto& e : t.edges) {
        uint32_t a = uint32_t(e.first >> 32), b = uint32_t(e.first);
        t.neighbors[next[a]++] = b;
        t.neighbors[next[b]++] = a;
    }
    for (uint32_t f = 0; f < m.face_count; ++f)
        for (int j = 0; j < 3; ++j) t.faces[face_next[t.geometry[m.indices[3 * f + j]]]++] = f;
    for (uint32_t i = 0; i < n; ++i)
        std::sort(t.neighbors.begin() + t.offsets[i], t.neighbors.begin() + t.offsets[i + 1]);
    // Single-fan check (action.cpp:109-144).
    std::vector<std::pair<uint32_t, uint32_t>> links;
    std::vector<uint32_t> reached;
    for (uint32_t u = 0; u < n; ++u) {
        if (t.face_offsets[u] == t.face_offsets[u + 1] || t.invalid[u]) continue;
        links.clear();
        for (auto k = t.face_offsets[u]; k < t.face_offsets[u + 1]; ++k) {
            uint32_t f = t.faces[k], other[2];
            unsigned count = 0;
            for (int j = 0; j < 3; ++j) {
                uint32_t v = t.geometry[m.indices[3 * f + j]];
                if (v != u && count < 2) other[count++] = v;
            }
            if (count != 2) {
                t.invalid[u] = 1;
                break;
            }
            links.emplace_back(other[0], other[1]);
        }
        if (t.invalid[u]) continue;
        reached.assign(1, links[0].first);
        for (size_t i = 0; i < reached.size(); ++i)
            for (auto [a, b] : links) {
                uint32_t v = a == reached[i] ? b : b == reached[i] ? a : kNone;
                if (v != kNone && std::find(reached.begin(), reached.end(), v) == reached.end())
                    reached.push_back(v);
            }
        if (reached.size() != t.offsets[u + 1] - t.offsets[u]) t.invalid[u] = 1;
    }
    return t;
}

// Without preserve_uv the reference's GPU state welds every corner to its
// attribute class ignoring uv (action_gpu.cu:1518-1532: insert/lookup_vertices
// with attributes, then weld_uv_indices), so uv seams stop being wedges. This
// mesh record has no normals or colours, so the class is the bitwise position
// class. `welded.m` views `*m` with the welded indices.
struct UvWelded {
    std::vector<uint32_t> indices;
    bo_mesh m;
};
UvWelded weld_uv_indices(const bo_mesh& m) {
    UvWelded w;
    const std::vector<uint32_t> root = weld(m, false);
    w.indices.resize(size_t(m.face_count) * 3);
    for (size_t i = 0; i < w.indices.size(); ++i) w.indices[i] = root[m.indices[i]];
    w.m = m;
    w.m.indices = w.indices.data();
    return w;
}
// The mesh the GPU state works on for `preserve_uv`: `m` itself, or its
// uv-welded copy held in `hold`.
const bo_mesh& state_mesh(const bo_mesh& m, bool preserve_uv, UvWelded& hold) {
    if (preserve_uv) return m;
    hold = weld_uv_indices(m);
    return hold.m;
}

bool has_neighbor(const Topology& t, uint32_t u, uint32_t v) {
    return std::binary_search(t.neighbors.begin() + t.offsets[u], t.neighbors.begin() + t.offsets[u + 1], v);
}
uint32_t map_vertex(const bo_edit& e, uint32_t id) {
    for (unsigned j = 0; j < e.wedges; ++j)
        if (id == e.source[j]) return e.target[j];
    return id;
}
void sort3(uint32_t* x) { std::sort(x, x + 3); }
double area2(const float* uv, uint32_t a, uint32_t b, uint32_t c) {
    return (double(uv[2 * b]) - uv[2 * a]) * (double(uv[2 * c + 1]) - uv[2 * a + 1]) -
           (double(uv[2 * b + 1]) - uv[2 * a + 1]) * (double(uv[2 * c]) - uv[2 * a]);
}

// action_gpu.cu:487-627 — directed legality; with placement the orientation and
// UV checks are deferred to validation of the placed trial.
bool legal(const bo_mesh& m, const Topology& t, bo_edit& edit, bool placement, bool preserve_uv) {
    Mesh mesh{&m};
    uint32_t u = edit.from, v = edit.to;
    if (t.invalid[u] || t.invalid[v]) return false;
    uint32_t opposite[2] = {kNone, kNone}, edge_faces = 0;
    for (auto k = t.face_offsets[u]; k < t.face_offsets[u + 1]; ++k) {
        uint32_t f = t.faces[k], a = kNone, b = kNone, w = kNone;
        for (int j = 0; j < 3; ++j) {
            uint32_t id = m.indices[3 * f + j], g = t.geometry[id];
            if (g == u) a = id;
            else if (g == v) b = id;
            else w = g;
        }
        if (a == kNone) return false;
        if (b != kNone) {
            if (edge_faces == 2 || w == kNone) return false;
            opposite[edge_faces++] = w;
            bool found = false;
            for (unsigned j = 0; j < edit.wedges; ++j) found |= edit.source[j] == a && edit.target[j] == b;
            if (!found) {
                if (edit.wedges == 2) return false;
                edit.source[edit.wedges] = a;
                edit.target[edit.wedges++] = b;
            }
        }
    }
    if (!edge_faces || edge_faces >= m.face_count || (edge_faces == 2 && opposite[0] == opposite[1]))
        return false;
    if (t.boundary[u] && (!t.boundary[v] || edge_faces != 1)) return false;
    uint32_t common = 0;
    for (auto k = t.offsets[u]; k < t.offsets[u + 1]; ++k) {
        uint32_t w = t.neighbors[k];
        if (has_neighbor(t, v, w)) {
            if (w != opposite[0] && (edge_faces < 2 || w != opposite[1])) return false;
            ++common;
        }
    }
    if (common != edge_faces) return false;
    if (edit.wedges == 2) {
        if (edit.source[0] == edit.source[1]) return false;
        if (edit.source[0] > edit.source[1]) {
            std::swap(edit.source[0], edit.source[1]);
            std::swap(edit.target[0], edit.target[1]);
        }
    }
    uint16_t first = mesh.material(t.faces[t.face_offsets[u]]);
    bool junction = false;
    for (auto k = t.face_offsets[u]; k < t.face_offsets[u + 1]; ++k) {
        uint32_t f = t.faces[k];
        junction |= mesh.material(f) != first;
        for (int j = 0; j < 3; ++j) {
            uint32_t id = m.indices[3 * f + j];
            if (t.geometry[id] == u) {
                bool mapped = false;
                for (unsigned l = 0; l < edit.wedges; ++l) mapped |= edit.source[l] == id;
                if (!mapped) return false;
            }
        }
    }
    if (junction)
        for (int direction = 0; direction < 2; ++direction) {
            uint32_t a = direction ? v : u, b = direction ? u : v;
            for (auto k = t.face_offsets[a]; k < t.face_offsets[a + 1]; ++k) {
                uint16_t mat = mesh.material(t.faces[k]);
                bool found = false;
                for (auto l = t.face_offsets[b]; l < t.face_offsets[b + 1]; ++l)
                    found |= mat == mesh.material(t.faces[l]);
                if (!found) return false;
            }
        }
    for (auto k = t.face_offsets[u]; k < t.face_offsets[u + 1]; ++k) {
        uint32_t f = t.faces[k], old[3], next[3], sorted[3];
        bool removed = false;
        for (int j = 0; j < 3; ++j) {
            old[j] = m.indices[3 * f + j];
            next[j] = map_vertex(edit, old[j]);
            sorted[j] = t.geometry[next[j]];
            removed |= t.geometry[old[j]] == v;
        }
        if (removed) continue;
        sort3(sorted);
        if (sorted[0] == sorted[1] || sorted[1] == sorted[2]) return false;
        for (int direction = 0; direction < 2; ++direction) {
            uint32_t a = direction ? u : v;
            uint32_t end = direction ? k : t.face_offsets[a + 1];
            for (auto l = t.face_offsets[a]; l < end; ++l) {
                uint32_t g = t.faces[l], other[3];
                bool skip = false;
                for (int j = 0; j < 3; ++j) {
                    uint32_t id = m.indices[3 * g + j];
                    skip |= direction && t.geometry[id] == v;
                    other[j] = t.geometry[direction ? map_vertex(edit, id) : id];
                }
                sort3(other);
                if (!skip && sorted[0] == other[0] && sorted[1] == other[1] && sorted[2] == other[2])
                    return false;
            }
        }
        if (placement) continue;
        V3 before = cross(sub(mesh.pos(old[1]), mesh.pos(old[0])), sub(mesh.pos(old[2]), mesh.pos(old[0])));
        V3 after = cross(sub(mesh.pos(next[1]), mesh.pos(next[0])), sub(mesh.pos(next[2]), mesh.pos(next[0])));
        if (length(after) <= 1e-15 || dot(before, after) <= .05 * length(before) * length(after)) return false;
        if (preserve_uv && m.uv) {
            double x = area2(m.uv, old[0], old[1], old[2]), y = area2(m.uv, next[0], next[1], next[2]);
            if (std::fabs(x) > 1e-20 && x * y <= 0) return false;
        }
    }
    edit.removed = uint8_t(edge_faces);
    return true;
}

// action_gpu.cu:626-643 — every directed edge in sorted (a<b) edge order, a->b first.
std::vector<bo_edit> enumerate(const bo_mesh& m, const Topology& t, bool placement, bool preserve_uv) {
    std::vector<bo_edit> out;
    for (auto& e : t.edges)
        for (int dir = 0; dir < 2; ++dir) {
            uint32_t a = uint32_t(e.first >> 32), b = uint32_t(e.first);
            bo_edit edit{};
            edit.from = dir ? b : a;
            edit.to = dir ? a : b;
            if (legal(m, t, edit, placement, preserve_uv)) {
                edit.valid = 1;
                out.push_back(edit);
            }
        }
    return out;
}

// action_gpu.cu:919-952 — closest point on a triangle as barycentric weights.
V3 barycentric(V3 p, V3 a, V3 b, V3 c) {
    V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return {1, 0, 0};
    V3 bp = sub(p, b);
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return {0, 1, 0};
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        double v = d1 / (d1 - d3);
        return {float(1 - v), float(v), 0};
    }
    V3 cp = sub(p, c);
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return {0, 0, 1};
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        double w = d2 / (d2 - d6);
        return {float(1 - w), 0, float(w)};
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return {0, float(1 - w), float(w)};
    }
    double sum = va + vb + vc;
    if (std::fabs(sum) < 1e-30) return {1, 0, 0};
    double v = vb / sum, w = vc / sum;
    return {float(1 - v - w), float(v), float(w)};
}
// action_gpu.cu:953-955
V3 blend3(V3 a, V3 b, V3 c, V3 w) { return add(add(scale3(a, w.x), scale3(b, w.y)), scale3(c, w.z)); }

// action_gpu.cu:22-24, 1172 — midpoint of the two class roots, float sum then halved.
V3 midpoint(const bo_mesh& m, const bo_edit& e) {
    return scale3(add(load3(m.positions, e.from), load3(m.positions, e.to)), .5);
}

struct Trial {
    std::vector<uint32_t> indices;
    std::vector<uint16_t> materials;
    std::vector<float> positions, uv;
    bool valid = true;
};

uint32_t hash_position(V3 p) {
    uint32_t h = position_bits(p.x) * 0x9e3779b9u;
    h = (h ^ position_bits(p.y)) * 0x85ebca6bu;
    return (h ^ position_bits(p.z)) * 0xc2b2ae35u;
}

// Trial build (action_gpu.cu:748-790), midpoint placement written to every slot of
// class `to` with uv transported from the closest original incident face
// (action_gpu.cu:962-1067), then validate_placement (action_gpu.cu:1103-1156).
// `original` is the episode's initial mesh (attribute charts); `ot` its topology.
// A batch applies several collapses with disjoint footprints at once
// (ActionState::trial(span), action.cpp:308-345): one remap over all wedges,
// each edit's placement on the slots of its own `to` class.
Trial make_trial(const bo_mesh& m, const Topology& t, const bo_mesh& original, const Topology& ot,
                 const std::vector<bo_edit>& batch, bool preserve_uv) {
    Trial out;
    const uint32_t n = m.vertex_count;
    std::vector<uint32_t> remap(n, kNone), owner(n, kNone);
    for (uint32_t k = 0; k < batch.size(); ++k) {
        const bo_edit& e = batch[k];
        for (unsigned j = 0; j < e.wedges; ++j) remap[e.source[j]] = e.target[j];
        owner[e.to] = k;
    }
    std::vector<uint8_t> keep(m.face_count);
    for (uint32_t f = 0; f < m.face_count; ++f) {
        uint32_t ids[3];
        bool changed = false;
        for (int j = 0; j < 3; ++j) {
            uint32_t i = m.indices[3 * f + j];
            if (remap[i] != kNone) {
                i = remap[i];
                changed = true;
            }
            ids[j] = t.geometry[i];
        }
        keep[f] = !(changed && (ids[0] == ids[1] || ids[1] == ids[2] || ids[0] == ids[2]));
        if (!keep[f]) continue;
        for (int j = 0; j < 3; ++j) {
            uint32_t i = m.indices[3 * f + j];
            out.indices.push_back(remap[i] == kNone ? i : remap[i]);
        }
        if (m.materials) out.materials.push_back(m.materials[f]);
    }
    // place_vertices
    std::vector<V3> placements(batch.size());
    for (uint32_t k = 0; k < batch.size(); ++k) placements[k] = midpoint(m, batch[k]);
    out.positions.assign(m.positions, m.positions + size_t(n) * 3);
    if (m.uv) out.uv.assign(m.uv, m.uv + size_t(n) * 2);
    for (uint32_t v = 0; v < n; ++v) {
        if (owner[t.geometry[v]] != kNone) {
            const bo_edit& e = batch[owner[t.geometry[v]]];
            const V3 p = placements[owner[t.geometry[v]]];
            out.positions[3 * v] = p.x, out.positions[3 * v + 1] = p.y, out.positions[3 * v + 2] = p.z;
            if (m.uv) {
                uint32_t roots[2] = {t.canonical[v], kNone};
                for (unsigned w = 0; w < e.wedges; ++w)
                    if (t.canonical[v] == t.canonical[e.target[w]]) roots[1] = t.canonical[e.source[w]];
                V3 ov = load3(original.positions, v);
                double best = dot(sub(p, ov), sub(p, ov));
                uint32_t ids[3] = {v, v, v};
                V3 weights{1, 0, 0};
                // Faces of the root's canonical class in the original mesh, ascending.
                for (int side = 0; side < 2; ++side) {
                    uint32_t root = roots[side];
                    if (root == kNone) continue;
                    for (uint32_t f = 0; f < original.face_count; ++f) {
                        bool incident = false;
                        for (int j = 0; j < 3; ++j) incident |= ot.canonical[original.indices[3 * f + j]] == root;
                        if (!incident) continue;
                        // A face with two corners in the class is listed twice; the
                        // strict comparison makes the repeat a no-op.
                        uint32_t a = original.indices[3 * f], b = original.indices[3 * f + 1],
                                 c = original.indices[3 * f + 2];
                        V3 A = load3(original.positions, a), B = load3(original.positions, b),
                           C = load3(original.positions, c);
                        V3 w = barycentric(p, A, B, C);
                        V3 delta = sub(p, blend3(A, B, C, w));
                        double distance = dot(delta, delta);
                        if (distance < best) {
                            best = distance;
                            ids[0] = a, ids[1] = b, ids[2] = c;
                            weights = w;
                        }
                    }
                }
                const float* ouv = original.uv;
                out.uv[2 * v] = float(double(ouv[2 * ids[0]]) * weights.x + double(ouv[2 * ids[1]]) * weights.y +
                                      double(ouv[2 * ids[2]]) * weights.z);
                out.uv[2 * v + 1] = float(double(ouv[2 * ids[0] + 1]) * weights.x +
                                          double(ouv[2 * ids[1] + 1]) * weights.y +
                                          double(ouv[2 * ids[2] + 1]) * weights.z);
            }
        }
        V3 q = load3(out.positions.data(), v);
        if (!finite3(q)) out.valid = false;
        if (m.uv && (!std::isfinite(out.uv[2 * v]) || !std::isfinite(out.uv[2 * v + 1]))) out.valid = false;
    }
    // validate_placement over kept faces of the current mesh.
    std::unordered_map<uint64_t, std::vector<uint32_t>> seen;
    auto key64 = [](V3 q) {
        return (uint64_t(position_bits(q.x)) << 32) ^ (uint64_t(position_bits(q.y)) * 0x9e3779b97f4a7c15ull) ^
               position_bits(q.z);
    };
    for (uint32_t f = 0; f < m.face_count && out.valid; ++f) {
        if (!keep[f]) continue;
        uint32_t old[3], next[3];
        for (int j = 0; j < 3; ++j) {
            old[j] = m.indices[3 * f + j];
            next[j] = remap[old[j]] == kNone ? old[j] : remap[old[j]];
        }
        const float* P = out.positions.data();
        V3 before = cross(sub(load3(m.positions, old[1]), load3(m.positions, old[0])),
                          sub(load3(m.positions, old[2]), load3(m.positions, old[0])));
        V3 after = cross(sub(load3(P, next[1]), load3(P, next[0])), sub(load3(P, next[2]), load3(P, next[0])));
        if (length(after) <= 1e-15 || dot(before, after) <= .05 * length(before) * length(after)) {
            out.valid = false;
            break;
        }
        if (preserve_uv && m.uv) {
            double x = area2(m.uv, old[0], old[1], old[2]), y = area2(out.uv.data(), next[0], next[1], next[2]);
            if (!std::isfinite(y) || (std::fabs(x) > 1e-20 && x * y <= 0)) {
                out.valid = false;
                break;
            }
        }
        for (uint32_t v : next) {
            V3 q = load3(P, v);
            auto& bucket = seen[key64(q)];
            bool placed = false;
            for (uint32_t o : bucket)
                if (position_key(load3(P, o)) == position_key(q)) {
                    if (t.geometry[v] != t.geometry[o]) out.valid = false;
                    placed = true;
                    break;
                }
            if (!placed) bucket.push_back(v);
        }
    }
    return out;
}
Trial make_trial(const bo_mesh& m, const Topology& t, const bo_mesh& original, const Topology& ot,
                 const bo_edit& e, bool preserve_uv) {
    return make_trial(m, t, original, ot, std::vector<bo_edit>{e}, preserve_uv);
}

// Greedy disjoint-footprint batch from ranked position `start` (select_batch,
// action_gpu.cu:865-899; ActionState::independent, action.cpp:261-304): skip
// edits removing more faces than remain, claim {from, to} and their class
// neighbours, stop at `maximum` edits or when nothing remains. Returns ranked
// positions.
std::vector<size_t> select_batch(const Topology& t, const std::vector<bo_edit>& edits,
                                 const std::vector<uint32_t>& order, size_t start, uint32_t maximum,
                                 uint32_t remaining) {
    std::vector<uint8_t> used(t.n);
    std::vector<size_t> out;
    for (size_t k = start; k < order.size() && remaining; ++k) {
        const bo_edit& e = edits[order[k]];
        if (e.removed > remaining) continue;
        bool overlaps = false;
        for (uint32_t u : {e.from, e.to}) {
            overlaps |= used[u] != 0;
            for (uint32_t j = t.offsets[u]; j < t.offsets[u + 1]; ++j) overlaps |= used[t.neighbors[j]] != 0;
        }
        if (overlaps) continue;
        for (uint32_t u : {e.from, e.to}) {
            used[u] = 1;
            for (uint32_t j = t.offsets[u]; j < t.offsets[u + 1]; ++j) used[t.neighbors[j]] = 1;
        }
        out.push_back(k);
        remaining -= e.removed;
        if (out.size() == maximum) break;
    }
    return out;
}

bo_mesh trial_view(const bo_mesh& m, const Trial& tr) {
    bo_mesh v = m;
    v.positions = tr.positions.data();
    v.indices = tr.indices.data();
    v.face_count = uint32_t(tr.indices.size() / 3);
    v.materials = m.materials ? tr.materials.data() : nullptr;
    v.uv = m.uv ? tr.uv.data() : nullptr;
    return v;
}

// Four gates on a built trial (generate.cpp:365-388).
bool audit_gates(const bo_mesh& cand, const bo_mesh& source, const bo_mesh& previous, const bo_bounds& b,
                 const bo_eval_settings gates[4], bo_verdict* out) {
    for (int g = 0; g < 4; ++g) {
        bo_eval_settings s = gates[g];
        uint64_t side = uint64_t(std::ceil(s.screen_size + 8));
        unsigned ss = s.supersample;
        while (ss < s.max_supersample) { // graph.cpp:5-18
            unsigned next = std::min<unsigned>(ss * 2, s.max_supersample);
            if (side * side * next * next > kMaxSamples) break;
            ss = next;
        }
        s.max_supersample = uint8_t(ss);
        const bo_mesh& ref = (g % 2) ? previous : source;
        bo_measurement m = evaluate(ref, cand, b, s);
        if (out) out->gates[g] = m;
        if (!measurement_passed(m)) {
            if (out) out->failed_gate = uint8_t(g + 1);
            return false;
        }
    }
    if (out) out->accepted = 1;
    return true;
}

// Working state of the greedy executor: owned streams of the current LOD.
struct ExecState {
    std::vector<float> pos, uv;
    std::vector<uint32_t> idx;
    std::vector<uint16_t> mat;
    std::vector<uint8_t> sided;
    bo_mesh view() const {
        bo_mesh m{};
        m.positions = pos.data();
        m.vertex_count = uint32_t(pos.size() / 3);
        m.indices = idx.data();
        m.face_count = uint32_t(idx.size() / 3);
        m.materials = mat.empty() ? nullptr : mat.data();
        m.double_sided = sided.empty() ? nullptr : sided.data();
        m.double_sided_count = uint32_t(sided.size());
        m.uv = uv.empty() ? nullptr : uv.data();
        return m;
    }
};

// ShortestEdge ranking of rank_actions (action_gpu.cu:822-825): minus the edge
// length over the origin diameter, with float rounding of the scaled delta.
float shortest_edge_score(const bo_mesh& m, const bo_edit& e, double diameter) {
    V3 d = scale3(sub(load3(m.positions, e.to), load3(m.positions, e.from)), 1 / diameter);
    return -float(length(d));
}

// CurrentPlane ranking of rank_actions (action_gpu.cu:826-840): minus the sum,
// over the faces of the `from` class, of the face's area weight times the
// squared distance of `to` to its plane, all over the diameter.
float current_plane_score(const bo_mesh& m, const Topology& t, const bo_edit& e, double diameter) {
    const double scale = std::max(1e-20, diameter);
    double cost = 0;
    for (uint32_t k = t.face_offsets[e.from]; k < t.face_offsets[e.from + 1]; ++k) {
        const uint32_t f = t.faces[k];
        V3 p = load3(m.positions, m.indices[3 * f]), q = load3(m.positions, m.indices[3 * f + 1]),
           r = load3(m.positions, m.indices[3 * f + 2]);
        V3 normal = cross(sub(q, p), sub(r, p));
        const double weight = length(normal);
        const V3 unit = weight > 0 ? scale3(normal, 1 / weight) : V3{0, 0, 0};
        const double distance = dot(unit, sub(load3(m.positions, e.to), p)) / scale;
        cost += distance * distance * weight / (scale * scale);
    }
    return float(-cost);
}
// Scores of the rankings the executor supports (neural.hpp:9): 1 Constant,
// 3 ShortestEdge, 4 CurrentPlane.
float rank_score(int ranking, const bo_mesh& m, const Topology& t, const bo_edit& e, double diameter) {
    if (ranking == 1) return 0.f;
    if (ranking == 4) return current_plane_score(m, t, e, diameter);
    return shortest_edge_score(m, e, diameter);
}

template <class F> int guarded(F f) {
    try {
        f();
        return 0;
    } catch (const std::length_error&) {
        return 2;
    } catch (const std::exception&) {
        return 1;
    }
}
} // namespace

extern "C" {

// mesh.cpp:12-20
int bo_barycentric(const float p[3], const float a[3], const float b[3], const float c[3], float w[3]) {
    if (!p || !a || !b || !c || !w) return 1;
    const V3 r = barycentric({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
    w[0] = r.x, w[1] = r.y, w[2] = r.z;
    return 0;
}

int bo_bounds_of(const bo_mesh* m, bo_bounds* out) {
    if (!m || !out || !m->vertex_count) return 1;
    V3 lo = load3(m->positions, 0), hi = lo;
    for (uint32_t i = 1; i < m->vertex_count; ++i) {
        V3 p = load3(m->positions, i);
        lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
        hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
    }
    out->center[0] = float((double(lo.x) + hi.x) * .5);
    out->center[1] = float((double(lo.y) + hi.y) * .5);
    out->center[2] = float((double(lo.z) + hi.z) * .5);
    out->radius = 0;
    for (uint32_t i = 0; i < m->vertex_count; ++i) {
        V3 p = load3(m->positions, i);
        double x = double(p.x) - out->center[0], y = double(p.y) - out->center[1],
               z = double(p.z) - out->center[2];
        out->radius = std::max(out->radius, std::sqrt(x * x + y * y + z * z));
    }
    return 0;
}

int bo_cameras(const bo_bounds* b, double screen, uint16_t ortho, uint16_t persp, uint32_t seed,
               bo_camera* out) {
    if (!b || !out) return 1;
    auto cams = make_cameras(*b, screen, ortho, persp, seed);
    std::copy(cams.begin(), cams.end(), out);
    return 0;
}

uint32_t bo_raster_size(double screen, uint8_t ss) { return raster_size(screen, ss); }

int bo_rasterize_coverage(const bo_mesh* m, const bo_bounds* b, const bo_camera* c, double screen,
                          uint8_t ss, int force_two, uint64_t* words, uint8_t* clipped) {
    return guarded([&] {
        Raster r = rasterize(Mesh{m}, *b, *c, screen, ss, force_two != 0);
        std::copy(r.words.begin(), r.words.end(), words);
        if (clipped) *clipped = r.clipped;
    });
}

int bo_coverage_distance(const uint64_t* a, const uint64_t* b, uint32_t width, uint32_t height,
                         uint8_t ss, double* out) {
    if (!ss) return 1;
    return guarded([&] {
        size_t words = (size_t(width) * height + 63) / 64;
        Raster ra, rb;
        ra.width = rb.width = width;
        ra.height = rb.height = height;
        ra.words.assign(a, a + words);
        rb.words.assign(b, b + words);
        *out = coverage_of(record_of(ra, rb), ss);
    });
}

int bo_distance_field(const uint64_t* words, uint32_t width, uint32_t height, float* out) {
    return guarded([&] {
        Raster r;
        r.width = width, r.height = height;
        r.words.assign(words, words + (size_t(width) * height + 63) / 64);
        auto f = distance_field(r);
        std::copy(f.begin(), f.end(), out);
    });
}

int bo_view_record_of(const bo_mesh* reference, const bo_mesh* candidate, const bo_bounds* b,
                      const bo_camera* c, double screen, uint8_t ss, int force_two,
                      bo_view_record* out) {
    return guarded([&] {
        Raster a = rasterize(Mesh{reference}, *b, *c, screen, ss, force_two != 0);
        Raster cc = rasterize(Mesh{candidate}, *b, *c, screen, ss, force_two != 0);
        *out = record_of(a, cc);
    });
}

void bo_finish_view(const bo_view_record* r, const bo_eval_settings* s, uint8_t ss, bo_measurement* out) {
    *out = default_measurement();
    finish_view(*out, *r, *s, ss);
}

int bo_evaluate(const bo_mesh* reference, const bo_mesh* candidate, const bo_bounds* b,
                const bo_eval_settings* s, bo_measurement* out) {
    return guarded([&] { *out = evaluate(*reference, *candidate, *b, *s); });
}

int bo_identical(const bo_mesh* a, const bo_mesh* b) { return identical(*a, *b); }

// graph.cpp:5-18
uint8_t bo_bounded_refinement(double screen, uint8_t supersample, uint8_t max_supersample) {
    uint64_t side = uint64_t(std::ceil(screen + 8));
    unsigned ss = supersample;
    while (ss < max_supersample) {
        unsigned next = std::min<unsigned>(ss * 2, max_supersample);
        if (side * side * next * next > kMaxSamples) break;
        ss = next;
    }
    return uint8_t(ss);
}

// chain.cpp:25-36 (Curve::at) and chain.cpp:101-118 (schedule).
int bo_schedule(double first, double last, uint32_t levels, const float* curve_xy, uint32_t points,
                double max_lod0, double* pixels, double* transition, double* source) {
    if (levels < 2 || !points) return 1;
    auto at = [&](double t) {
        if (t <= curve_xy[0]) return double(curve_xy[1]);
        for (uint32_t i = 1; i < points; ++i)
            if (t <= curve_xy[2 * i]) {
                double u = (t - curve_xy[2 * i - 2]) / (curve_xy[2 * i] - curve_xy[2 * i - 2]);
                return curve_xy[2 * i - 1] * (1 - u) + curve_xy[2 * i + 1] * u;
            }
        return double(curve_xy[2 * points - 1]);
    };
    pixels[0] = first;
    transition[0] = source[0] = 0;
    double cumulative = 0;
    for (uint32_t i = 1; i < levels; ++i) {
        double p = first * std::pow(last / first, double(i) / (levels - 1));
        double delta = at(levels == 2 ? 0 : double(i - 1) / (levels - 2));
        cumulative = cumulative * p / pixels[i - 1] + delta;
        pixels[i] = p;
        transition[i] = delta;
        source[i] = max_lod0 > 0 ? std::min(cumulative, max_lod0) : cumulative;
    }
    return 0;
}

int64_t bo_actions(const bo_mesh* m, int placement, int preserve_uv, bo_edit* out, uint64_t capacity) {
    int64_t count = -1;
    int status = guarded([&] {
        UvWelded hold;
        const bo_mesh& sm = state_mesh(*m, preserve_uv != 0, hold);
        auto t = build_topology(sm, preserve_uv != 0);
        auto edits = enumerate(sm, t, placement != 0, preserve_uv != 0);
        for (size_t i = 0; i < edits.size() && i < capacity; ++i) out[i] = edits[i];
        count = int64_t(edits.size());
    });
    return status ? -1 : count;
}

int bo_topology_flags(const bo_mesh* m, uint32_t* geometry, uint8_t* boundary, uint8_t* invalid) {
    return guarded([&] {
        auto t = build_topology(*m, true);
        std::copy(t.geometry.begin(), t.geometry.end(), geometry);
        std::copy(t.boundary.begin(), t.boundary.end(), boundary);
        std::copy(t.invalid.begin(), t.invalid.end(), invalid);
    });
}

int64_t bo_trial_midpoint(const bo_mesh* m, const bo_edit* e, int preserve_uv, uint32_t* indices,
                          float* positions, float* uv, uint8_t* valid) {
    int64_t faces = -1;
    int status = guarded([&] {
        UvWelded hold;
        const bo_mesh& sm = state_mesh(*m, preserve_uv != 0, hold);
        auto t = build_topology(sm, preserve_uv != 0);
        bo_edit edit{};
        edit.from = e->from, edit.to = e->to;
        if (edit.from >= sm.vertex_count || edit.to >= sm.vertex_count || edit.from == edit.to ||
            !has_neighbor(t, edit.from, edit.to) || !legal(sm, t, edit, true, preserve_uv != 0))
            throw std::invalid_argument("illegal collapse");
        Trial tr = make_trial(sm, t, sm, t, edit, preserve_uv != 0);
        std::copy(tr.indices.begin(), tr.indices.end(), indices);
        std::copy(tr.positions.begin(), tr.positions.end(), positions);
        if (uv && m->uv) std::copy(tr.uv.begin(), tr.uv.end(), uv);
        *valid = tr.valid;
        faces = int64_t(tr.indices.size() / 3);
    });
    return status ? -1 : faces;
}

// Greedy executor with batches of one (execute_actions, action.cpp:453-525;
// GpuActionState::execute, action_gpu.cu:1947-2086): rank the legal midpoint
// collapses (ShortestEdge), walk them in rank order skipping those that would
// remove more faces than remain above target, audit each through the four
// gates against source and previous, commit the first accepted, re-rank; stop
// at the target, the trial budget, no legal action or no accepted action.
// stop: 0 target reached, 1 trial budget, 2 no legal actions, 3 no accepted action.
int bo_execute(const bo_mesh* source, const bo_mesh* previous, uint32_t target, uint32_t budget,
               const bo_eval_settings gates[4], int preserve_uv, uint32_t* commits_from_to, uint32_t capacity,
               uint32_t* commits, uint32_t* trials, uint32_t* out_indices, uint32_t* out_faces, float* out_positions,
               uint8_t* stop) {
    return bo_execute_batched(source, previous, target, budget, gates, preserve_uv, 1, commits_from_to, capacity,
                              commits, trials, out_indices, out_faces, out_positions, stop);
}

// The same walk with batches of up to `batch` independent collapses: select a
// disjoint batch from the current ranked position, audit its combined trial,
// halve it on rejection, and after a rejected singleton continue one past the
// batch's first edit (execute_actions, action.cpp:486-515; select_batch and
// verdict, action_gpu.cu:865-915).
int bo_execute_batched(const bo_mesh* source, const bo_mesh* previous, uint32_t target, uint32_t budget,
                       const bo_eval_settings gates[4], int preserve_uv, uint32_t batch,
                       uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits, uint32_t* trials,
                       uint32_t* out_indices, uint32_t* out_faces, float* out_positions, uint8_t* stop) {
    return bo_execute_from(source, previous, nullptr, target, budget, gates, preserve_uv, batch, 3, commits_from_to,
                           capacity, commits, trials, out_indices, out_faces, out_positions, stop, nullptr);
}

// The same walk starting from `start` (a later state of `source`: same vertex
// slots, fewer faces) instead of from the source itself; the geometric
// classes stay those welded on the source (a chain's levels continue one
// state, generate.cpp:456-562).
}
namespace {
// Endpoint trial of the reference CPU executor (ActionState::trial(span),
// action.cpp:308-345): the wedge remap of every edit, faces that become
// degenerate in classes dropped, positions unchanged.
Trial make_endpoint_trial(const bo_mesh& m, const Topology& t, const std::vector<bo_edit>& batch) {
    Trial out;
    std::vector<uint32_t> remap(m.vertex_count, kNone);
    for (const bo_edit& e : batch)
        for (unsigned j = 0; j < e.wedges; ++j) remap[e.source[j]] = e.target[j];
    for (uint32_t f = 0; f < m.face_count; ++f) {
        uint32_t ids[3];
        bool changed = false;
        for (int j = 0; j < 3; ++j) {
            ids[j] = m.indices[3 * f + j];
            if (remap[ids[j]] != kNone) ids[j] = remap[ids[j]], changed = true;
        }
        if (changed && (t.geometry[ids[0]] == t.geometry[ids[1]] || t.geometry[ids[1]] == t.geometry[ids[2]] ||
                        t.geometry[ids[0]] == t.geometry[ids[2]]))
            continue;
        out.indices.insert(out.indices.end(), ids, ids + 3);
        if (m.materials) out.materials.push_back(m.materials[f]);
    }
    out.positions.assign(m.positions, m.positions + size_t(m.vertex_count) * 3);
    if (m.uv) out.uv.assign(m.uv, m.uv + size_t(m.vertex_count) * 2);
    return out;
}

// The greedy walk of execute_actions (action.cpp:453-525) over midpoint
// collapses (legality with placement, make_trial) or, with `endpoint`, over
// the reference CPU executor's endpoint collapses (legality without
// placement, make_endpoint_trial).
int execute_walk(const bo_mesh* source, const bo_mesh* previous, const bo_mesh* start, uint32_t target,
                 uint32_t budget, const bo_eval_settings gates[4], int preserve_uv, uint32_t batch, int ranking,
                 bool endpoint, uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits, uint32_t* trials,
                 uint32_t* out_indices, uint32_t* out_faces, float* out_positions, uint8_t* stop, float* out_uv) {
    if (!batch || batch > 64 || (ranking != 1 && ranking != 3 && ranking != 4)) return 1;
    if (start && start->vertex_count != source->vertex_count) return 1;
    return guarded([&] {
        ExecState st;
        const bo_mesh& from = start ? *start : *source;
        st.pos.assign(from.positions, from.positions + size_t(from.vertex_count) * 3);
        st.idx.assign(from.indices, from.indices + size_t(from.face_count) * 3);
        // The state's classes and uv-transport source: the source, uv-welded
        // without preserve_uv like the state itself (once, at construction).
        UvWelded hold;
        const bo_mesh& welded_source = endpoint ? *source : state_mesh(*source, preserve_uv != 0, hold);
        if (!endpoint && !preserve_uv) {
            const std::vector<uint32_t> root = weld(*source, false);
            for (uint32_t& i : st.idx) i = root[i];
        }
        if (from.materials) st.mat.assign(from.materials, from.materials + from.face_count);
        if (source->double_sided) st.sided.assign(source->double_sided, source->double_sided + source->double_sided_count);
        if (from.uv) st.uv.assign(from.uv, from.uv + size_t(from.vertex_count) * 2);
        bo_bounds b{};
        bo_bounds_of(source, &b);
        const double diameter = std::max(1e-20, b.radius * 2);
        const bo_mesh& prev = previous ? *previous : *source;
        const Topology classes = build_topology(welded_source, preserve_uv != 0);
        const bo_mesh original = welded_source;
        target = std::max<uint32_t>(1, target);
        uint32_t n_commits = 0, n_trials = 0;
        uint8_t reason = 3;
        for (;;) {
            bo_mesh m = st.view();
            if (m.face_count <= target) {
                reason = 0;
                break;
            }
            if (n_trials >= budget) {
                reason = 1;
                break;
            }
            Topology t = build_topology(m, preserve_uv != 0, &classes);
            std::vector<bo_edit> edits = enumerate(m, t, !endpoint, preserve_uv != 0);
            if (edits.empty()) {
                reason = 2;
                break;
            }
            std::vector<float> scores(edits.size());
            for (size_t i = 0; i < edits.size(); ++i) scores[i] = rank_score(ranking, m, t, edits[i], diameter);
            std::vector<uint32_t> order(edits.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) { return scores[a] > scores[c]; });
            const uint32_t remaining = m.face_count - target;
            bool accepted = false;
            for (size_t pos = 0; pos < order.size() && n_trials < budget && !accepted;) {
                std::vector<size_t> picked = select_batch(t, edits, order, pos, batch, remaining);
                if (picked.empty()) break;
                const size_t first = picked.front();
                while (n_trials < budget) {
                    std::vector<bo_edit> chosen;
                    for (size_t k : picked) chosen.push_back(edits[order[k]]);
                    Trial tr = endpoint ? make_endpoint_trial(m, t, chosen)
                                        : make_trial(m, t, original, classes, chosen, preserve_uv != 0);
                    ++n_trials;
                    if (tr.valid && audit_gates(trial_view(m, tr), *source, prev, b, gates, nullptr)) {
                        for (const bo_edit& e : chosen) {
                            if (n_commits < capacity) {
                                commits_from_to[2 * n_commits] = e.from;
                                commits_from_to[2 * n_commits + 1] = e.to;
                            }
                            ++n_commits;
                        }
                        st.idx = tr.indices;
                        st.pos = tr.positions;
                        if (!st.mat.empty()) st.mat = tr.materials;
                        if (!st.uv.empty()) st.uv = tr.uv;
                        accepted = true;
                        break;
                    }
                    if (picked.size() == 1) break;
                    picked.resize(picked.size() / 2);
                }
                pos = first + 1;
            }
            if (!accepted) {
                reason = n_trials >= budget ? 1 : 3;
                break;
            }
        }
        *commits = n_commits;
        *trials = n_trials;
        *out_faces = uint32_t(st.idx.size() / 3);
        std::copy(st.idx.begin(), st.idx.end(), out_indices);
        std::copy(st.pos.begin(), st.pos.end(), out_positions);
        if (out_uv) std::copy(st.uv.begin(), st.uv.end(), out_uv);
        *stop = reason;
    });
}
} // namespace
extern "C" {

int bo_execute_from(const bo_mesh* source, const bo_mesh* previous, const bo_mesh* start, uint32_t target,
                    uint32_t budget, const bo_eval_settings gates[4], int preserve_uv, uint32_t batch, int ranking,
                    uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits, uint32_t* trials,
                    uint32_t* out_indices, uint32_t* out_faces, float* out_positions, uint8_t* stop,
                    float* out_uv) {
    return execute_walk(source, previous, start, target, budget, gates, preserve_uv, batch, ranking, false,
                        commits_from_to, capacity, commits, trials, out_indices, out_faces, out_positions, stop,
                        out_uv);
}

int bo_execute_endpoint(const bo_mesh* source, uint32_t target, uint32_t budget, const bo_eval_settings gates[4],
                        uint32_t batch, uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits,
                        uint32_t* trials, uint32_t* out_indices, uint32_t* out_faces, uint8_t* stop) {
    std::vector<float> positions(size_t(source->vertex_count) * 3);
    return execute_walk(source, nullptr, nullptr, target, budget, gates, 0, batch, 3, true, commits_from_to,
                        capacity, commits, trials, out_indices, out_faces, positions.data(), stop, nullptr);
}

// Four-gate acceptance of one candidate (generate.cpp:365-388, chain.cpp:470-483):
// source@search, previous@search, source@audit, previous@audit; first failure
// rejects. Each gate's max_supersample is pre-bounded (generate.cpp:356-358).
int bo_audit_candidate(const bo_mesh* parent, const bo_edit* e, const bo_mesh* source,
                       const bo_mesh* previous, const bo_bounds* b, const bo_eval_settings gates[4],
                       int preserve_uv, bo_verdict* out) {
    return guarded([&] {
        *out = bo_verdict{};
        UvWelded hold;
        parent = &state_mesh(*parent, preserve_uv != 0, hold);
        auto t = build_topology(*parent, preserve_uv != 0);
        // The edit's wedges come from legality (action_gpu.cu:487-643), as in
        // the reference executor; only from/to are taken from the caller.
        bo_edit edit{};
        edit.from = e->from, edit.to = e->to;
        if (edit.from >= parent->vertex_count || edit.to >= parent->vertex_count || edit.from == edit.to ||
            !has_neighbor(t, edit.from, edit.to) || !legal(*parent, t, edit, true, preserve_uv != 0)) {
            out->failed_gate = 5;
            return;
        }
        Trial tr = make_trial(*parent, t, *parent, t, edit, preserve_uv != 0);
        out->placement_valid = tr.valid;
        if (!tr.valid) {
            out->failed_gate = 6;
            return;
        }
        bo_mesh cand = trial_view(*parent, tr);
        for (int g = 0; g < 4; ++g) {
            bo_eval_settings s = gates[g];
            s.max_supersample = bo_bounded_refinement(s.screen_size, s.supersample, s.max_supersample);
            const bo_mesh& ref = (g % 2) ? *previous : *source;
            out->gates[g] = evaluate(ref, cand, *b, s);
            if (!measurement_passed(out->gates[g])) {
                out->failed_gate = uint8_t(g + 1);
                return;
            }
        }
        out->accepted = 1;
    });
}
}
