// C shim over BlitzRemesher's own CPU sources — TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the reference's unmodified src/evaluate.cpp,
// src/mesh.cpp, src/neural/action.cpp and src/neural/graph.cpp (see
// oracle/Makefile) into oracle/_ref/libblitz_ref.so. It lets the tests pin the
// oracle restatement against the reference itself and lets the benchmark time
// the reference CPU audit. Nothing in the product links it.
#include "blitz/evaluate.hpp"
#include "coverage.hpp"
#include "neural/action.hpp"
#include "neural/audit_measurement.hpp"
#include "neural/internal.hpp"

#include <cstring>
#include <random>
#include <stdexcept>

using namespace blitz;

extern "C" {
struct br_mesh {
    const float* positions;
    uint32_t vertex_count;
    const uint32_t* indices;
    uint32_t face_count;
    const uint16_t* materials;
    const uint8_t* double_sided;
    uint32_t double_sided_count;
    const float* uv;
};
struct br_bounds {
    float center[3];
    double radius;
};
struct br_camera {
    float right[3], up[3], forward[3];
    double distance, focal, scale;
    uint8_t perspective;
    uint8_t pad[7];
};
struct br_eval_settings {
    double screen_size, limit, max_changed_area;
    uint16_t views_orthographic, views_perspective;
    uint32_t views_seed;
    uint8_t supersample, max_supersample, force_two_sided, conservative_screen;
    uint8_t profile;
    uint8_t pad[3];
};
struct br_measurement {
    double error, coverage, coverage_upper, changed_area, normal_degrees;
    uint32_t worst_view, changed_area_worst_view, views_evaluated;
    uint8_t supersample, complete, passed, resource_limited, cancelled;
    uint8_t pad[3];
};
}

namespace {
MeshView view(const br_mesh& m) {
    MeshView v;
    v.positions = Stream<Vec3>(reinterpret_cast<const Vec3*>(m.positions), m.vertex_count);
    if (m.uv) v.uv = Stream<Vec2>(reinterpret_cast<const Vec2*>(m.uv), m.vertex_count);
    v.indices = {m.indices, size_t(m.face_count) * 3};
    if (m.materials) v.materials = {m.materials, m.face_count};
    if (m.double_sided) v.double_sided = {m.double_sided, m.double_sided_count};
    return v;
}
Bounds bounds_of(const br_bounds& b) { return {{b.center[0], b.center[1], b.center[2]}, b.radius}; }
Camera camera_of(const br_camera& c) {
    Camera k;
    k.right = {c.right[0], c.right[1], c.right[2]};
    k.up = {c.up[0], c.up[1], c.up[2]};
    k.forward = {c.forward[0], c.forward[1], c.forward[2]};
    k.distance = c.distance, k.focal = c.focal, k.scale = c.scale, k.perspective = c.perspective;
    return k;
}
br_camera export_camera(const Camera& k) {
    br_camera c{};
    c.right[0] = k.right.x, c.right[1] = k.right.y, c.right[2] = k.right.z;
    c.up[0] = k.up.x, c.up[1] = k.up.y, c.up[2] = k.up.z;
    c.forward[0] = k.forward.x, c.forward[1] = k.forward.y, c.forward[2] = k.forward.z;
    c.distance = k.distance, c.focal = k.focal, c.scale = k.scale, c.perspective = k.perspective;
    return c;
}
EvalSettings settings_of(const br_eval_settings& s) {
    EvalSettings e;
    e.profile = Profile(s.profile);
    e.screen_size = s.screen_size;
    e.limit = s.limit;
    e.max_changed_area = s.max_changed_area;
    e.views = {s.views_orthographic, s.views_perspective, s.views_seed};
    e.supersample = s.supersample;
    e.max_supersample = s.max_supersample;
    e.force_two_sided = s.force_two_sided;
    e.conservative_screen = s.conservative_screen;
    return e;
}
br_measurement export_measurement(const Measurement& m) {
    br_measurement o{};
    o.error = m.error, o.coverage = m.coverage, o.coverage_upper = m.coverage_upper;
    o.changed_area = m.changed_area, o.normal_degrees = m.normal_degrees;
    o.worst_view = m.worst_view, o.changed_area_worst_view = m.changed_area_worst_view;
    o.views_evaluated = m.views_evaluated, o.supersample = m.supersample;
    o.complete = m.complete, o.passed = m.passed, o.resource_limited = m.resource_limited;
    o.cancelled = m.cancelled;
    return o;
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
int br_bounds_of(const br_mesh* m, br_bounds* out) {
    return guarded([&] {
        auto b = blitz::bounds(view(*m));
        out->center[0] = b.center.x, out->center[1] = b.center.y, out->center[2] = b.center.z;
        out->radius = b.radius;
    });
}
int br_cameras(const br_bounds* b, double screen, uint16_t ortho, uint16_t persp, uint32_t seed,
               br_camera* out) {
    return guarded([&] {
        auto cams = cameras(bounds_of(*b), screen, ViewSet{ortho, persp, seed});
        for (size_t i = 0; i < cams.size(); ++i) out[i] = export_camera(cams[i]);
    });
}
int br_rasterize_coverage(const br_mesh* m, const br_bounds* b, const br_camera* c, double screen,
                          uint8_t ss, int force_two, uint64_t* words, uint8_t* clipped) {
    return guarded([&] {
        auto r = detail::rasterize_coverage(view(*m), bounds_of(*b), camera_of(*c), screen, ss, force_two != 0);
        std::memcpy(words, r.words.data(), r.words.size() * 8);
        *clipped = r.clipped;
    });
}
int br_coverage_distance(const uint64_t* a, const uint64_t* b, uint32_t width, uint32_t height,
                         uint8_t ss, int scalar, double* out) {
    return guarded([&] {
        size_t n = (size_t(width) * height + 63) / 64;
        detail::CoverageRaster ra{width, height, {a, a + n}, false}, rb{width, height, {b, b + n}, false};
        *out = detail::coverage_distance(ra, rb, ss, scalar != 0);
    });
}
int br_evaluate(const br_mesh* reference, const br_mesh* candidate, const br_bounds* b,
                const br_eval_settings* s, br_measurement* out) {
    return guarded([&] {
        *out = export_measurement(evaluate(view(*reference), view(*candidate), bounds_of(*b), settings_of(*s)));
    });
}
uint8_t br_bounded_refinement(double screen, uint8_t ss, uint8_t max_ss) {
    EvalSettings e;
    e.screen_size = screen, e.supersample = ss, e.max_supersample = max_ss;
    return neural::bounded_refinement(e);
}
// Endpoint-collapse action set of the reference CPU executor (action.cpp:371-452).
int64_t br_actions(const br_mesh* m, uint32_t* from_to, uint64_t capacity) {
    int64_t count = -1;
    int status = guarded([&] {
        neural::ActionState state(view(*m));
        std::array<float, neural::conditions> c{};
        auto rows = state.actions(c);
        for (size_t i = 0; i < rows.size() && i < capacity; ++i) {
            from_to[2 * i] = rows[i].action.from;
            from_to[2 * i + 1] = rows[i].action.to;
        }
        count = int64_t(rows.size());
    });
    return status ? -1 : count;
}
// Endpoint trial of the reference CPU executor (action.cpp:305-345).
int64_t br_trial_endpoint(const br_mesh* m, uint32_t from, uint32_t to, uint32_t* indices) {
    int64_t faces = -1;
    int status = guarded([&] {
        neural::ActionState state(view(*m));
        auto lod = state.trial(neural::Action{from, to, 0});
        std::memcpy(indices, lod.data.indices.data(), lod.data.indices.size() * 4);
        faces = int64_t(lod.data.indices.size() / 3);
    });
    return status ? -1 : faces;
}
// The reference CPU executor itself (neural::execute_actions,
// action.cpp:453-525): endpoint collapses, batches of 1..64, a ShortestEdge
// ranker (minus the edge length over the source diameter, each component of
// the scaled delta rounded to float: the formula of rank_actions,
// action_gpu.cu:822-825) and the four-gate ActionGate over blitz::evaluate
// (source and previous are both the input; each gate's max_supersample
// pre-bounded, graph.cpp:5-18; pass = audit_measurement_passed). Writes the
// final indices; stop: 0 target reached, 1 trial budget, 2 no legal actions,
// 3 no accepted action.
int br_execute_actions(const br_mesh* m, uint32_t target, uint32_t budget, const br_eval_settings gates[4],
                       uint32_t batch, uint32_t* out_indices, uint32_t* out_faces, uint64_t* trials,
                       uint64_t* accepted, uint64_t* rejected, uint8_t* stop) {
    return guarded([&] {
        const MeshView input = view(*m);
        const Bounds b = bounds(input);
        const double diameter = std::max(1e-20, b.radius * 2);
        neural::ActionRanker rank = [&](const neural::ActionState& state,
                                        std::span<const neural::ActionRecord> rows) {
            std::vector<float> scores(rows.size());
            const MeshView v = state.view();
            for (size_t i = 0; i < rows.size(); ++i) {
                const Vec3 d = (v.positions[rows[i].action.to] - v.positions[rows[i].action.from]) * (1 / diameter);
                scores[i] = -float(length(d));
            }
            return scores;
        };
        neural::ActionGate gate = [&](MeshView candidate) {
            for (int g = 0; g < 4; ++g) {
                EvalSettings s = settings_of(gates[g]);
                s.max_supersample = neural::bounded_refinement(s);
                if (!neural::audit_measurement_passed(evaluate(input, candidate, b, s))) return false;
            }
            return true;
        };
        std::array<float, neural::conditions> c{};
        neural::ActionStats stats;
        Lod lod = neural::execute_actions(input, c, target, budget, rank, gate, &stats, {}, batch);
        std::memcpy(out_indices, lod.data.indices.data(), lod.data.indices.size() * 4);
        *out_faces = uint32_t(lod.data.indices.size() / 3);
        *trials = stats.trials, *accepted = stats.accepted, *rejected = stats.rejected;
        *stop = uint8_t(stats.stop_reason);
    });
}
// The random mask pairs of tests/precision.cpp:82-91 (mt19937 seed 2921, 13x11).
void br_precision_masks(uint32_t seed, uint32_t trials, uint64_t* a_out, uint64_t* b_out) {
    std::mt19937 random(seed);
    for (uint32_t t = 0; t < trials; ++t) {
        uint64_t a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
        for (size_t i = 0; i < 143; ++i) {
            if (random() % 5 == 0) a[i / 64] |= uint64_t(1) << (i % 64);
            if (random() % 7 == 0) b[i / 64] |= uint64_t(1) << (i % 64);
        }
        std::memcpy(a_out + 3 * t, a, 24);
        std::memcpy(b_out + 3 * t, b, 24);
    }
}
}
