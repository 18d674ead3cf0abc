// Host runtime and C ABI of the B200 candidate-audit engine.
//
// A session owns the source (LOD0), the bound previous LOD, the current state
// with its collapse topology, the audit plans (cameras + resident reference
// masks and state counts per view) and all scratch. Every buffer is allocated
// through the session pool, which enforces blitz_neural_options_v2::memory_mib.
#include "../../include/blitz_audit.h"
#include "kernels.cuh"
#include "surrogate.cuh"

#include <algorithm>
#include <type_traits>
#include <chrono>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace b200 {

struct Failure : std::runtime_error {
    blitz_status status;
    Failure(blitz_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define B200_CUDA(x)                                                                                              \
    do {                                                                                                         \
        cudaError_t e_ = (x);                                                                                    \
        if (e_ != cudaSuccess)                                                                                   \
            throw Failure(e_ == cudaErrorMemoryAllocation ? BLITZ_OUT_OF_MEMORY : BLITZ_INTERNAL_ERROR,          \
                          std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #x);                           \
    } while (0)

// ---------------------------------------------------------------------------
// Device memory with a byte budget.
struct Pool {
    size_t limit = 0, used = 0, peak = 0, allocations = 0;
    void* get(size_t bytes) {
        if (!bytes) return nullptr;
        if (used + bytes > limit)
            throw Failure(BLITZ_OUT_OF_MEMORY, "audit workspace exceeds memory_mib budget");
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Failure(BLITZ_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        used += bytes;
        peak = std::max(peak, used);
        ++allocations;
        return p;
    }
    void put(void* p, size_t bytes) {
        if (p) {
            cudaFree(p);
            used -= bytes;
        }
    }
};

template <class T> struct Buf {
    Pool* pool = nullptr;
    T* p = nullptr;
    size_t n = 0;
    Buf() = default;
    Buf(Pool& pl, size_t count) : pool(&pl), p(static_cast<T*>(pl.get(count * sizeof(T)))), n(count) {}
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    Buf(Buf&& o) noexcept : pool(o.pool), p(o.p), n(o.n) { o.p = nullptr, o.n = 0; }
    Buf& operator=(Buf&& o) noexcept {
        if (this != &o) {
            release();
            pool = o.pool, p = o.p, n = o.n;
            o.p = nullptr, o.n = 0;
        }
        return *this;
    }
    ~Buf() { release(); }
    void release() {
        if (pool && p) pool->put(p, n * sizeof(T));
        p = nullptr, n = 0;
    }
    void ensure(Pool& pl, size_t count) {
        if (n < count) {
            release();
            *this = Buf(pl, count);
        }
    }
};

// ---------------------------------------------------------------------------
// Host mesh copied out of a borrowed blitz_mesh (streams may be strided).
struct HostMesh {
    std::vector<float> pos, normals, uv, tangents;
    std::vector<uint8_t> colors;
    std::vector<uint32_t> idx;
    std::vector<uint16_t> mat;
    std::vector<uint8_t> sided;
    uint32_t nv() const { return uint32_t(pos.size() / 3); }
    uint32_t nf() const { return uint32_t(idx.size() / 3); }
};

template <class T>
static void copy_stream(const blitz_stream& s, size_t n, size_t comps, std::vector<T>& out, const char* name) {
    if (!s.count) return;
    if (!s.data || s.count != n || s.stride < comps * sizeof(T))
        throw Failure(BLITZ_INVALID_ARGUMENT, std::string("invalid ") + name + " stream");
    out.resize(n * comps);
    const unsigned char* b = static_cast<const unsigned char*>(s.data);
    for (size_t i = 0; i < n; ++i) std::memcpy(out.data() + i * comps, b + i * s.stride, comps * sizeof(T));
}

// Descriptor checks of c_api.cpp and validate(MeshView) (mesh.cpp:29-42).
static HostMesh import_mesh(const blitz_mesh* m) {
    if (!m || m->struct_size != sizeof(blitz_mesh) || m->abi_version != BLITZ_ABI_VERSION)
        throw Failure(BLITZ_INVALID_ARGUMENT, "invalid mesh descriptor");
    HostMesh h;
    size_t n = m->positions.count;
    if (!n || n >= UINT32_MAX || !m->indices || !m->index_count || m->index_count % 3 || m->index_count >= UINT32_MAX)
        throw Failure(BLITZ_INVALID_ARGUMENT, "mesh requires nonempty triangle indices and 32-bit representable counts");
    copy_stream<float>(m->positions, n, 3, h.pos, "position");
    copy_stream<float>(m->normals, n, 3, h.normals, "normal");
    copy_stream<float>(m->uv, n, 2, h.uv, "uv");
    copy_stream<uint8_t>(m->colors, n, 4, h.colors, "color");
    copy_stream<float>(m->tangents, n, 4, h.tangents, "tangent");
    h.idx.assign(m->indices, m->indices + m->index_count);
    size_t nf = m->index_count / 3;
    if (m->material_count) {
        if (!m->materials || m->material_count != nf)
            throw Failure(BLITZ_INVALID_ARGUMENT, "material count differs from triangle count");
        h.mat.assign(m->materials, m->materials + nf);
    }
    if (m->double_sided_count) {
        if (!m->double_sided) throw Failure(BLITZ_INVALID_ARGUMENT, "invalid double-sided flags");
        h.sided.assign(m->double_sided, m->double_sided + m->double_sided_count);
    }
    for (uint32_t i : h.idx)
        if (i >= n) throw Failure(BLITZ_INVALID_ARGUMENT, "index outside vertex stream");
    for (float f : h.pos)
        if (!std::isfinite(f)) throw Failure(BLITZ_INVALID_ARGUMENT, "nonfinite position or normal");
    for (float f : h.normals)
        if (!std::isfinite(f)) throw Failure(BLITZ_INVALID_ARGUMENT, "nonfinite position or normal");
    for (float f : h.uv)
        if (!std::isfinite(f)) throw Failure(BLITZ_INVALID_ARGUMENT, "nonfinite UV");
    return h;
}

// Attribute classes of the GPU state (action_gpu.cu:57-60 same_attributes,
// 178-211 insert/lookup_vertices with attributes): slots with bitwise equal
// positions, normals and colours, and with `with_uv` also uv and tangents,
// share a class named by its smallest slot.
static std::vector<uint32_t> attribute_roots(const HostMesh& h, bool with_uv) {
    const uint32_t n = h.nv();
    auto key = [&](uint32_t i) {
        std::vector<uint32_t> k;
        auto add = [&](const auto& v, size_t comps) {
            if (v.empty()) return;
            using T = typename std::decay_t<decltype(v)>::value_type;
            for (size_t c = 0; c < comps; ++c) {
                uint32_t b = 0;
                std::memcpy(&b, &v[i * comps + c], sizeof(T));
                k.push_back(b);
            }
        };
        add(h.pos, 3);
        add(h.normals, 3);
        add(h.colors, 4);
        if (with_uv) add(h.uv, 2), add(h.tangents, 4);
        return k;
    };
    std::vector<std::vector<uint32_t>> keys(n);
    for (uint32_t i = 0; i < n; ++i) keys[i] = key(i);
    std::vector<uint32_t> order(n), root(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(),
              [&](uint32_t a, uint32_t b) { return keys[a] != keys[b] ? keys[a] < keys[b] : a < b; });
    for (uint32_t k = 0; k < n; ++k)
        root[order[k]] = k && keys[order[k]] == keys[order[k - 1]] ? root[order[k - 1]] : order[k];
    return root;
}

struct Bounds {
    float center[3];
    double radius;
};
// mesh.cpp:12-20
static Bounds bounds_of(const HostMesh& m) {
    Bounds b{};
    float lo[3] = {m.pos[0], m.pos[1], m.pos[2]}, hi[3] = {lo[0], lo[1], lo[2]};
    for (uint32_t i = 1; i < m.nv(); ++i)
        for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], m.pos[3 * i + k]), hi[k] = std::max(hi[k], m.pos[3 * i + k]);
    for (int k = 0; k < 3; ++k) b.center[k] = float((double(lo[k]) + hi[k]) * .5);
    for (uint32_t i = 0; i < m.nv(); ++i) {
        double x = double(m.pos[3 * i]) - b.center[0], y = double(m.pos[3 * i + 1]) - b.center[1],
               z = double(m.pos[3 * i + 2]) - b.center[2];
        b.radius = std::max(b.radius, std::sqrt(x * x + y * y + z * z));
    }
    return b;
}

// Cameras on the host with the platform libm, as the reference
// (evaluate.cpp:16-20, 108-124): Fibonacci sphere, seed rotation, ortho first.
struct F3 {
    float x, y, z;
};
static double dotd(F3 a, F3 b) { return double(a.x) * b.x + double(a.y) * b.y + double(a.z) * b.z; }
static F3 crossf(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static F3 normalizedf(F3 a) {
    double l = std::sqrt(dotd(a, a));
    if (!(l > 0)) return {0, 0, 0};
    double s = 1 / l;
    return {float(a.x * s), float(a.y * s), float(a.z * s)};
}
static F3 rotatef(F3 v, uint32_t seed) {
    double a = (seed % 65521) * .000731, b = ((seed >> 8) % 32749) * .000913;
    double x = v.x * std::cos(a) - v.y * std::sin(a), y = v.x * std::sin(a) + v.y * std::cos(a);
    return {float(x), float(y * std::cos(b) - v.z * std::sin(b)), float(y * std::sin(b) + v.z * std::cos(b))};
}
static std::vector<Camera> make_cameras(const Bounds& b, double screen, uint16_t ortho, uint16_t persp, uint32_t seed) {
    constexpr double pi = 3.14159265358979323846;
    std::vector<Camera> out;
    for (int projection = 0; projection < 2; ++projection) {
        unsigned count = projection ? persp : ortho;
        for (unsigned i = 0; i < count; ++i) {
            double z = 1 - 2 * (i + .5) / count, r = std::sqrt(std::max(0.0, 1 - z * z)),
                   angle = i * pi * (3 - std::sqrt(5.0));
            F3 fwd = normalizedf(rotatef({float(r * std::cos(angle)), float(z), float(r * std::sin(angle))},
                                         seed + projection * 104729u));
            F3 hint = std::abs(fwd.y) > .99 ? F3{1, 0, 0} : F3{0, 1, 0};
            F3 right = normalizedf(crossf(hint, fwd)), up = normalizedf(crossf(fwd, right));
            double height = std::max(1024.0, 2 * screen), focal = height / (2 * std::tan(pi / 6));
            double distance = b.radius * std::sqrt(1 + std::pow(2 * focal / screen, 2));
            Camera c{};
            c.right[0] = right.x, c.right[1] = right.y, c.right[2] = right.z;
            c.up[0] = up.x, c.up[1] = up.y, c.up[2] = up.z;
            c.forward[0] = fwd.x, c.forward[1] = fwd.y, c.forward[2] = fwd.z;
            c.distance = distance, c.focal = focal, c.scale = screen / (b.radius * 2), c.perspective = projection;
            out.push_back(c);
        }
    }
    return out;
}

// evaluation_settings.hpp:10-23 (coverage profile).
static GateSettings gate_of(const blitz_eval_settings* s, const Bounds& b) {
    if (!s || s->struct_size != sizeof(blitz_eval_settings))
        throw Failure(BLITZ_INVALID_ARGUMENT, "invalid evaluation settings descriptor");
    if (s->profile != 0) throw Failure(BLITZ_UNAVAILABLE, "only the coverage profile is implemented");
    bool center_ok = std::isfinite(b.center[0]) && std::isfinite(b.center[1]) && std::isfinite(b.center[2]);
    if (!(s->screen_size > 0) || !std::isfinite(s->screen_size) || s->screen_size > 16384 || !(b.radius > 0) ||
        !std::isfinite(b.radius) || !center_ok || !(s->limit >= 0) || !std::isfinite(s->limit) || !s->supersample ||
        s->max_supersample < s->supersample || s->max_supersample > 32 || !std::isfinite(s->max_changed_area) ||
        s->max_changed_area < 0 || s->max_changed_area > 1)
        throw Failure(BLITZ_INVALID_ARGUMENT, "invalid evaluation settings");
    if (!s->views_orthographic && !s->views_perspective)
        throw Failure(BLITZ_INVALID_ARGUMENT, "at least one camera required");
    GateSettings g{};
    g.screen_size = s->screen_size, g.limit = s->limit, g.max_changed_area = s->max_changed_area;
    g.views = uint32_t(s->views_orthographic) + s->views_perspective;
    g.supersample = s->supersample, g.max_supersample = s->max_supersample;
    g.conservative_screen = s->conservative_screen;
    return g;
}

// ---------------------------------------------------------------------------
struct DeviceMesh {
    Buf<float> pos, uv;
    Buf<uint32_t> idx;
    Buf<uint16_t> mat;
    Buf<uint8_t> sided;
    DevMesh view{};
    void upload(Pool& pool, const HostMesh& h, cudaStream_t s) {
        pos = Buf<float>(pool, h.pos.size());
        idx = Buf<uint32_t>(pool, h.idx.size());
        B200_CUDA(cudaMemcpyAsync(pos.p, h.pos.data(), h.pos.size() * 4, cudaMemcpyHostToDevice, s));
        B200_CUDA(cudaMemcpyAsync(idx.p, h.idx.data(), h.idx.size() * 4, cudaMemcpyHostToDevice, s));
        if (!h.uv.empty()) {
            uv = Buf<float>(pool, h.uv.size());
            B200_CUDA(cudaMemcpyAsync(uv.p, h.uv.data(), h.uv.size() * 4, cudaMemcpyHostToDevice, s));
        }
        if (!h.mat.empty()) {
            mat = Buf<uint16_t>(pool, h.mat.size());
            B200_CUDA(cudaMemcpyAsync(mat.p, h.mat.data(), h.mat.size() * 2, cudaMemcpyHostToDevice, s));
        }
        if (!h.sided.empty()) {
            sided = Buf<uint8_t>(pool, h.sided.size());
            B200_CUDA(cudaMemcpyAsync(sided.p, h.sided.data(), h.sided.size(), cudaMemcpyHostToDevice, s));
        }
        view = DevMesh{pos.p, idx.p, mat.p, sided.p, uv.p, h.nv(), h.nf(), uint32_t(h.sided.size()), 0};
    }
};

static bool same_data(const HostMesh& a, const HostMesh& b) {
    return a.pos == b.pos && a.idx == b.idx && a.mat == b.mat && a.sided == b.sided && a.normals == b.normals &&
           a.colors == b.colors && a.uv == b.uv;
}
// evaluate.cpp:77-82 — positions, normals, colours, indices, materials, sides.
static bool identical(const HostMesh& a, const HostMesh& b) {
    return a.pos == b.pos && a.normals == b.normals && a.colors == b.colors && a.idx == b.idx && a.mat == b.mat &&
           a.sided == b.sided;
}

struct Topology {
    Buf<uint32_t> geometry, canonical, face_offsets, faces, cursor, entries, nbr_offsets, neighbors, slot_offsets,
        slots, scan, table;
    Buf<uint8_t> nbr_count, boundary, invalid;
    Buf<uint32_t> edge_base, offsets, flat;
    Buf<uint8_t> valid;
    Buf<Edit> edit_slots, edits;
    Buf<uint32_t> positions; // live position table
    uint32_t table_cap = 0, pos_cap = 0, total_nbrs = 0, actions = 0;
    DevTopology view{};
    // uv transport: source faces per canonical class
    Buf<uint32_t> uv_offsets, uv_faces;
    UvSource uvs{};
    const UvSource* uv() const { return uvs.uv ? &uvs : nullptr; }
};

static uint32_t pow2_at_least(uint64_t n) {
    uint64_t c = 2;
    while (c < n) c *= 2;
    if (c > (1ull << 31)) throw Failure(BLITZ_OUT_OF_MEMORY, "hash table exceeds u32");
    return uint32_t(c);
}

struct PlanKey {
    int reference;
    uint16_t ortho, persp;
    uint32_t seed;
    double screen;
    uint32_t ss, force_two;
    bool operator<(const PlanKey& o) const {
        return std::tie(reference, ortho, persp, seed, screen, ss, force_two) <
               std::tie(o.reference, o.ortho, o.persp, o.seed, o.screen, o.ss, o.force_two);
    }
};

// A plan keeps, per view, the reference mask (CPU semantics) and the current
// state's per-sample face counts, coverage and popcounts against the
// reference. Once the state differs from the reference, a plan also keeps the
// reference's exact distance field (built then, not before) and the state's
// 32x32 tile maxima (from a field computed per refresh and not kept), so
// candidates of such a state stay on the incremental path at every raster
// size up to 4160 x 4160.
struct Plan {
    PlanKey key{};
    uint32_t size = 0, views = 0, words = 0;
    bool resource_limited = false, tiled = false, ref_box_clip = false;
    Buf<Camera> cameras;
    std::vector<Camera> hcams;
    Buf<uint32_t> ref_bits, state_bits, ref_field;
    Buf<int32_t> t1, t2;
    Buf<uint8_t> state_count;
    Buf<PlanView> dviews;
    std::vector<PlanView> hviews;
    bool state_is_ref = true;
    bool deep = false; // a raster of this plan had a sample under more than 255 faces
    uint64_t state_revision = ~0ull;
    Buf<ViewRecord> records;
    Buf<uint32_t> raster_state;      // 4 words per view
    Buf<unsigned long long> pop;     // 4 counts per view
    std::vector<uint32_t> hstate;
    std::vector<unsigned long long> hpop;
    // The last combined trial evaluated on this plan, laid out like the state
    // data (so a commit of that trial swaps it in).
    Buf<uint8_t> trial_count;
    Buf<uint32_t> trial_bits, trial_state;
    Buf<int32_t> trial_t1, trial_t2, trial_max;
    Buf<unsigned long long> trial_pop;
    std::vector<uint32_t> trial_hstate;
    std::vector<unsigned long long> trial_hpop;
    std::vector<int32_t> trial_hmax;
    uint64_t trial_tag = 0;
    PlanDev dev{};
};

struct Scratch {
    Buf<uint32_t> a, c, g, d2, maxes, state;
    Buf<int32_t> sv;
    Buf<long long> sn, sd;
    Buf<unsigned long long> pop;
    size_t samples = 0;
    // per-view scratch of the batched reference fields (row distances,
    // envelope stacks)
    Buf<uint32_t> vg;
    // 32-bit face counts of all views of a plan with deep overlaps
    Buf<uint32_t> wide;
    Buf<int32_t> vsv;
    Buf<long long> vsn, vsd;
    size_t view_entries = 0;
};

// Surrogate parameters on one device: FP32 masters (W1 128x64, b1 128, W2
// 128x128, b2 128, W3 16x128, b3 16), Adam moments, BF16 copies at the same
// offsets, gradient accumulators and the feature normalisation.
constexpr uint32_t kOffW1 = 0, kOffB1 = 8192, kOffW2 = 8320, kOffB2 = 24704, kOffW3 = 24832, kOffB3 = 26880,
                   kParams = 26896;
struct SurrogateModel {
    int device = 0;
    cudaStream_t stream = nullptr;
    Pool pool;
    Buf<float> master, grads, m, v, norm, loss;
    Buf<__nv_bfloat16> wb;
    Buf<uint8_t> mask;
    Buf<uint32_t> error;
    uint32_t step = 0;
    SurrogateDev dev() const {
        SurrogateDev d{};
        d.w1b = wb.p + kOffW1, d.w2b = wb.p + kOffW2, d.w3b = wb.p + kOffW3;
        d.b1 = master.p + kOffB1, d.b2 = master.p + kOffB2, d.b3 = master.p + kOffB3;
        d.mean = norm.p, d.inv_std = norm.p + kSurrogateIn;
        d.gw1 = grads.p + kOffW1, d.gw2 = grads.p + kOffW2, d.gw3 = grads.p + kOffW3;
        d.gb1 = grads.p + kOffB1, d.gb2 = grads.p + kOffB2, d.gb3 = grads.p + kOffB3;
        return d;
    }
    ~SurrogateModel() {
        master.release(), grads.release(), m.release(), v.release(), norm.release(), loss.release();
        wb.release(), mask.release(), error.release();
        if (stream) cudaStreamDestroy(stream);
    }
};
// Parameters that exist (the padding of W1's inputs and of W3/b3's outputs
// stays zero).
static bool surrogate_param_live(uint32_t i) {
    if (i < kOffB1) return (i % 64) < uint32_t(kSurrogateIn);
    if (i >= kOffW3 && i < kOffB3) return (i - kOffW3) / 128 < 2;
    if (i >= kOffB3) return i - kOffB3 < 2;
    return true;
}

struct Session {
    int device = 0;
    cudaStream_t stream = nullptr;
    Pool pool;
    blitz_neural_options_v2 options{};
    HostMesh source_h, previous_h;
    bool previous_is_source = true;
    DeviceMesh source, previous, state;
    uint32_t state_faces = 0;       // live faces of the state
    uint64_t state_revision = 0;    // bumped by every commit
    bool state_is_source = true;    // no commit since creation or reset
    Bounds bounds{};
    Topology topo;
    std::map<PlanKey, std::unique_ptr<Plan>> plans;
    Scratch scratch;
    Buf<CandidateRecord> records;
    Buf<uint8_t> verdict_dev;
    Buf<Measurement> meas_dev;
    Buf<blitz_collapse> collapse_dev;
    Buf<uint32_t> exact_count, work_queue, spill, spill_huge, spill_giant;
    Buf<const ViewRecord*> record_table;
    Buf<uint32_t> plan_views, plan_ss;
    Buf<GateDev> gate_table;
    Buf<int32_t> view_maxima; // per view max t1 / t2 of a plan (chain confirmation)
    // exact path and commits
    DeviceMesh trial;
    Buf<uint32_t> trial_keep, trial_offsets;
    Buf<TrialInfo> trial_info;
    Buf<blitz_collapse> trial_collapse;
    // surrogate pruning (non-owning model; buffers at the edit capacity)
    struct SurrogateModel* surrogate = nullptr;
    Buf<float> sur_features, sur_out, sur_keys_in, sur_keys_out;
    Buf<uint32_t> sur_idx_in, sur_idx_out, sur_flags, sur_rank_flags, sur_offsets, sur_order;
    Buf<unsigned char> sur_sort_temp;
    size_t sur_sort_bytes = 0;
    // batched executor
    Buf<uint32_t> batch_selected, batch_ctl, batch_out, batch_used, batch_remap, batch_owner, batch_table,
        batch_info;
    Buf<float> batch_placements;
    uint32_t batch_table_cap = 0;
    uint64_t trial_tag = 0;
    // executor ranking
    Buf<float> scores, sorted_scores;
    Buf<uint32_t> order, sorted_order;
    Buf<unsigned char> sort_temp;
    size_t sort_bytes = 0;
    blitz_neural_info info{};
    uint64_t internal_errors = 0;
    std::vector<uint8_t> table_signature; // last uploaded verdict tables
    // profiling: device times of candidate calls; work counters as well
    // (per-unit clock and counter atomics in the audit kernels) when counting
    bool profiling = false, counting = false;
    blitz_audit_profile profile{};
    Buf<unsigned long long> stats;
    cudaEvent_t ev[6] = {};

    ~Session() {
        plans.clear();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct DeviceScope {
    int previous = 0;
    explicit DeviceScope(int id) {
        B200_CUDA(cudaGetDevice(&previous));
        B200_CUDA(cudaSetDevice(id));
    }
    ~DeviceScope() { cudaSetDevice(previous); }
};

// Geometric classes of the episode's first mesh, welded once; topology
// buffers at the session's capacity (the state only loses faces).
static void init_topology(Session& S) {
    Topology& t = S.topo;
    const DevMesh& m = S.state.view;
    const uint32_t n = m.nv, nf = m.nf;
    Pool& P = S.pool;
    t.table_cap = pow2_at_least(2ull * n);
    t.geometry = Buf<uint32_t>(P, n);
    t.table = Buf<uint32_t>(P, t.table_cap);
    launch_weld(m, t.table.p, t.table_cap, false, t.geometry.p, S.stream);
    t.face_offsets = Buf<uint32_t>(P, n + 1);
    t.faces = Buf<uint32_t>(P, 3ull * nf);
    t.cursor = Buf<uint32_t>(P, 2ull * (n + 1));
    t.entries = Buf<uint32_t>(P, 6ull * nf);
    t.nbr_offsets = Buf<uint32_t>(P, n + 1);
    t.neighbors = Buf<uint32_t>(P, 6ull * nf);
    t.nbr_count = Buf<uint8_t>(P, 6ull * nf);
    t.boundary = Buf<uint8_t>(P, n);
    t.invalid = Buf<uint8_t>(P, n);
    t.slot_offsets = Buf<uint32_t>(P, n + 1);
    t.slots = Buf<uint32_t>(P, n);
    size_t scan_words = std::max(scan_scratch_words(n + 1), scan_scratch_words(uint32_t(6ull * nf + 1)));
    t.scan = Buf<uint32_t>(P, scan_words + 64);
    t.edge_base = Buf<uint32_t>(P, n + 1);
    t.valid = Buf<uint8_t>(P, 6ull * nf + 1);
    t.edit_slots = Buf<Edit>(P, 6ull * nf + 1);
    t.offsets = Buf<uint32_t>(P, 6ull * nf + 1);
    t.edits = Buf<Edit>(P, 6ull * nf + 1);
    t.flat = Buf<uint32_t>(P, 1);
    t.pos_cap = pow2_at_least(4ull * n);
    t.positions = Buf<uint32_t>(P, t.pos_cap);
    // Attribute classes (action_gpu.cu:1518-1525), with uv and tangents only
    // under preserve_uv (without it the indices were welded to these classes
    // at creation); then each class's source faces in ascending order for
    // place_vertices.
    const std::vector<uint32_t> cls = attribute_roots(S.source_h, S.options.preserve_uv != 0);
    t.canonical = Buf<uint32_t>(P, n);
    B200_CUDA(cudaMemcpyAsync(t.canonical.p, cls.data(), size_t(n) * 4, cudaMemcpyHostToDevice, S.stream));
    const uint32_t* canonical = t.canonical.p;
    if (m.uv) {
        std::vector<uint32_t> offsets(size_t(n) + 1, 0), faces;
        const std::vector<uint32_t>& idx = S.source_h.idx;
        auto corners = [&](uint32_t f, uint32_t* c) {
            for (int j = 0; j < 3; ++j) c[j] = cls[idx[3 * f + j]];
            if (c[1] == c[0]) c[1] = kNone;
            if (c[2] == c[0] || c[2] == c[1]) c[2] = kNone;
        };
        for (uint32_t f = 0; f < nf; ++f) {
            uint32_t c[3];
            corners(f, c);
            for (uint32_t k : c)
                if (k != kNone) ++offsets[k + 1];
        }
        for (uint32_t v = 0; v < n; ++v) offsets[v + 1] += offsets[v];
        faces.resize(offsets[n]);
        std::vector<uint32_t> fill(offsets.begin(), offsets.end() - 1);
        for (uint32_t f = 0; f < nf; ++f) {
            uint32_t c[3];
            corners(f, c);
            for (uint32_t k : c)
                if (k != kNone) faces[fill[k]++] = f;
        }
        t.uv_offsets = Buf<uint32_t>(P, offsets.size());
        t.uv_faces = Buf<uint32_t>(P, std::max<size_t>(1, faces.size()));
        B200_CUDA(cudaMemcpyAsync(t.uv_offsets.p, offsets.data(), offsets.size() * 4, cudaMemcpyHostToDevice,
                                  S.stream));
        if (!faces.empty())
            B200_CUDA(cudaMemcpyAsync(t.uv_faces.p, faces.data(), faces.size() * 4, cudaMemcpyHostToDevice,
                                      S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
        const DevMesh& src = S.source.view;
        t.uvs = UvSource{src.pos, src.uv, src.idx, t.uv_offsets.p, t.uv_faces.p, S.options.preserve_uv != 0};
    }
    t.view = DevTopology{t.geometry.p, canonical, t.face_offsets.p, t.faces.p, t.nbr_offsets.p, t.neighbors.p,
                         t.nbr_count.p, t.boundary.p, t.invalid.p, t.slot_offsets.p, t.slots.p};
}

// Class CSR, fans, legal actions, flat faces and live positions of the state
// (action_gpu.cu:1607-1622 rebuild(), on the classes welded at creation).
static void rebuild_topology(Session& S) {
    Topology& t = S.topo;
    const DevMesh& m = S.state.view;
    const uint32_t n = m.nv;
    cudaStream_t st = S.stream;
    launch_topology(m, t.geometry.p, t.face_offsets.p, t.faces.p, t.cursor.p, nullptr, t.entries.p, t.nbr_offsets.p,
                    t.neighbors.p, t.nbr_count.p, t.boundary.p, t.invalid.p, t.slot_offsets.p,
                    t.slots.p, t.scan.p, nullptr, st);
    B200_CUDA(cudaMemcpyAsync(&t.total_nbrs, t.nbr_offsets.p + n, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    launch_enumerate(m, t.view, t.edge_base.p, t.valid.p, t.edit_slots.p, t.offsets.p, t.edits.p, t.scan.p,
                     t.total_nbrs, false, st);
    B200_CUDA(cudaMemcpyAsync(&t.actions, t.offsets.p + t.total_nbrs, 4, cudaMemcpyDeviceToHost, st));
    launch_flat_faces(m, t.flat.p, st);
    launch_position_table(m, t.view, t.positions.p, t.pos_cap, st);
    B200_CUDA(cudaStreamSynchronize(st));
    B200_CUDA(cudaGetLastError());
}

static uint32_t mask_words(uint32_t size) {
    uint64_t samples = uint64_t(size) * size;
    return uint32_t(((samples + 63) / 64) * 2 + 2); // u64 layout plus one padding word pair
}

// Rasterizes a device mesh for one view; state_dev receives {first box clip,
// any clip, clipped faces, count overflow}.
static void raster(Session& S, const DevMesh& m, const Camera* cam_host, uint32_t ss, uint32_t size, bool force_two,
                   bool cpu_semantics, uint32_t* bits, uint8_t* counts, uint32_t* state_dev) {
    launch_raster(m, cam_host, S.bounds.center, ss, size, force_two, cpu_semantics, bits, counts, state_dev, S.stream);
}

static void ensure_scratch(Session& S, uint32_t size);

static size_t count_stride(size_t samples) { return (samples + 3) & ~size_t(3); }

static uint32_t field_chunk(Session& S, const Plan& p);
// 32-bit counters for a saturated refresh of all views of `p` when they fit
// a sixteenth of the workspace (at least 256 MiB) and half of what is free,
// else null (compare-and-swap counts).
static uint32_t* wide_counts(Session& S, const Plan& p) {
    Scratch& x = S.scratch;
    const size_t need = size_t(p.size) * p.size * p.views;
    if (x.wide.n >= need) return x.wide.p;
    const size_t room = S.pool.limit - S.pool.used + x.wide.n * 4;
    if (need * 4 > std::max(size_t(256) << 20, S.pool.limit / 16) || need * 4 > room / 2) return nullptr;
    x.wide.release();
    x.wide = Buf<uint32_t>(S.pool, need);
    return x.wide.p;
}
// The reference's exact distance field and the tile-maxima arrays of a plan,
// built the first time its state differs from the reference.
static void ensure_tile_data(Session& S, Plan& p) {
    if (p.ref_field.p) return;
    const size_t samples = size_t(p.size) * p.size;
    const uint32_t tiles = ((p.size + 31) / 32) * ((p.size + 31) / 32);
    cudaStream_t st = S.stream;
    ensure_scratch(S, p.size);
    p.ref_field = Buf<uint32_t>(S.pool, samples * p.views);
    p.t1 = Buf<int32_t>(S.pool, size_t(tiles) * p.views);
    p.t2 = Buf<int32_t>(S.pool, size_t(tiles) * p.views);
    B200_CUDA(cudaMemsetAsync(p.t1.p, 0xff, size_t(tiles) * p.views * 4, st));
    B200_CUDA(cudaMemsetAsync(p.t2.p, 0xff, size_t(tiles) * p.views * 4, st));
    // many views per launch (the field chunk's scratch)
    const uint32_t chunk = field_chunk(S, p);
    Scratch& x = S.scratch;
    for (uint32_t v0 = 0; v0 < p.views; v0 += chunk)
        launch_fields_views(p.ref_bits.p + size_t(p.words) * v0, p.words, std::min(chunk, p.views - v0), p.size,
                            x.vg.p, p.ref_field.p + samples * v0, x.vsv.p, x.vsn.p, x.vsd.p, st);
}

// Views per reference-field launch whose scratch (row distances and
// envelope stacks: 24 bytes a sample) fits the budget below; sizes the
// scratch for it.
static uint32_t field_chunk(Session& S, const Plan& p) {
    const size_t samples = size_t(p.size) * p.size;
    Scratch& x = S.scratch;
    // An eighth of the workspace (at least 256 MiB), at most half of what is
    // free (counting the scratch held now): at 4160 x 4160 samples a view
    // needs 415 MB, and one view per launch leaves most SMs idle.
    const size_t floor_bytes = size_t(256) << 20;
    const size_t room = S.pool.limit - S.pool.used + x.view_entries * 24;
    const size_t budget = std::max(floor_bytes, std::min(S.pool.limit / 8, room / 2));
    const uint32_t chunk = uint32_t(std::max<size_t>(1, std::min<size_t>(p.views, budget / (samples * 24))));
    const size_t entries = samples * chunk;
    if (x.view_entries < entries) {
        x.vg.release(), x.vsv.release(), x.vsn.release(), x.vsd.release();
        x.view_entries = 0;
        x.vg = Buf<uint32_t>(S.pool, entries);
        x.vsv = Buf<int32_t>(S.pool, entries);
        x.vsn = Buf<long long>(S.pool, entries);
        x.vsd = Buf<long long>(S.pool, entries);
        x.view_entries = entries;
    }
    return chunk;
}

// Brings the plan's state data (counts, coverage, tile maxima, popcounts)
// up to the session's current state.
static void refresh_state(Session& S, Plan& p) {
    const PlanKey& key = p.key;
    const size_t samples = size_t(p.size) * p.size, cstride = count_stride(samples);
    const bool ref_is_source = key.reference == 0 || S.previous_is_source;
    p.state_is_ref = S.state_is_source && ref_is_source && !p.ref_box_clip;
    cudaStream_t st = S.stream;
    DevMesh live = S.state.view;
    live.nf = S.state_faces;
    const bool own_bits = p.tiled || !p.state_is_ref;
    if (own_bits && !p.state_bits.p) {
        // The padding words past the last sample stay zero for good.
        p.state_bits = Buf<uint32_t>(S.pool, size_t(p.words) * p.views);
        B200_CUDA(cudaMemsetAsync(p.state_bits.p, 0, size_t(p.words) * p.views * 4, st));
    }
    if (!p.raster_state.p) {
        p.raster_state = Buf<uint32_t>(S.pool, 4 * size_t(p.views));
        p.pop = Buf<unsigned long long>(S.pool, 4 * size_t(p.views));
        p.hstate.assign(4 * size_t(p.views), 0);
        p.hpop.assign(4 * size_t(p.views), 0);
    }
    const uint32_t* sbits = own_bits ? p.state_bits.p : p.ref_bits.p;
    const bool fields = p.tiled && !p.state_is_ref;
    const uint32_t tiles = ((p.size + 31) / 32) * ((p.size + 31) / 32);
    if (fields) ensure_tile_data(S, p);
    // Tile maxima by searches from the reference-only samples: no state
    // field, all views in one launch.
    const uint32_t chunk = p.views;
    std::vector<unsigned long long>& hpop = p.hpop;
    std::vector<uint32_t>& hstate = p.hstate;
    // Counts of up to 255 faces per sample; a plan with more is rebuilt with
    // counts held at 255 (exact for the audits).
    for (int pass = p.deep ? 1 : 0; pass < 2; ++pass) {
        const bool saturate = pass == 1;
        uint32_t* const wide = saturate ? wide_counts(S, p) : nullptr;
        for (uint32_t v0 = 0; v0 < p.views; v0 += chunk) {
            const uint32_t n = std::min(chunk, p.views - v0);
            const size_t w0 = size_t(p.words) * v0, s0 = samples * v0, t0 = size_t(tiles) * v0;
            launch_refresh_views(live, p.cameras.p + v0, n, S.bounds.center, key.ss, p.size, key.force_two,
                                 p.state_count.p + cstride * v0, cstride, p.raster_state.p + 4 * v0,
                                 own_bits ? p.state_bits.p + w0 : nullptr, p.ref_bits.p + w0, p.words,
                                 p.pop.p + 4 * v0, fields ? p.ref_field.p + s0 : nullptr, nullptr, nullptr,
                                 nullptr, nullptr, nullptr, fields ? p.t1.p + t0 : nullptr,
                                 fields ? p.t2.p + t0 : nullptr, saturate, st, wide);
        }
        B200_CUDA(cudaMemcpyAsync(hpop.data(), p.pop.p, hpop.size() * 8, cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaMemcpyAsync(hstate.data(), p.raster_state.p, hstate.size() * 4, cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaStreamSynchronize(st));
        B200_CUDA(cudaGetLastError());
        bool overflow = false;
        for (uint32_t v = 0; v < p.views; ++v) overflow |= hstate[4 * v + 3] != 0;
        if (!overflow) break;
        p.deep = true;
    }
    for (uint32_t v = 0; v < p.views; ++v) {
        PlanView& pv = p.hviews[v];
        pv.state_bits = sbits + size_t(v) * p.words;
        pv.state_count = p.state_count.p + cstride * v;
        pv.tile_t1 = p.t1.p ? p.t1.p + tiles * v : nullptr;
        pv.tile_t2 = p.t2.p ? p.t2.p + tiles * v : nullptr;
        pv.ref_field = p.ref_field.p ? p.ref_field.p + samples * v : nullptr;
        pv.changed = uint32_t(hpop[4 * v]);
        pv.total = uint32_t(hpop[4 * v + 1]);
        pv.cov_ref = uint32_t(hpop[4 * v + 2]);
        pv.cov_state = uint32_t(hpop[4 * v + 3]);
        pv.clip_state = hstate[4 * v + 2];
    }
    B200_CUDA(cudaMemcpyAsync(p.dviews.p, p.hviews.data(), p.views * sizeof(PlanView), cudaMemcpyHostToDevice, st));
    p.dev.state_is_ref = p.state_is_ref;
    p.state_revision = S.state_revision;
    B200_CUDA(cudaStreamSynchronize(st));
}

static Plan& plan_for(Session& S, const PlanKey& key) {
    auto it = S.plans.find(key);
    if (it != S.plans.end()) {
        Plan& p = *it->second;
        if (!p.resource_limited && p.state_revision != S.state_revision) refresh_state(S, p);
        return p;
    }
    auto plan = std::make_unique<Plan>();
    Plan& p = *plan;
    p.key = key;
    p.size = raster_size(key.screen, key.ss);
    p.views = uint32_t(key.ortho) + key.persp;
    if (uint64_t(p.size) * p.size > kMaxSamples) {
        p.resource_limited = true;
        return *(S.plans[key] = std::move(plan));
    }
    p.words = mask_words(p.size);
    p.tiled = p.size <= 4160;
    p.hcams = make_cameras(S.bounds, key.screen, key.ortho, key.persp, key.seed);
    p.cameras = Buf<Camera>(S.pool, p.hcams.size());
    cudaStream_t st = S.stream;
    B200_CUDA(cudaMemcpyAsync(p.cameras.p, p.hcams.data(), p.hcams.size() * sizeof(Camera), cudaMemcpyHostToDevice, st));
    const DeviceMesh& ref = key.reference == 0 || S.previous_is_source ? S.source : S.previous;
    const size_t samples = size_t(p.size) * p.size;
    p.ref_bits = Buf<uint32_t>(S.pool, size_t(p.words) * p.views);
    p.state_count = Buf<uint8_t>(S.pool, count_stride(samples) * p.views);
    B200_CUDA(cudaMemsetAsync(p.ref_bits.p, 0, size_t(p.words) * p.views * 4, st));
    Buf<uint32_t> state(S.pool, 4 * size_t(p.views));
    for (uint32_t v = 0; v < p.views; ++v)
        raster(S, ref.view, &p.hcams[v], key.ss, p.size, key.force_two, true, p.ref_bits.p + size_t(v) * p.words,
               nullptr, state.p + 4 * v);
    std::vector<uint32_t> hstate(4 * size_t(p.views));
    B200_CUDA(cudaMemcpyAsync(hstate.data(), state.p, hstate.size() * 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    p.hviews.assign(p.views, PlanView{});
    for (uint32_t v = 0; v < p.views; ++v) {
        p.ref_box_clip |= hstate[4 * v] != kNone;
        p.hviews[v].ref_bits = p.ref_bits.p + size_t(v) * p.words;
        p.hviews[v].clipped_ref = hstate[4 * v + 1];
    }
    p.dviews = Buf<PlanView>(S.pool, p.views);
    p.dev.cameras = p.cameras.p;
    p.dev.views = p.dviews.p;
    for (int k = 0; k < 3; ++k) p.dev.center[k] = S.bounds.center[k];
    p.dev.nviews = p.views, p.dev.ss = key.ss, p.dev.size = p.size, p.dev.force_two = key.force_two;
    p.dev.d2_floor = 0, p.dev.d2_ceiling = 0xffffffffu;
    refresh_state(S, p);
    return *(S.plans[key] = std::move(plan));
}

static uint32_t mask_words_for(size_t samples) { return uint32_t(((samples + 63) / 64) * 2 + 2); }

// Full-path scratch for rasters of up to `samples` samples (any width x height).
static void ensure_scratch_samples(Session& S, size_t samples) {
    Scratch& x = S.scratch;
    if (x.samples >= samples && x.a.p) return;
    uint32_t words = mask_words_for(samples);
    x.a = Buf<uint32_t>(S.pool, words);
    x.c = Buf<uint32_t>(S.pool, words);
    x.g = Buf<uint32_t>(S.pool, samples);
    x.d2 = Buf<uint32_t>(S.pool, samples);
    x.sv = Buf<int32_t>(S.pool, samples);
    x.sn = Buf<long long>(S.pool, samples);
    x.sd = Buf<long long>(S.pool, samples);
    x.maxes = Buf<uint32_t>(S.pool, 2);
    x.state = Buf<uint32_t>(S.pool, 8);
    x.pop = Buf<unsigned long long>(S.pool, 4);
    x.samples = samples;
}
static void ensure_scratch(Session& S, uint32_t size) { ensure_scratch_samples(S, size_t(size) * size); }

// Coverage distance of two device masks already in scratch a/c (evaluate.cpp:196-209):
// fills rec (changed, total, ca, cb) and the max squared distance.
static void mask_distance(Session& S, uint32_t width, uint32_t height, ViewRecord& rec, double& max_d2) {
    Scratch& x = S.scratch;
    cudaStream_t st = S.stream;
    uint32_t words = mask_words_for(size_t(width) * height);
    launch_popcounts(x.a.p, x.c.p, words, x.pop.p, st);
    unsigned long long pop[4];
    B200_CUDA(cudaMemcpyAsync(pop, x.pop.p, sizeof(pop), cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    rec.changed = uint32_t(pop[0]);
    rec.total = uint32_t(pop[1]);
    rec.ca = pop[2] > 0;
    rec.cb = pop[3] > 0;
    max_d2 = 0;
    if (rec.changed && rec.ca && rec.cb) {
        B200_CUDA(cudaMemsetAsync(x.maxes.p, 0, 8, st));
        launch_distance(x.a.p, x.c.p, width, height, x.g.p, x.d2.p, x.sv.p, x.sn.p, x.sd.p, x.maxes.p, st);
        launch_distance(x.c.p, x.a.p, width, height, x.g.p, x.d2.p, x.sv.p, x.sn.p, x.sd.p, x.maxes.p + 1, st);
        uint32_t m[2];
        B200_CUDA(cudaMemcpyAsync(m, x.maxes.p, 8, cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaStreamSynchronize(st));
        float fa, fc;
        std::memcpy(&fa, &m[0], 4);
        std::memcpy(&fc, &m[1], 4);
        max_d2 = std::max(double(fa), double(fc));
    }
}

// One view at one sampling through the full-raster path.
static void full_view(Session& S, const DevMesh& ref, const DevMesh& cand, const Camera* cam_host, uint32_t ss,
                      uint32_t size, bool force_two, ViewRecord& rec, double& max_d2) {
    ensure_scratch(S, size);
    Scratch& x = S.scratch;
    uint32_t words = mask_words(size);
    cudaStream_t st = S.stream;
    B200_CUDA(cudaMemsetAsync(x.a.p, 0, size_t(words) * 4, st));
    B200_CUDA(cudaMemsetAsync(x.c.p, 0, size_t(words) * 4, st));
    raster(S, ref, cam_host, ss, size, force_two, true, x.a.p, nullptr, x.state.p);
    raster(S, cand, cam_host, ss, size, force_two, true, x.c.p, nullptr, x.state.p + 4);
    uint32_t state[8];
    B200_CUDA(cudaMemcpyAsync(state, x.state.p, sizeof(state), cudaMemcpyDeviceToHost, st));
    rec = ViewRecord{};
    mask_distance(S, size, size, rec, max_d2);
    rec.flags = (state[1] ? kRecClippedRef : 0) | (state[5] ? kRecClippedCand : 0);
}

// evaluate_impl (evaluate.cpp:312-352) over the full-raster path. `recs`
// (host, one per view, or null) are the incremental path's records of this
// candidate at the gate's first sampling: a record without flags equals the
// full raster's and is used as is, so only flagged views (fallback, clipped,
// distance beyond 2^24) and refinements are rasterized in full.
static Measurement evaluate_full(Session& S, const DevMesh& ref, const DevMesh& cand, const blitz_eval_settings* es,
                                 const GateSettings& g, const ViewRecord* recs = nullptr) {
    Measurement result = default_measurement();
    result.supersample = g.supersample;
    auto cams = make_cameras(S.bounds, g.screen_size, es->views_orthographic, es->views_perspective, es->views_seed);
    for (uint32_t v = 0; v < cams.size(); ++v) {
        Measurement cur = default_measurement();
        cur.worst_view = v;
        for (uint32_t ss = g.supersample;; ss = std::min<uint32_t>(g.max_supersample, ss * 2)) {
            if (recs && ss == g.supersample && recs[v].flags == 0) {
                finish_view(cur, recs[v], g, ss, double(recs[v].max_d2));
                if (refinement_done(cur, g, ss)) break;
                continue;
            }
            uint32_t size = raster_size(g.screen_size, ss);
            if (uint64_t(size) * size > kMaxSamples) {
                result.complete = 0;
                result.passed = 0;
                result.resource_limited = 1;
                result.error = INFINITY;
                return result;
            }
            ViewRecord rec;
            double max_d2;
            full_view(S, ref, cand, &cams[v], ss, size, es->force_two_sided, rec, max_d2);
            finish_view(cur, rec, g, ss, max_d2);
            if (refinement_done(cur, g, ss)) break;
        }
        if (!aggregate_view(result, cur, v)) return result;
    }
    return result;
}

struct GateRef {
    const blitz_eval_settings* es;
    GateSettings g;
    int reference;
};

// Candidate whose verdict needs the full-raster path from gate `first`.
// Full-trial buffers at the source's capacity (the state only loses faces).
static void ensure_trial_buffers(Session& S) {
    if (S.trial.pos.p) return;
    const DevMesh& src = S.source.view;
    S.trial.pos = Buf<float>(S.pool, 3ull * src.nv);
    S.trial.idx = Buf<uint32_t>(S.pool, 3ull * src.nf);
    if (src.mat) S.trial.mat = Buf<uint16_t>(S.pool, src.nf);
    if (src.uv) S.trial.uv = Buf<float>(S.pool, 2ull * src.nv);
    S.trial_keep = Buf<uint32_t>(S.pool, src.nf + 1);
    S.trial_offsets = Buf<uint32_t>(S.pool, src.nf + 1);
    S.trial_info = Buf<TrialInfo>(S.pool, 1);
    S.trial_collapse = Buf<blitz_collapse>(S.pool, 1);
}

static void trial_views(Session& S, Plan& p, const DevMesh& cand, uint64_t tag, const TrialDelta* delta = nullptr);
static bool gate_from_trial(const Plan& p, const GateSettings& g, Measurement& result);

// Global-memory scratch of the huge audit tier, one per device and shared by
// all sessions on it (allocated on first need, kept until exit). Launches that
// use it are ordered on the device by an event: a session's stream waits for
// the previous user before its huge-tier launch and records the event after.
struct HugeScratch {
    std::mutex lock;
    unsigned char* p = nullptr;
    uint32_t blocks = 0;
    unsigned char* giant = nullptr; // giant tier, for rasters above 1024 x 1024
    cudaEvent_t done = nullptr;
};
constexpr uint32_t kGiantBlocks = 8;
static HugeScratch& huge_scratch(int device) {
    static HugeScratch per_device[64];
    if (device < 0 || device >= 64) throw Failure(BLITZ_INVALID_ARGUMENT, "device index out of range");
    return per_device[device];
}

// Plans of rasters above 256 x 256 can hold regions beyond the large tier.
static void run_audit(Session& S, Plan& p, uint32_t n, unsigned long long* stats, cudaStream_t st) {
    S.work_queue.ensure(S.pool, 8);
    S.spill.ensure(S.pool, size_t(n) * p.views + 1);
    AuditJob job{};
    job.plan = p.dev, job.recs = S.records.p, job.out = p.records.p, job.total = uint64_t(n) * p.views;
    if (p.size <= 256) {
        launch_audit(job, stats, S.work_queue.p, S.spill.p, nullptr, nullptr, 0, st);
        return;
    }
    S.spill_huge.ensure(S.pool, size_t(n) * p.views + 1);
    HugeScratch& h = huge_scratch(S.device);
    std::lock_guard<std::mutex> guard(h.lock);
    if (!h.p) {
        int sms = 148;
        B200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S.device));
        const uint32_t blocks = uint32_t(std::max(1, sms / 2));
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, audit_huge_scratch_bytes(blocks));
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Failure(BLITZ_OUT_OF_MEMORY, "huge-tier audit scratch");
        }
        B200_CUDA(cudaEventCreateWithFlags(&h.done, cudaEventDisableTiming));
        h.p = static_cast<unsigned char*>(q);
        h.blocks = blocks;
    } else {
        B200_CUDA(cudaStreamWaitEvent(st, h.done, 0));
    }
    GiantTier giant{};
    if (p.size > 1024) {
        if (!h.giant) {
            void* q = nullptr;
            cudaError_t e = cudaMalloc(&q, audit_giant_scratch_bytes(kGiantBlocks));
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw Failure(BLITZ_OUT_OF_MEMORY, "giant-tier audit scratch");
            }
            h.giant = static_cast<unsigned char*>(q);
        }
        S.spill_giant.ensure(S.pool, size_t(n) * p.views + 1);
        giant = GiantTier{S.spill_giant.p, h.giant, kGiantBlocks};
    }
    launch_audit(job, stats, S.work_queue.p, S.spill.p, S.spill_huge.p, h.p, h.blocks, st, kAuditTierSmall,
                 giant.scratch ? &giant : nullptr);
    B200_CUDA(cudaEventRecord(h.done, st));
}

// Plan of gate `gi` (gates 1 and 3 against the source, 2 and 4 against the
// bound previous LOD).
static PlanKey plan_key_of(const Session& S, int gi, const blitz_eval_settings& es) {
    return PlanKey{(gi % 2) && !S.previous_is_source ? 1 : 0, es.views_orthographic, es.views_perspective,
                   es.views_seed, es.screen_size, es.supersample, es.force_two_sided};
}

// One gate of a built trial: all views at once from the plan's reference
// fields when the plan keeps them and no view clips or refines, else the
// per-view full-raster path.
static Measurement gate_of_trial(Session& S, const DevMesh& cand, const GateRef& gate, int gi, uint64_t tag,
                                 const ViewRecord* recs_dev = nullptr, const TrialDelta* delta = nullptr) {
    Plan& p = plan_for(S, plan_key_of(S, gi, *gate.es));
    Measurement r;
    if (!p.resource_limited && p.tiled) {
        if (p.trial_tag != tag) trial_views(S, p, cand, tag, delta);
        if (gate_from_trial(p, gate.g, r)) return r;
    }
    std::vector<ViewRecord> recs;
    if (recs_dev && !p.resource_limited) {
        recs.resize(p.views);
        B200_CUDA(cudaMemcpyAsync(recs.data(), recs_dev, p.views * sizeof(ViewRecord), cudaMemcpyDeviceToHost,
                                  S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
    }
    const DevMesh& ref = gate.reference == 0 || S.previous_is_source ? S.source.view : S.previous.view;
    return evaluate_full(S, ref, cand, gate.es, gate.g, recs.empty() ? nullptr : recs.data());
}

static void exact_candidate(Session& S, const blitz_collapse& col, const GateRef* gates, int first,
                            blitz_candidate_verdict& v, Measurement* meas,
                            const ViewRecord* const* gate_records = nullptr) {
    const DevMesh& m = S.state.view;
    Topology& t = S.topo;
    ensure_trial_buffers(S);
    B200_CUDA(cudaMemcpyAsync(S.trial_collapse.p, &col, sizeof(col), cudaMemcpyHostToDevice, S.stream));
    launch_trial(m, t.view, S.trial_collapse.p, S.trial_info.p, S.trial_keep.p, S.trial_offsets.p, S.trial.idx.p, S.trial.mat.p,
                 S.trial.pos.p, t.scan.p, S.stream, t.uv(), S.trial.uv.p);
    uint32_t faces = 0;
    B200_CUDA(cudaMemcpyAsync(&faces, S.trial_offsets.p + m.nf, 4, cudaMemcpyDeviceToHost, S.stream));
    B200_CUDA(cudaStreamSynchronize(S.stream));
    DevMesh cand = m;
    cand.pos = S.trial.pos.p;
    cand.idx = S.trial.idx.p;
    cand.mat = m.mat ? S.trial.mat.p : nullptr;
    cand.nf = faces;
    v.exact_path = 1;
    v.failed_gate = 0;
    v.accepted = 0;
    const uint64_t tag = ++S.trial_tag;
    for (int gi = first; gi < 4; ++gi) {
        Measurement r = gate_of_trial(S, cand, gates[gi], gi, tag, gate_records ? gate_records[gi] : nullptr);
        if (meas) meas[gi] = r;
        if (!measurement_accepted(r)) {
            v.failed_gate = uint8_t(gi + 1);
            return;
        }
    }
    v.accepted = 1;
}

// Gates, distinct plans and the gate -> plan map of one audit call.
struct AuditSetup {
    GateRef gates[4];
    std::vector<PlanKey> keys;
    uint32_t plan_of[4];
    std::vector<Plan*> plans;
};
// The largest squared distance at which a view still passes gate g on
// coverage (finish_view's error <= limit, evaluate.cpp:271-298), or -1 when
// no distance does: the error is non-decreasing in the distance, so a binary
// search over the integers with the same FP64 expressions finds it.
static int64_t pass_threshold(const GateSettings& g, uint32_t ss) {
    auto passes = [&](uint64_t d2) {
        ViewRecord r{};
        r.changed = r.total = 1;
        r.ca = r.cb = 1;
        Measurement cur = default_measurement();
        finish_view(cur, r, g, ss, double(d2));
        return cur.error <= g.limit;
    };
    if (!passes(0)) return -1;
    uint64_t lo = 0, hi = 0xffffffffull;
    if (passes(hi)) return int64_t(hi);
    while (lo + 1 < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (passes(mid)) lo = mid;
        else hi = mid;
    }
    return int64_t(lo);
}

// verdict_only: the caller takes verdicts only (no Measurements), so each
// plan's audit may stop measuring a view once its verdicts are certain
// (PlanDev d2_floor / d2_ceiling); else the audit measures exactly.
static void setup_audit(Session& S, const blitz_eval_settings gates_in[4], AuditSetup& a,
                        bool verdict_only = false) {
    a.keys.clear();
    a.plans.clear();
    for (int g = 0; g < 4; ++g) {
        a.gates[g].es = &gates_in[g];
        a.gates[g].g = gate_of(&gates_in[g], S.bounds);
        a.gates[g].g.max_supersample = uint8_t(
            bounded_refinement(a.gates[g].g.screen_size, a.gates[g].g.supersample, a.gates[g].g.max_supersample));
        a.gates[g].reference = g % 2;
        const PlanKey k = plan_key_of(S, g, gates_in[g]);
        auto it = std::find_if(a.keys.begin(), a.keys.end(), [&](const PlanKey& o) { return !(o < k) && !(k < o); });
        a.plan_of[g] = uint32_t(it - a.keys.begin());
        if (it == a.keys.end()) a.keys.push_back(k);
    }
    for (auto& k : a.keys) {
        Plan& p = plan_for(S, k);
        if (p.resource_limited) throw Failure(BLITZ_BUDGET_LIMITED, "raster exceeds per-view sample budget");
        a.plans.push_back(&p);
    }
    for (size_t i = 0; i < a.plans.size(); ++i) {
        Plan& p = *a.plans[i];
        p.dev.d2_floor = 0, p.dev.d2_ceiling = 0xffffffffu;
        if (!verdict_only) continue;
        int64_t lo = INT64_MAX, hi = -1;
        for (int g = 0; g < 4; ++g) {
            if (a.plan_of[g] != i) continue;
            const int64_t t = pass_threshold(a.gates[g].g, p.key.ss);
            lo = std::min(lo, t), hi = std::max(hi, t);
        }
        p.dev.d2_floor = uint32_t(std::max<int64_t>(lo, 0));
        p.dev.d2_ceiling = uint32_t(std::max<int64_t>(hi, 0));
    }
}
// Per-plan record tables of k_verdicts for n candidates (records sized here).
// Returns whether anything was uploaded: tables equal to the last upload's
// (same plans, record buffers, gates) are not sent again.
static bool upload_verdict_tables(Session& S, const AuditSetup& a, uint32_t n, cudaStream_t st) {
    std::vector<const ViewRecord*> table(a.plans.size());
    std::vector<uint32_t> pviews(a.plans.size()), pss(a.plans.size());
    for (size_t i = 0; i < a.plans.size(); ++i) {
        Plan& p = *a.plans[i];
        p.records.ensure(S.pool, std::max<size_t>(1, size_t(n) * p.views));
        table[i] = p.records.p;
        pviews[i] = p.views;
        pss[i] = p.key.ss;
    }
    S.record_table.ensure(S.pool, 4);
    S.plan_views.ensure(S.pool, 4);
    S.plan_ss.ensure(S.pool, 4);
    S.gate_table.ensure(S.pool, 4);
    S.exact_count.ensure(S.pool, 1);
    GateDev gd[4];
    std::memset(gd, 0, sizeof gd);
    for (int g = 0; g < 4; ++g) gd[g] = GateDev{a.gates[g].g, a.plan_of[g]};
    std::vector<uint8_t> sig;
    auto put = [&](const void* q, size_t k) {
        const uint8_t* c = static_cast<const uint8_t*>(q);
        sig.insert(sig.end(), c, c + k);
    };
    put(table.data(), table.size() * sizeof(void*)), put(pviews.data(), pviews.size() * 4);
    put(pss.data(), pss.size() * 4), put(gd, sizeof gd), put(&S.record_table.p, sizeof(void*));
    if (sig == S.table_signature) return false;
    B200_CUDA(cudaMemcpyAsync(S.record_table.p, table.data(), table.size() * sizeof(void*), cudaMemcpyHostToDevice, st));
    B200_CUDA(cudaMemcpyAsync(S.plan_views.p, pviews.data(), pviews.size() * 4, cudaMemcpyHostToDevice, st));
    B200_CUDA(cudaMemcpyAsync(S.plan_ss.p, pss.data(), pss.size() * 4, cudaMemcpyHostToDevice, st));
    B200_CUDA(cudaMemcpyAsync(S.gate_table.p, gd, sizeof(gd), cudaMemcpyHostToDevice, st));
    S.table_signature = std::move(sig);
    return true;
}
// Candidates whose verdict needs the full-raster path (k_verdicts flagged
// them): resolved one by one from their resume gate.
static void resolve_exact(Session& S, AuditSetup& a, const blitz_collapse* cands_dev, uint32_t nn,
                          blitz_candidate_verdict* out_dev, Measurement* meas_dev, cudaStream_t st) {
    std::vector<blitz_candidate_verdict> hv(nn);
    B200_CUDA(cudaMemcpyAsync(hv.data(), out_dev, nn * sizeof(blitz_candidate_verdict), cudaMemcpyDeviceToHost, st));
    std::vector<blitz_collapse> hc(nn);
    B200_CUDA(cudaMemcpyAsync(hc.data(), cands_dev, nn * sizeof(blitz_collapse), cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    cudaStream_t saved = S.stream;
    S.stream = st;
    for (uint32_t c = 0; c < nn; ++c) {
        if (!hv[c].exact_path) continue;
        int first = hv[c].reserved; // resume gate
        Measurement m4[4];
        if (meas_dev) {
            B200_CUDA(cudaMemcpyAsync(m4, meas_dev + size_t(c) * 4, sizeof(m4), cudaMemcpyDeviceToHost, st));
            B200_CUDA(cudaStreamSynchronize(st));
        }
        const ViewRecord* recs[4];
        for (int g = 0; g < 4; ++g) {
            const Plan& p = *a.plans[a.plan_of[g]];
            recs[g] = p.records.p + size_t(c) * p.views;
        }
        exact_candidate(S, hc[c], a.gates, first, hv[c], meas_dev ? m4 : nullptr, recs);
        hv[c].reserved = 0;
        B200_CUDA(cudaMemcpyAsync(out_dev + c, &hv[c], sizeof(hv[c]), cudaMemcpyHostToDevice, st));
        if (meas_dev) B200_CUDA(cudaMemcpyAsync(meas_dev + size_t(c) * 4, m4, sizeof(m4), cudaMemcpyHostToDevice, st));
        B200_CUDA(cudaStreamSynchronize(st));
    }
    S.stream = saved;
}

static void audit_candidates(Session& S, const blitz_collapse* cands_dev, const blitz_collapse* cands_host, size_t n,
                             const blitz_eval_settings gates_in[4], blitz_candidate_verdict* out_dev,
                             Measurement* meas_dev, cudaStream_t st) {
    if (n > UINT32_MAX / 2) throw Failure(BLITZ_INVALID_ARGUMENT, "too many candidates");
    (void)cands_host;
    AuditSetup a;
    setup_audit(S, gates_in, a, meas_dev == nullptr);
    const uint32_t nn = uint32_t(n);
    Topology& t = S.topo;
    S.records.ensure(S.pool, nn);
    const bool prof = S.profiling && nn, counted = prof && S.counting;
    if (prof) {
        S.stats.ensure(S.pool, kAuditStats);
        B200_CUDA(cudaMemsetAsync(S.stats.p, 0, kAuditStats * 8, st));
        B200_CUDA(cudaEventRecord(S.ev[0], st));
    }
    launch_prepare(S.state.view, t.view, S.state.view, t.view, cands_dev, nn, t.positions.p, t.pos_cap, t.flat.p,
                   S.options.preserve_uv != 0, S.records.p, st, t.uv());
    if (prof) B200_CUDA(cudaEventRecord(S.ev[1], st));
    S.profile.launches += nn ? 1 : 0;
    upload_verdict_tables(S, a, nn, st);
    for (Plan* pp : a.plans) {
        run_audit(S, *pp, nn, counted ? S.stats.p : nullptr, st);
        if (nn) S.profile.launches += 1, S.profile.audit_launches += 1;
    }
    if (prof) B200_CUDA(cudaEventRecord(S.ev[4], st));
    B200_CUDA(cudaMemsetAsync(S.exact_count.p, 0, 4, st));
    if (prof) B200_CUDA(cudaEventRecord(S.ev[2], st));
    launch_verdicts(S.record_table.p, S.plan_views.p, S.plan_ss.p, S.gate_table.p, S.records.p, nn, out_dev, meas_dev,
                    S.exact_count.p, st);
    if (nn) S.profile.launches += 1;
    if (prof) B200_CUDA(cudaEventRecord(S.ev[3], st));
    uint32_t exact = 0;
    B200_CUDA(cudaMemcpyAsync(&exact, S.exact_count.p, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    B200_CUDA(cudaGetLastError());
    if (prof) {
        float ta = 0, tb = 0, tc = 0;
        B200_CUDA(cudaEventElapsedTime(&ta, S.ev[0], S.ev[1]));
        B200_CUDA(cudaEventElapsedTime(&tb, S.ev[1], S.ev[4]));
        B200_CUDA(cudaEventElapsedTime(&tc, S.ev[2], S.ev[3]));
        unsigned long long h[4];
        B200_CUDA(cudaMemcpy(h, S.stats.p, sizeof(h), cudaMemcpyDeviceToHost));
        S.profile.prepare_ms += ta;
        S.profile.audit_ms += tb;
        S.profile.verdict_ms += tc;
        if (!counted) h[0] = h[1] = h[2] = 0;
        S.profile.units += h[0];
        S.profile.region_samples += h[1];
        S.profile.changed_samples += h[2];
        S.profile.record_bytes += uint64_t(nn) * sizeof(CandidateRecord) * a.plans.size();
    }
    if (exact) resolve_exact(S, a, cands_dev, nn, out_dev, meas_dev, st);
    S.info.decoded += nn;
}

// Applies an accepted collapse to the state: trial build on the GPU
// (remap, keep, compaction, placement; action_gpu.cu:748-790, 962-1067), the
// trial becomes the state (commit, 1729-1750), then the topology is rebuilt on
// the creation-time classes.
static void commit_collapse(Session& S, const blitz_collapse& col) {
    ensure_trial_buffers(S);
    DevMesh& m = S.state.view;
    cudaStream_t st = S.stream;
    B200_CUDA(cudaMemcpyAsync(S.trial_collapse.p, &col, sizeof(col), cudaMemcpyHostToDevice, st));
    launch_trial(m, S.topo.view, S.trial_collapse.p, S.trial_info.p, S.trial_keep.p, S.trial_offsets.p, S.trial.idx.p,
                 S.trial.mat.p, S.trial.pos.p, S.topo.scan.p, st, S.topo.uv(), S.trial.uv.p);
    uint32_t faces = 0;
    B200_CUDA(cudaMemcpyAsync(&faces, S.trial_offsets.p + m.nf, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    if (!faces) throw Failure(BLITZ_INVALID_ARGUMENT, "collapse would remove the entire mesh");
    B200_CUDA(cudaMemcpyAsync(S.state.idx.p, S.trial.idx.p, size_t(faces) * 12, cudaMemcpyDeviceToDevice, st));
    B200_CUDA(cudaMemcpyAsync(S.state.pos.p, S.trial.pos.p, size_t(m.nv) * 12, cudaMemcpyDeviceToDevice, st));
    if (m.mat) B200_CUDA(cudaMemcpyAsync(S.state.mat.p, S.trial.mat.p, size_t(faces) * 2, cudaMemcpyDeviceToDevice, st));
    if (m.uv) B200_CUDA(cudaMemcpyAsync(S.state.uv.p, S.trial.uv.p, size_t(m.nv) * 8, cudaMemcpyDeviceToDevice, st));
    m.nf = faces;
    S.state_faces = faces;
    ++S.state_revision;
    S.state_is_source = false;
    rebuild_topology(S);
}

static void prune_ranked(Session& S, uint32_t actions, uint32_t keep, float px, float px2);

// Ranking scores of the state's legal edits: 1 Constant, 3 ShortestEdge,
// 4 CurrentPlane (rank_actions, action_gpu.cu:809-844), or 0 Learned: the
// attached surrogate's acceptance logits.
static void rank_edits(Session& S, uint32_t actions, double diameter, int ranking, const blitz_eval_settings* gates,
                       float* scores, uint32_t* order, cudaStream_t st) {
    Topology& t = S.topo;
    if (ranking != 0) {
        launch_rank(S.state.view, t.view, t.edits.p, t.offsets.p + t.total_nbrs, actions, diameter, ranking, scores,
                    order, st);
        return;
    }
    if (!S.surrogate) throw Failure(BLITZ_INVALID_ARGUMENT, "learned ranking needs an attached surrogate");
    const float px = float(gates[0].screen_size / std::max(1e-20, 2 * S.bounds.radius));
    const float px2 = float(gates[2].screen_size / std::max(1e-20, 2 * S.bounds.radius));
    const size_t cap = 6ull * S.source.view.nf + 1;
    S.sur_features.ensure(S.pool, cap * kSurrogateIn);
    S.sur_out.ensure(S.pool, 2 * cap);
    launch_features(S.state.view, t.view, t.edits.p, t.offsets.p + t.total_nbrs, actions, px, px2,
                    S.sur_features.p, st);
    B200_CUDA(launch_mlp(S.surrogate->dev(), S.sur_features.p, actions, S.sur_out.p, nullptr, 0.f, nullptr,
                         S.surrogate->error.p, 148, st));
    launch_prune_prepare(S.sur_out.p, actions, scores, order, st);
}

static void reset_state(Session& S) {
    cudaStream_t st = S.stream;
    const DevMesh& src = S.source.view;
    B200_CUDA(cudaMemcpyAsync(S.state.idx.p, src.idx, size_t(src.nf) * 12, cudaMemcpyDeviceToDevice, st));
    B200_CUDA(cudaMemcpyAsync(S.state.pos.p, src.pos, size_t(src.nv) * 12, cudaMemcpyDeviceToDevice, st));
    if (src.mat) B200_CUDA(cudaMemcpyAsync(S.state.mat.p, src.mat, size_t(src.nf) * 2, cudaMemcpyDeviceToDevice, st));
    if (src.uv) B200_CUDA(cudaMemcpyAsync(S.state.uv.p, src.uv, size_t(src.nv) * 8, cudaMemcpyDeviceToDevice, st));
    S.state.view.nf = src.nf;
    S.state_faces = src.nf;
    ++S.state_revision;
    S.state_is_source = true;
    rebuild_topology(S);
}

// ---------------------------------------------------------------------------
// Batched executor.

// Gate settings and plans of the four gates (generate.cpp:365-388): gates 1
// and 3 against the source, 2 and 4 against the bound previous LOD.
static void resolve_gates(Session& S, const blitz_eval_settings gates_in[4], GateRef gates[4], PlanKey keys[4]) {
    for (int g = 0; g < 4; ++g) {
        gates[g].es = &gates_in[g];
        gates[g].g = gate_of(&gates_in[g], S.bounds);
        gates[g].g.max_supersample = uint8_t(
            bounded_refinement(gates[g].g.screen_size, gates[g].g.supersample, gates[g].g.max_supersample));
        gates[g].reference = g % 2;
        keys[g] = PlanKey{(g % 2) && !S.previous_is_source ? 1 : 0, gates_in[g].views_orthographic,
                          gates_in[g].views_perspective, gates_in[g].views_seed, gates_in[g].screen_size,
                          gates_in[g].supersample, gates_in[g].force_two_sided};
    }
}

// Per-view data of a whole candidate mesh against the plan's reference, all
// views in a handful of launches (counts, coverage, tile maxima from the
// reference field and from searches, popcounts, per-view maxima), left in
// the plan's trial buffers.
static void trial_views(Session& S, Plan& p, const DevMesh& cand, uint64_t tag, const TrialDelta* delta) {
    cudaStream_t st = S.stream;
    const size_t samples = size_t(p.size) * p.size, cstride = count_stride(samples);
    const uint32_t tiles = ((p.size + 31) / 32) * ((p.size + 31) / 32);
    auto ensure_trial = [&](Plan& q) {
        if (q.trial_count.p) return;
        q.trial_count = Buf<uint8_t>(S.pool, cstride * q.views);
        q.trial_bits = Buf<uint32_t>(S.pool, size_t(q.words) * q.views);
        B200_CUDA(cudaMemsetAsync(q.trial_bits.p, 0, size_t(q.words) * q.views * 4, st));
        q.trial_state = Buf<uint32_t>(S.pool, 4 * size_t(q.views));
        q.trial_t1 = Buf<int32_t>(S.pool, size_t(tiles) * q.views);
        q.trial_t2 = Buf<int32_t>(S.pool, size_t(tiles) * q.views);
        q.trial_max = Buf<int32_t>(S.pool, 2 * size_t(q.views));
        q.trial_pop = Buf<unsigned long long>(S.pool, 4 * size_t(q.views));
        q.trial_hstate.assign(4 * size_t(q.views), 0);
        q.trial_hpop.assign(4 * size_t(q.views), 0);
        q.trial_hmax.assign(2 * size_t(q.views), 0);
    };
    ensure_trial(p);
    ensure_tile_data(S, p);
    // Plans of the same views (cameras, screen, supersample, sides) against
    // the other reference: the trial's counts and coverage are the same, so
    // they take copies and only their tile maxima and popcounts against their
    // own reference are computed.
    std::vector<Plan*> same_views;
    for (auto& kv : S.plans) {
        Plan& q = *kv.second;
        const PlanKey &a = q.key, &b = p.key;
        if (&q == &p || q.resource_limited || !q.tiled || q.trial_tag == tag || a.reference == b.reference ||
            a.ortho != b.ortho || a.persp != b.persp || a.seed != b.seed || a.screen != b.screen || a.ss != b.ss ||
            a.force_two != b.force_two || q.size != p.size || q.views != p.views)
            continue;
        ensure_trial(q);
        ensure_tile_data(S, q);
        same_views.push_back(&q);
    }
    const uint32_t chunk = p.views; // no state field (tile maxima by searches): all views at once
    auto read_back = [&](Plan& q) {
        launch_view_maxima(q.trial_t1.p, q.trial_t2.p, tiles, q.views, q.trial_max.p, st);
        B200_CUDA(cudaMemcpyAsync(q.trial_hpop.data(), q.trial_pop.p, q.trial_hpop.size() * 8, cudaMemcpyDeviceToHost,
                                  st));
        B200_CUDA(cudaMemcpyAsync(q.trial_hstate.data(), q.trial_state.p, q.trial_hstate.size() * 4,
                                  cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaMemcpyAsync(q.trial_hmax.data(), q.trial_max.p, q.trial_hmax.size() * 4, cudaMemcpyDeviceToHost,
                                  st));
    };
    for (int pass = p.deep ? 1 : 0; pass < 2; ++pass) { // as in refresh_state
        const bool saturate = pass == 1;
        uint32_t* const wide = saturate ? wide_counts(S, p) : nullptr;
        // Exact (not held) state counts of the current state: the trial's are
        // those plus the changed faces' deltas, instead of a full count.
        const bool incremental = !saturate && delta && !p.deep && p.state_count.p &&
                                 p.state_revision == S.state_revision;
        if (incremental) {
            B200_CUDA(cudaMemcpyAsync(p.trial_count.p, p.state_count.p, cstride * p.views, cudaMemcpyDeviceToDevice,
                                      st));
            B200_CUDA(cudaMemcpyAsync(p.trial_state.p, p.raster_state.p, 16 * size_t(p.views),
                                      cudaMemcpyDeviceToDevice, st));
            DevMesh state = S.state.view;
            state.nf = S.state_faces;
            launch_count_delta_views(state, *delta, p.cameras.p, p.views, S.bounds.center, p.key.ss, p.size,
                                     p.key.force_two, p.trial_count.p, cstride, p.trial_state.p, st);
        }
        for (uint32_t v0 = 0; v0 < p.views; v0 += chunk) {
            const uint32_t n = std::min(chunk, p.views - v0);
            const size_t w0 = size_t(p.words) * v0, s0 = samples * v0, t0 = size_t(tiles) * v0;
            launch_refresh_views(cand, p.cameras.p + v0, n, S.bounds.center, p.key.ss, p.size, p.key.force_two,
                                 p.trial_count.p + cstride * v0, cstride, p.trial_state.p + 4 * v0,
                                 p.trial_bits.p + w0, p.ref_bits.p + w0, p.words, p.trial_pop.p + 4 * v0,
                                 p.ref_field.p + s0, nullptr, nullptr, nullptr, nullptr, nullptr,
                                 p.trial_t1.p + t0, p.trial_t2.p + t0, saturate, st, wide, !incremental);
            for (Plan* q : same_views) {
                B200_CUDA(cudaMemcpyAsync(q->trial_count.p + cstride * v0, p.trial_count.p + cstride * v0,
                                          cstride * n, cudaMemcpyDeviceToDevice, st));
                B200_CUDA(cudaMemcpyAsync(q->trial_bits.p + w0, p.trial_bits.p + w0, size_t(p.words) * n * 4,
                                          cudaMemcpyDeviceToDevice, st));
                B200_CUDA(cudaMemcpyAsync(q->trial_state.p + 4 * v0, p.trial_state.p + 4 * v0, 16 * size_t(n),
                                          cudaMemcpyDeviceToDevice, st));
                launch_compare_views(n, p.size, p.trial_bits.p + w0, q->ref_bits.p + w0, p.words, q->ref_field.p + s0,
                                     nullptr, q->trial_t1.p + t0, q->trial_t2.p + t0, q->trial_pop.p + 4 * v0, st);
            }
        }
        read_back(p);
        for (Plan* q : same_views) read_back(*q);
        B200_CUDA(cudaStreamSynchronize(st));
        B200_CUDA(cudaGetLastError());
        bool overflow = false;
        for (uint32_t v = 0; v < p.views; ++v) overflow |= p.trial_hstate[4 * v + 3] != 0;
        if (!overflow) break;
        p.deep = true;
    }
    p.trial_tag = tag;
    for (Plan* q : same_views) q->trial_tag = tag;
    S.profile.launches += 8 + 6 * same_views.size();
}

// evaluate_impl (evaluate.cpp:312-352) over the per-view data of trial_views.
// Returns false when a view would refine to a finer sampling (the caller then
// takes the full-raster path for the gate).
static bool gate_from_trial(const Plan& p, const GateSettings& g, Measurement& result) {
    result = default_measurement();
    result.supersample = g.supersample;
    for (uint32_t v = 0; v < p.views; ++v) {
        ViewRecord rec{};
        rec.changed = uint32_t(p.trial_hpop[4 * v]);
        rec.total = uint32_t(p.trial_hpop[4 * v + 1]);
        rec.ca = p.trial_hpop[4 * v + 2] > 0;
        rec.cb = p.trial_hpop[4 * v + 3] > 0;
        rec.flags = uint8_t((p.hviews[v].clipped_ref ? kRecClippedRef : 0) |
                            (p.trial_hstate[4 * v + 2] ? kRecClippedCand : 0));
        // A clipped view's reference raster stops at the first clipped face;
        // its changed area comes from the full-raster path.
        if (rec.flags) return false;
        double max_d2 = 0;
        if (rec.changed && rec.ca && rec.cb)
            max_d2 = double(std::max(std::max(p.trial_hmax[2 * v], p.trial_hmax[2 * v + 1]), 0));
        Measurement cur = default_measurement();
        cur.worst_view = v;
        finish_view(cur, rec, g, p.key.ss, max_d2);
        if (!refinement_done(cur, g, p.key.ss)) return false;
        if (!aggregate_view(result, cur, v)) return true;
    }
    return true;
}

// The four gates of the combined trial in the session's trial buffers.
// Returns the failed gate (1..4) or 0 when accepted.
static int gates_of_trial(Session& S, const DevMesh& cand, const GateRef gates[4], const PlanKey keys[4],
                          uint64_t tag, const TrialDelta* delta = nullptr) {
    (void)keys;
    for (int gi = 0; gi < 4; ++gi)
        if (!measurement_accepted(gate_of_trial(S, cand, gates[gi], gi, tag, nullptr, delta))) return gi + 1;
    return 0;
}

// Makes the trial in the session's trial buffers the state; plans that
// evaluated this trial take its data as their state data.
static void commit_trial(Session& S, uint32_t faces, uint64_t tag) {
    DevMesh& m = S.state.view;
    cudaStream_t st = S.stream;
    B200_CUDA(cudaMemcpyAsync(S.state.idx.p, S.trial.idx.p, size_t(faces) * 12, cudaMemcpyDeviceToDevice, st));
    B200_CUDA(cudaMemcpyAsync(S.state.pos.p, S.trial.pos.p, size_t(m.nv) * 12, cudaMemcpyDeviceToDevice, st));
    if (m.mat) B200_CUDA(cudaMemcpyAsync(S.state.mat.p, S.trial.mat.p, size_t(faces) * 2, cudaMemcpyDeviceToDevice, st));
    if (m.uv) B200_CUDA(cudaMemcpyAsync(S.state.uv.p, S.trial.uv.p, size_t(m.nv) * 8, cudaMemcpyDeviceToDevice, st));
    m.nf = faces;
    S.state_faces = faces;
    ++S.state_revision;
    S.state_is_source = false;
    for (auto& kv : S.plans) {
        Plan& p = *kv.second;
        if (p.resource_limited || !p.tiled || p.trial_tag != tag || !p.state_bits.p) continue;
        std::swap(p.state_count, p.trial_count);
        std::swap(p.state_bits, p.trial_bits);
        std::swap(p.t1, p.trial_t1);
        std::swap(p.t2, p.trial_t2);
        std::swap(p.raster_state, p.trial_state);
        std::swap(p.pop, p.trial_pop);
        std::swap(p.hstate, p.trial_hstate);
        std::swap(p.hpop, p.trial_hpop);
        p.trial_tag = 0;
        const size_t samples = size_t(p.size) * p.size, cstride = count_stride(samples);
        const uint32_t tiles = ((p.size + 31) / 32) * ((p.size + 31) / 32);
        p.state_is_ref = false;
        for (uint32_t v = 0; v < p.views; ++v) {
            PlanView& pv = p.hviews[v];
            pv.state_bits = p.state_bits.p + size_t(v) * p.words;
            pv.state_count = p.state_count.p + cstride * v;
            pv.tile_t1 = p.t1.p + size_t(tiles) * v;
            pv.tile_t2 = p.t2.p + size_t(tiles) * v;
            pv.ref_field = p.ref_field.p + samples * v;
            pv.changed = uint32_t(p.hpop[4 * v]);
            pv.total = uint32_t(p.hpop[4 * v + 1]);
            pv.cov_ref = uint32_t(p.hpop[4 * v + 2]);
            pv.cov_state = uint32_t(p.hpop[4 * v + 3]);
            pv.clip_state = p.hstate[4 * v + 2];
        }
        B200_CUDA(cudaMemcpyAsync(p.dviews.p, p.hviews.data(), p.views * sizeof(PlanView), cudaMemcpyHostToDevice, st));
        p.dev.state_is_ref = 0;
        p.state_revision = S.state_revision;
    }
    rebuild_topology(S);
}

// Builds the combined trial of the first `count` selected edits; returns its
// face count and whether validate_placement rejected it.
static uint32_t build_batch_trial(Session& S, uint32_t count, bool& invalid) {
    const DevMesh& m = S.state.view;
    Topology& t = S.topo;
    cudaStream_t st = S.stream;
    launch_batch_trial(m, t.view, t.edits.p, S.batch_selected.p, count, S.batch_remap.p, S.batch_owner.p,
                       S.batch_placements.p, S.trial_keep.p, S.trial_offsets.p, S.trial.idx.p, S.trial.mat.p,
                       S.trial.pos.p, S.batch_table.p, S.batch_table_cap, S.batch_info.p, t.scan.p, st, t.uv(),
                       S.trial.uv.p);
    uint32_t host[2] = {0, 0};
    B200_CUDA(cudaMemcpyAsync(&host[0], S.trial_offsets.p + m.nf, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaMemcpyAsync(&host[1], S.batch_info.p, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    B200_CUDA(cudaGetLastError());
    S.profile.launches += 5;
    invalid = host[1] != 0;
    return host[0];
}

// Executor with batches of up to `batch` collapses (GpuActionState::execute,
// action_gpu.cu:1947-2086 with select_batch and verdict, 865-915;
// execute_actions, action.cpp:453-525): rank, select a disjoint batch from the
// ranked position, audit the combined trial through the four gates, halve it
// on rejection; a rejected singleton moves the position one past the batch's
// first edit; an accepted batch is committed and the edits re-ranked.
// Surrogate pruning of the ranked edits: features and MLP scores of every
// legal edit, the `keep` edits with the highest acceptance logits, and the
// ShortestEdge order restricted to them (S.sur_order).
static void prune_ranked(Session& S, uint32_t actions, uint32_t keep, float px, float px2) {
    SurrogateModel& model = *S.surrogate;
    Topology& t = S.topo;
    cudaStream_t st = S.stream;
    const size_t cap = 6ull * S.source.view.nf + 1;
    S.sur_features.ensure(S.pool, cap * kSurrogateIn);
    S.sur_out.ensure(S.pool, 2 * cap);
    S.sur_keys_in.ensure(S.pool, cap);
    S.sur_keys_out.ensure(S.pool, cap);
    S.sur_idx_in.ensure(S.pool, cap);
    S.sur_idx_out.ensure(S.pool, cap);
    S.sur_flags.ensure(S.pool, cap);
    S.sur_rank_flags.ensure(S.pool, cap + 1);
    S.sur_offsets.ensure(S.pool, cap + 1);
    S.sur_order.ensure(S.pool, cap);
    launch_features(S.state.view, t.view, t.edits.p, t.offsets.p + t.total_nbrs, actions, px, px2,
                    S.sur_features.p, st);
    B200_CUDA(launch_mlp(model.dev(), S.sur_features.p, actions, S.sur_out.p, nullptr, 0.f, nullptr, model.error.p,
                         148, st));
    launch_prune_prepare(S.sur_out.p, actions, S.sur_keys_in.p, S.sur_idx_in.p, st);
    size_t bytes = S.sort_bytes;
    B200_CUDA(sort_scores_desc(S.sur_keys_in.p, S.sur_keys_out.p, S.sur_idx_in.p, S.sur_idx_out.p, actions,
                               S.sort_temp.p, bytes, st));
    launch_prune_order(S.sur_idx_out.p, actions, keep, S.sur_flags.p, S.sorted_order.p, S.sur_rank_flags.p,
                       S.sur_offsets.p, t.scan.p, S.sur_order.p, st);
    S.profile.launches += 7;
}

static void execute_batched(Session& S, uint32_t target, uint32_t budget, const blitz_eval_settings gates_in[4],
                            uint32_t batch, uint32_t keep_permille, uint32_t* commits_out, size_t capacity,
                            blitz_audit_execution& out, int ranking = 3) {
    target = std::max<uint32_t>(1, target);
    cudaStream_t st = S.stream;
    Topology& t = S.topo;
    const DevMesh& src = S.source.view;
    const double diameter = std::max(1e-20, S.bounds.radius * 2);
    const size_t cap = 6ull * src.nf + 1;
    S.scores.ensure(S.pool, cap);
    S.sorted_scores.ensure(S.pool, cap);
    S.order.ensure(S.pool, cap);
    S.sorted_order.ensure(S.pool, cap);
    if (!S.sort_temp.p) {
        size_t bytes = 0;
        B200_CUDA(sort_scores_desc(nullptr, nullptr, nullptr, nullptr, uint32_t(cap), nullptr, bytes, st));
        S.sort_temp = Buf<unsigned char>(S.pool, bytes);
        S.sort_bytes = bytes;
    }
    ensure_trial_buffers(S);
    if (!S.batch_selected.p) {
        S.batch_selected = Buf<uint32_t>(S.pool, 64);
        S.batch_ctl = Buf<uint32_t>(S.pool, 2);
        S.batch_out = Buf<uint32_t>(S.pool, 3);
        S.batch_used = Buf<uint32_t>(S.pool, (src.nv + 31) / 32 + 1);
        S.batch_remap = Buf<uint32_t>(S.pool, src.nv);
        S.batch_owner = Buf<uint32_t>(S.pool, src.nv);
        S.batch_table_cap = uint32_t(pow2_at_least(2ull * src.nv));
        S.batch_table = Buf<uint32_t>(S.pool, S.batch_table_cap);
        S.batch_info = Buf<uint32_t>(S.pool, 1);
        S.batch_placements = Buf<float>(S.pool, 3 * 64);
    }
    GateRef gates[4];
    PlanKey keys[4];
    resolve_gates(S, gates_in, gates, keys);
    const float px = float(gates_in[0].screen_size / std::max(1e-20, 2 * S.bounds.radius));
    const float px2 = float(gates_in[2].screen_size / std::max(1e-20, 2 * S.bounds.radius));
    uint32_t fallbacks = 0;
    uint32_t commits = 0, trials = 0;
    uint64_t audited = 0;
    uint8_t reason = 3;
    std::vector<blitz_collapse> chosen(64);
    for (;;) {
        const uint32_t faces = S.state_faces;
        if (faces <= target) {
            reason = 0;
            break;
        }
        if (trials >= budget) {
            reason = 1;
            break;
        }
        const uint32_t actions = t.actions;
        if (!actions) {
            reason = 2;
            break;
        }
        rank_edits(S, actions, diameter, ranking, gates_in, S.scores.p, S.order.p, st);
        size_t bytes = S.sort_bytes;
        B200_CUDA(sort_scores_desc(S.scores.p, S.sorted_scores.p, S.order.p, S.sorted_order.p, actions, S.sort_temp.p,
                                   bytes, st));
        bool accepted = false;
        // With a surrogate the walk first covers the pruned order; the full
        // order is the fallback when nothing there is accepted.
        const uint32_t* walk_order = S.sorted_order.p;
        uint32_t walk_count = actions;
        bool pruned = false;
        if (keep_permille && S.surrogate) {
            const uint32_t keep = std::max<uint32_t>(1, uint32_t((uint64_t(actions) * keep_permille + 999) / 1000));
            if (keep < actions) {
                prune_ranked(S, actions, keep, px, px2);
                walk_order = S.sur_order.p;
                walk_count = keep;
                pruned = true;
            }
        }
        uint32_t position = 0;
        for (;;) {
        while (position < walk_count && trials < budget && !accepted) {
            const uint32_t ctl[2] = {position, faces - target};
            B200_CUDA(cudaMemcpyAsync(S.batch_ctl.p, ctl, 8, cudaMemcpyHostToDevice, st));
            B200_CUDA(launch_select_batch(t.view, t.edits.p, walk_order, walk_count, S.batch_ctl.p, batch,
                                          S.state.view.nv, S.batch_used.p, S.batch_selected.p, S.batch_out.p, st));
            uint32_t sel[3];
            B200_CUDA(cudaMemcpyAsync(sel, S.batch_out.p, 12, cudaMemcpyDeviceToHost, st));
            B200_CUDA(cudaStreamSynchronize(st));
            S.profile.launches += 1;
            uint32_t count = sel[0];
            const uint32_t first = sel[1];
            if (!count) break;
            while (count && trials < budget) {
                bool invalid = false;
                const uint32_t trial_faces = build_batch_trial(S, count, invalid);
                const uint64_t tag = ++S.trial_tag;
                ++trials;
                audited += count;
                DevMesh cand = S.state.view;
                cand.pos = S.trial.pos.p;
                cand.idx = S.trial.idx.p;
                cand.mat = S.state.view.mat ? S.trial.mat.p : nullptr;
                cand.nf = trial_faces;
                // the trial as changes of the state (incremental face counts)
                const TrialDelta delta{t.geometry.p, S.batch_remap.p, S.batch_owner.p, S.trial_keep.p,
                                       S.trial_offsets.p, cand};
                if (!invalid && trial_faces && gates_of_trial(S, cand, gates, keys, tag, &delta) == 0) {
                    S.collapse_dev.ensure(S.pool, 64);
                    launch_gather_window(t.edits.p, S.batch_selected.p, 0, count, S.collapse_dev.p, st);
                    B200_CUDA(cudaMemcpyAsync(chosen.data(), S.collapse_dev.p, count * sizeof(blitz_collapse),
                                              cudaMemcpyDeviceToHost, st));
                    B200_CUDA(cudaStreamSynchronize(st));
                    for (uint32_t k = 0; k < count; ++k) {
                        if (commits < capacity && commits_out) {
                            commits_out[2 * commits] = chosen[k].from;
                            commits_out[2 * commits + 1] = chosen[k].to;
                        }
                        ++commits;
                    }
                    commit_trial(S, trial_faces, tag);
                    accepted = true;
                    break;
                }
                if (count > 1) {
                    count /= 2;
                } else {
                    count = 0;
                    position = first + 1;
                }
            }
        }
        if (accepted || !pruned || trials >= budget) break;
        // exhaustive fallback over the full ranked order
        pruned = false;
        walk_order = S.sorted_order.p;
        walk_count = actions;
        position = 0;
        ++fallbacks;
        }
        if (!accepted) {
            reason = trials >= budget ? 1 : 3;
            break;
        }
    }
    if (S.surrogate) {
        uint32_t err = 0;
        B200_CUDA(cudaMemcpyAsync(&err, S.surrogate->error.p, 4, cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaStreamSynchronize(st));
        if (err) throw Failure(BLITZ_INTERNAL_ERROR, "surrogate tensor-core wait timed out");
    }
    out.commits = commits;
    out.trials = trials;
    out.final_faces = S.state_faces;
    out.audited = audited;
    out.stop_reason = reason;
    out.reserved[0] = uint8_t(std::min<uint32_t>(fallbacks, 255));
}

// Greedy executor with batches of one (GpuActionState::execute,
// action_gpu.cu:1947-2086; execute_actions, action.cpp:453-525): rank the legal
// midpoint collapses by ShortestEdge, walk them in rank order skipping those
// that would remove more faces than remain above the target, audit each
// through the four gates and commit the first accepted, then re-rank. Every
// trial of the walk is audited against the same state, so the walk is audited
// speculatively in ranked windows (one batched launch each) and replayed in
// order on the host; the result equals the serial loop trial for trial.
static void execute(Session& S, uint32_t target, uint32_t budget, const blitz_eval_settings gates[4],
                    uint32_t* commits_out, size_t capacity, blitz_audit_execution& out, int ranking = 3) {
    target = std::max<uint32_t>(1, target);
    cudaStream_t st = S.stream;
    Topology& t = S.topo;
    const double diameter = std::max(1e-20, S.bounds.radius * 2);
    const size_t cap = 6ull * S.source.view.nf + 1;
    S.scores.ensure(S.pool, cap);
    S.sorted_scores.ensure(S.pool, cap);
    S.order.ensure(S.pool, cap);
    S.sorted_order.ensure(S.pool, cap);
    if (!S.sort_temp.p) {
        size_t bytes = 0;
        B200_CUDA(sort_scores_desc(nullptr, nullptr, nullptr, nullptr, uint32_t(cap), nullptr, bytes, st));
        S.sort_temp = Buf<unsigned char>(S.pool, bytes);
        S.sort_bytes = bytes;
    }
    uint32_t window = 64;
    uint32_t commits = 0, trials = 0;
    uint64_t audited = 0;
    uint8_t reason = 3;
    std::vector<blitz_candidate_verdict> hv;
    std::vector<blitz_collapse> hc;
    for (;;) {
        const uint32_t faces = S.state_faces;
        if (faces <= target) {
            reason = 0;
            break;
        }
        if (trials >= budget) {
            reason = 1;
            break;
        }
        const uint32_t actions = t.actions;
        if (!actions) {
            reason = 2;
            break;
        }
        rank_edits(S, actions, diameter, ranking, gates, S.scores.p, S.order.p, st);
        size_t bytes = S.sort_bytes;
        B200_CUDA(sort_scores_desc(S.scores.p, S.sorted_scores.p, S.order.p, S.sorted_order.p, actions, S.sort_temp.p,
                                   bytes, st));
        const uint32_t remaining = faces - target;
        bool accepted = false;
        blitz_collapse chosen{};
        for (uint32_t position = 0; position < actions && trials < budget && !accepted;) {
            const uint32_t n = std::min(window, actions - position);
            S.collapse_dev.ensure(S.pool, n);
            S.verdict_dev.ensure(S.pool, size_t(n) * sizeof(blitz_candidate_verdict));
            launch_gather_window(t.edits.p, S.sorted_order.p, position, n, S.collapse_dev.p, st);
            auto* vd = reinterpret_cast<blitz_candidate_verdict*>(S.verdict_dev.p);
            audit_candidates(S, S.collapse_dev.p, nullptr, n, gates, vd, nullptr, st);
            audited += n;
            hv.resize(n);
            hc.resize(n);
            B200_CUDA(cudaMemcpyAsync(hv.data(), vd, n * sizeof(blitz_candidate_verdict), cudaMemcpyDeviceToHost, st));
            B200_CUDA(cudaMemcpyAsync(hc.data(), S.collapse_dev.p, n * sizeof(blitz_collapse), cudaMemcpyDeviceToHost, st));
            B200_CUDA(cudaStreamSynchronize(st));
            for (uint32_t k = 0; k < n && trials < budget; ++k) {
                if (hv[k].removed > remaining) continue;
                ++trials;
                if (hv[k].accepted) {
                    accepted = true;
                    chosen = hc[k];
                    break;
                }
            }
            position += n;
            if (!accepted) window = std::min<uint32_t>(window * 2, 8192);
        }
        if (!accepted) {
            reason = trials >= budget ? 1 : 3;
            break;
        }
        if (commits < capacity && commits_out) {
            commits_out[2 * commits] = chosen.from;
            commits_out[2 * commits + 1] = chosen.to;
        }
        ++commits;
        commit_collapse(S, chosen);
        window = std::max<uint32_t>(32, window / 2);
    }
    out.commits = commits;
    out.trials = trials;
    out.final_faces = S.state_faces;
    out.audited = audited;
    out.stop_reason = reason;
}

} // namespace b200

// ---------------------------------------------------------------------------
// C ABI
using namespace b200;

struct blitz_audit_session {
    Session s;
};

namespace {
void message(char* out, size_t n, const char* text) {
    if (out && n) {
        size_t k = std::min(n - 1, std::strlen(text));
        std::memcpy(out, text, k);
        out[k] = 0;
    }
}
template <class F> blitz_status guarded(char* error, size_t cap, F f) {
    message(error, cap, "");
    try {
        f();
        return BLITZ_OK;
    } catch (const Failure& e) {
        message(error, cap, e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        message(error, cap, "host allocation failed");
        return BLITZ_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        message(error, cap, e.what());
        return BLITZ_INTERNAL_ERROR;
    } catch (...) {
        message(error, cap, "unknown failure");
        return BLITZ_INTERNAL_ERROR;
    }
}
uint64_t now_ns() {
    return uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                        std::chrono::steady_clock::now().time_since_epoch())
                        .count());
}
} // namespace

extern "C" {

uint32_t blitz_abi_version(void) { return BLITZ_ABI_VERSION; }

blitz_status blitz_neural_options_v2_init(blitz_neural_options_v2* out, size_t n) {
    if (!out || n != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    *out = blitz_neural_options_v2{};
    out->struct_size = sizeof(*out);
    out->version = 2;
    out->device = 0;
    out->memory_mib = 6144;
    out->action_trials = 64;
    out->ranking_seed = 0xB1172026u;
    out->exact_position_bps = 500;
    out->action_batch = 32;
    out->origin = 0;
    out->ranking = 0;
    out->confirmation = 1;
    out->raster_backend = 0;
    out->vertex_storage = 3;
    out->preserve_uv = 1;
    out->overdraw_tiebreak = 1;
    out->cache_rasters = 1;
    out->mask_only_coverage = 1;
    out->direct_targets = 1;
    out->view_batch = 4;
    out->candidate_batch = 1;
    return BLITZ_OK;
}

blitz_status blitz_eval_settings_init(blitz_eval_settings* out, size_t n) {
    if (!out || n != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    *out = blitz_eval_settings{};
    out->struct_size = sizeof(*out);
    out->profile = 0;
    out->supersample = 8;
    out->max_supersample = 32;
    out->views_orthographic = 642;
    out->views_perspective = 64;
    out->views_seed = 0xB1172026u;
    out->screen_size = 512;
    out->limit = 2;
    out->max_changed_area = 1;
    return BLITZ_OK;
}

blitz_status blitz_audit_session_create(const blitz_mesh* source, const blitz_neural_options_v2* options,
                                        blitz_audit_session** out, char* error, size_t cap) {
    if (out) *out = nullptr;
    return guarded(error, cap, [&] {
        if (!out) throw Failure(BLITZ_INVALID_ARGUMENT, "null session destination");
        blitz_neural_options_v2 o;
        blitz_neural_options_v2_init(&o, sizeof(o));
        if (options) {
            if (options->struct_size != sizeof(*options) || options->version != 2 || options->reserved[0] ||
                options->reserved[1] || options->reserved[2] || options->preserve_uv > 1)
                throw Failure(BLITZ_INVALID_ARGUMENT, "invalid neural v2 descriptor");
            if (options->raster_backend != 0) throw Failure(BLITZ_UNAVAILABLE, "only the CUDA raster backend exists");
            o = *options;
        }
        if (o.memory_mib < 128) throw Failure(BLITZ_INVALID_ARGUMENT, "memory_mib below 128");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count <= o.device || o.device < 0) {
            cudaGetLastError();
            throw Failure(BLITZ_UNAVAILABLE, "no CUDA device for the audit session");
        }
        HostMesh h = import_mesh(source);
        Bounds b = bounds_of(h);
        if (!(b.radius > 0) || !std::isfinite(b.radius))
            throw Failure(BLITZ_INVALID_ARGUMENT, "zero or invalid source extent");
        if (!o.preserve_uv) {
            // Without preserve_uv the GPU state welds every corner to its
            // attribute class ignoring uv and tangents (action_gpu.cu:1527-1532
            // weld_uv_indices), so uv seams are no wedges; the welded indices
            // are the session's source and state (the same triangles).
            const std::vector<uint32_t> root = attribute_roots(h, false);
            for (uint32_t& i : h.idx) i = root[i];
        }
        auto session = std::make_unique<blitz_audit_session>();
        Session& S = session->s;
        S.device = o.device;
        S.options = o;
        S.pool.limit = size_t(o.memory_mib) << 20;
        DeviceScope scope(S.device);
        B200_CUDA(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking));
        S.source_h = std::move(h);
        S.bounds = b;
        S.source.upload(S.pool, S.source_h, S.stream);
        S.state.upload(S.pool, S.source_h, S.stream);
        S.state_faces = S.state.view.nf;
        init_topology(S);
        rebuild_topology(S);
        *out = session.release();
    });
}

void blitz_audit_session_destroy(blitz_audit_session* s) {
    if (!s) return;
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(s->s.device);
    delete s;
    cudaSetDevice(previous);
}

blitz_status blitz_audit_bind_reference(blitz_audit_session* s, const blitz_mesh* previous, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s) throw Failure(BLITZ_INVALID_ARGUMENT, "null session");
        Session& S = s->s;
        DeviceScope scope(S.device);
        if (!previous) {
            S.previous_is_source = true;
            S.previous = DeviceMesh{};
            S.previous_h = HostMesh{};
        } else {
            HostMesh h = import_mesh(previous);
            if (same_data(h, S.source_h)) {
                S.previous_is_source = true;
                S.previous = DeviceMesh{};
                S.previous_h = HostMesh{};
            } else {
                S.previous_h = std::move(h);
                S.previous.upload(S.pool, S.previous_h, S.stream);
                S.previous_is_source = false;
            }
        }
        // Plans against the previous reference are stale.
        for (auto it = S.plans.begin(); it != S.plans.end();)
            it = it->first.reference == 1 ? S.plans.erase(it) : std::next(it);
        B200_CUDA(cudaStreamSynchronize(S.stream));
    });
}

blitz_status blitz_audit_evaluate(blitz_audit_session* s, const blitz_mesh* reference, const blitz_mesh* candidate,
                                  const blitz_eval_settings* settings, blitz_measurement* out, char* error,
                                  size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !out) throw Failure(BLITZ_INVALID_ARGUMENT, "null session or output");
        Session& S = s->s;
        DeviceScope scope(S.device);
        uint64_t t0 = now_ns();
        GateSettings g = gate_of(settings, S.bounds);
        HostMesh ref = import_mesh(reference), cand = import_mesh(candidate);
        Measurement result = default_measurement();
        result.supersample = g.supersample;
        if (!identical(ref, cand)) {
            DeviceMesh dr, dc;
            dr.upload(S.pool, ref, S.stream);
            dc.upload(S.pool, cand, S.stream);
            result = evaluate_full(S, dr.view, dc.view, settings, g);
            B200_CUDA(cudaStreamSynchronize(S.stream));
        }
        std::memcpy(out, &result, sizeof(*out));
        S.info.gpu_audit_ns += now_ns() - t0;
    });
}

blitz_status blitz_audit_raster(blitz_audit_session* s, const blitz_mesh* mesh, double screen, uint8_t ss,
                                uint16_t ortho, uint16_t persp, uint32_t seed, uint32_t view, uint8_t force_two,
                                uint64_t* words, size_t word_capacity, uint32_t* size_out, uint8_t* clipped,
                                char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !words || !size_out || !clipped) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        if (!ss || !std::isfinite(screen) || screen <= 0 || screen > 16384)
            throw Failure(BLITZ_INVALID_ARGUMENT, "invalid raster extent");
        if (view >= uint32_t(ortho) + persp) throw Failure(BLITZ_INVALID_ARGUMENT, "view outside camera set");
        uint32_t size = raster_size(screen, ss);
        if (uint64_t(size) * size > kMaxSamples) throw Failure(BLITZ_BUDGET_LIMITED, "raster exceeds per-view memory budget");
        size_t n = (size_t(size) * size + 63) / 64;
        if (word_capacity < n) throw Failure(BLITZ_INVALID_ARGUMENT, "word buffer too small");
        HostMesh h = import_mesh(mesh);
        DeviceMesh d;
        d.upload(S.pool, h, S.stream);
        auto cams = make_cameras(S.bounds, screen, ortho, persp, seed);
        Buf<Camera> cam(S.pool, 1);
        B200_CUDA(cudaMemcpyAsync(cam.p, &cams[view], sizeof(Camera), cudaMemcpyHostToDevice, S.stream));
        Buf<uint32_t> bits(S.pool, mask_words(size));
        Buf<uint32_t> state(S.pool, 4);
        B200_CUDA(cudaMemsetAsync(bits.p, 0, bits.n * 4, S.stream));
        raster(S, d.view, &cams[view], ss, size, force_two, true, bits.p, nullptr, state.p);
        uint32_t st[4];
        B200_CUDA(cudaMemcpyAsync(words, bits.p, n * 8, cudaMemcpyDeviceToHost, S.stream));
        B200_CUDA(cudaMemcpyAsync(st, state.p, sizeof(st), cudaMemcpyDeviceToHost, S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
        *size_out = size;
        *clipped = st[1] != 0;
    });
}

blitz_status blitz_audit_coverage_distance(blitz_audit_session* s, const uint64_t* a, const uint64_t* b,
                                           uint32_t width, uint32_t height, uint8_t ss, int masks_on_device,
                                           double* out, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !a || !b || !out) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        if (!width || !height || !ss) throw Failure(BLITZ_INVALID_ARGUMENT, "raster shapes differ");
        const size_t samples = size_t(width) * height;
        if (samples > kMaxSamples) throw Failure(BLITZ_BUDGET_LIMITED, "raster exceeds per-view memory budget");
        Session& S = s->s;
        DeviceScope scope(S.device);
        ensure_scratch_samples(S, samples);
        Scratch& x = S.scratch;
        const size_t n = (samples + 63) / 64;
        const cudaMemcpyKind kind = masks_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        B200_CUDA(cudaMemsetAsync(x.a.p, 0, size_t(mask_words_for(samples)) * 4, S.stream));
        B200_CUDA(cudaMemsetAsync(x.c.p, 0, size_t(mask_words_for(samples)) * 4, S.stream));
        B200_CUDA(cudaMemcpyAsync(x.a.p, a, n * 8, kind, S.stream));
        B200_CUDA(cudaMemcpyAsync(x.c.p, b, n * 8, kind, S.stream));
        ViewRecord rec{};
        double max_d2 = 0;
        mask_distance(S, width, height, rec, max_d2);
        *out = coverage_value(rec, ss, max_d2);
    });
}

blitz_status blitz_audit_actions(blitz_audit_session* s, blitz_collapse* out, size_t capacity, size_t* count,
                                 char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !count || (capacity && !out)) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        *count = S.topo.actions;
        size_t k = std::min<size_t>(capacity, S.topo.actions);
        if (!k) return;
        std::vector<Edit> edits(k);
        B200_CUDA(cudaMemcpyAsync(edits.data(), S.topo.edits.p, k * sizeof(Edit), cudaMemcpyDeviceToHost, S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
        for (size_t i = 0; i < k; ++i) out[i] = blitz_collapse{edits[i].from, edits[i].to, 0, {0, 0, 0}};
    });
}

blitz_status blitz_audit_candidates_device(blitz_audit_session* s, const blitz_collapse* candidates_device, size_t n,
                                           const blitz_eval_settings gates[4], blitz_candidate_verdict* out_device,
                                           blitz_measurement* measurements_device, void* stream, char* error,
                                           size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !gates || (n && (!candidates_device || !out_device)))
            throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        uint64_t t0 = now_ns();
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : S.stream;
        audit_candidates(S, candidates_device, nullptr, n, gates, out_device,
                         reinterpret_cast<Measurement*>(measurements_device), st);
        S.info.gpu_audit_ns += now_ns() - t0;
    });
}

blitz_status blitz_audit_candidates(blitz_audit_session* s, const blitz_collapse* candidates, size_t n,
                                    const blitz_eval_settings gates[4], blitz_candidate_verdict* out,
                                    blitz_measurement* measurements, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !gates || (n && (!candidates || !out))) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        uint64_t t0 = now_ns();
        S.collapse_dev.ensure(S.pool, std::max<size_t>(n, 1));
        S.verdict_dev.ensure(S.pool, std::max<size_t>(n, 1) * sizeof(blitz_candidate_verdict));
        if (measurements) S.meas_dev.ensure(S.pool, std::max<size_t>(n, 1) * 4);
        if (n)
            B200_CUDA(cudaMemcpyAsync(S.collapse_dev.p, candidates, n * sizeof(blitz_collapse), cudaMemcpyHostToDevice,
                                      S.stream));
        auto* vd = reinterpret_cast<blitz_candidate_verdict*>(S.verdict_dev.p);
        audit_candidates(S, S.collapse_dev.p, candidates, n, gates, vd, measurements ? S.meas_dev.p : nullptr, S.stream);
        if (n) {
            B200_CUDA(cudaMemcpyAsync(out, vd, n * sizeof(*out), cudaMemcpyDeviceToHost, S.stream));
            if (measurements)
                B200_CUDA(cudaMemcpyAsync(measurements, S.meas_dev.p, n * 4 * sizeof(blitz_measurement),
                                          cudaMemcpyDeviceToHost, S.stream));
        }
        B200_CUDA(cudaStreamSynchronize(S.stream));
        for (size_t i = 0; i < n; ++i) out[i].accepted ? ++S.info.legal_collapses : ++S.info.rejected_collapses;
        S.info.gpu_audit_ns += now_ns() - t0;
    });
}

blitz_status blitz_audit_execute(blitz_audit_session* s, uint32_t target_faces, uint32_t trial_budget,
                                 const blitz_eval_settings gates[4], uint32_t* commits_from_to, size_t capacity,
                                 blitz_audit_execution* out, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !gates || !out || out->struct_size != sizeof(*out))
            throw Failure(BLITZ_INVALID_ARGUMENT, "null argument or bad execution descriptor");
        Session& S = s->s;
        DeviceScope scope(S.device);
        for (int g = 0; g < 4; ++g) gate_of(&gates[g], S.bounds);
        uint64_t t0 = now_ns();
        blitz_audit_execution r{};
        r.struct_size = sizeof(r);
        execute(S, target_faces, trial_budget, gates, commits_from_to, capacity, r);
        *out = r;
        S.info.gpu_audit_ns += now_ns() - t0;
        S.info.legal_collapses += r.commits;
        S.info.rejected_collapses += r.trials - r.commits;
    });
}

void blitz_execute_options_init(blitz_execute_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(*o);
    o->batch = 1;
    o->ranking = 3;
}

blitz_status blitz_audit_execute_ex(blitz_audit_session* s, uint32_t target_faces, uint32_t trial_budget,
                                    const blitz_eval_settings gates[4], const blitz_execute_options* options,
                                    uint32_t* commits_from_to, size_t capacity, blitz_audit_execution* out,
                                    char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !gates || !out || !options || out->struct_size != sizeof(*out) ||
            options->struct_size != sizeof(*options))
            throw Failure(BLITZ_INVALID_ARGUMENT, "null argument or bad execution descriptor");
        if (options->batch < 1 || options->batch > 64)
            throw Failure(BLITZ_INVALID_ARGUMENT, "action batch outside 1..64");
        if (options->ranking != 0 && options->ranking != 1 && options->ranking != 3 && options->ranking != 4)
            throw Failure(BLITZ_INVALID_ARGUMENT, "ranking must be learned (0), constant (1), shortest edge (3) or "
                                                  "current plane (4)");
        if (options->ranking == 0 && !s->s.surrogate)
            throw Failure(BLITZ_INVALID_ARGUMENT, "learned ranking needs an attached surrogate");
        if (options->keep_permille > 1000)
            throw Failure(BLITZ_INVALID_ARGUMENT, "surrogate keep share above 1000 permille");

        if (options->keep_permille && !s->s.surrogate)
            throw Failure(BLITZ_INVALID_ARGUMENT, "no surrogate attached to the session");
        for (uint32_t r : options->reserved)
            if (r) throw Failure(BLITZ_INVALID_ARGUMENT, "reserved execution options must be zero");
        Session& S = s->s;
        DeviceScope scope(S.device);
        for (int g = 0; g < 4; ++g) gate_of(&gates[g], S.bounds);
        uint64_t t0 = now_ns();
        blitz_audit_execution r{};
        r.struct_size = sizeof(r);
        if (options->batch == 1 && !options->keep_permille)
            execute(S, target_faces, trial_budget, gates, commits_from_to, capacity, r, int(options->ranking));
        else
            execute_batched(S, target_faces, trial_budget, gates, options->batch, options->keep_permille,
                            commits_from_to, capacity, r, int(options->ranking));
        *out = r;
        S.info.gpu_audit_ns += now_ns() - t0;
        S.info.legal_collapses += r.commits;
        S.info.rejected_collapses += r.trials - std::min(r.trials, r.commits);
    });
}

blitz_status blitz_audit_state(blitz_audit_session* s, uint32_t* indices, size_t index_capacity, float* positions,
                               size_t position_capacity, uint32_t* face_count, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !face_count) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        const DevMesh& m = S.state.view;
        *face_count = S.state_faces;
        if (indices && index_capacity >= size_t(S.state_faces) * 3)
            B200_CUDA(cudaMemcpyAsync(indices, m.idx, size_t(S.state_faces) * 12, cudaMemcpyDeviceToHost, S.stream));
        if (positions && position_capacity >= size_t(m.nv) * 3)
            B200_CUDA(cudaMemcpyAsync(positions, m.pos, size_t(m.nv) * 12, cudaMemcpyDeviceToHost, S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
    });
}

blitz_status blitz_audit_state_uv(blitz_audit_session* s, float* uv, size_t uv_capacity, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !uv) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        const DevMesh& m = S.state.view;
        if (!m.uv) throw Failure(BLITZ_INVALID_ARGUMENT, "the session's mesh has no uv");
        if (uv_capacity < size_t(m.nv) * 2) throw Failure(BLITZ_INVALID_ARGUMENT, "uv capacity below 2 per vertex");
        B200_CUDA(cudaMemcpyAsync(uv, m.uv, size_t(m.nv) * 8, cudaMemcpyDeviceToHost, S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
    });
}

blitz_status blitz_audit_state_materials(blitz_audit_session* s, uint16_t* materials, size_t capacity,
                                         uint32_t* face_count, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !face_count) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        Session& S = s->s;
        DeviceScope scope(S.device);
        const DevMesh& m = S.state.view;
        *face_count = S.state_faces;
        if (!m.mat) throw Failure(BLITZ_INVALID_ARGUMENT, "the session's mesh has no materials");
        if (materials && capacity >= S.state_faces) {
            B200_CUDA(cudaMemcpyAsync(materials, m.mat, size_t(S.state_faces) * 2, cudaMemcpyDeviceToHost, S.stream));
            B200_CUDA(cudaStreamSynchronize(S.stream));
        }
    });
}

blitz_status blitz_audit_reset(blitz_audit_session* s, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s) throw Failure(BLITZ_INVALID_ARGUMENT, "null session");
        Session& S = s->s;
        DeviceScope scope(S.device);
        reset_state(S);
    });
}

blitz_status blitz_audit_profile_enable(blitz_audit_session* s, int enable) {
    return guarded(nullptr, 0, [&] {
        if (!s) throw Failure(BLITZ_INVALID_ARGUMENT, "null session");
        Session& S = s->s;
        DeviceScope scope(S.device);
        if (enable && !S.ev[0])
            for (auto& e : S.ev) B200_CUDA(cudaEventCreate(&e));
        if (enable < 0 || enable > 2) throw Failure(BLITZ_INVALID_ARGUMENT, "profile mode is 0, 1 or 2");
        S.profiling = enable != 0;
        S.counting = enable == 1;
        S.profile = blitz_audit_profile{};
    });
}

blitz_status blitz_audit_profile_read(const blitz_audit_session* s, blitz_audit_profile* out) {
    if (!s || !out || out->struct_size != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    blitz_audit_profile p = s->s.profile;
    p.struct_size = sizeof(p);
    p.enabled = s->s.profiling;
    *out = p;
    return BLITZ_OK;
}

blitz_status blitz_audit_session_info(const blitz_audit_session* s, blitz_neural_info* out) {
    if (!s || !out || out->struct_size != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    blitz_neural_info i = s->s.info;
    i.struct_size = sizeof(i);
    *out = i;
    return BLITZ_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Learned audit surrogate (no reference counterpart).
struct blitz_surrogate {
    SurrogateModel m;
};

namespace {
uint64_t mix64(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
// Uploads the FP32 masters, refreshes the BF16 copies and resets Adam.
void upload_params(SurrogateModel& M, const float* params, const float* mean, const float* inv_std) {
    cudaStream_t st = M.stream;
    std::vector<float> p(params, params + kParams);
    for (uint32_t i = 0; i < kParams; ++i)
        if (!surrogate_param_live(i)) p[i] = 0;
    std::vector<__nv_bfloat16> pb(kParams);
    for (uint32_t i = 0; i < kParams; ++i) pb[i] = __float2bfloat16_rn(p[i]);
    B200_CUDA(cudaMemcpyAsync(M.master.p, p.data(), kParams * 4, cudaMemcpyHostToDevice, st));
    B200_CUDA(cudaMemcpyAsync(M.wb.p, pb.data(), kParams * 2, cudaMemcpyHostToDevice, st));
    B200_CUDA(cudaMemsetAsync(M.m.p, 0, kParams * 4, st));
    B200_CUDA(cudaMemsetAsync(M.v.p, 0, kParams * 4, st));
    B200_CUDA(cudaMemsetAsync(M.grads.p, 0, kParams * 4, st));
    if (mean) B200_CUDA(cudaMemcpyAsync(M.norm.p, mean, kSurrogateIn * 4, cudaMemcpyHostToDevice, st));
    if (inv_std) B200_CUDA(cudaMemcpyAsync(M.norm.p + kSurrogateIn, inv_std, kSurrogateIn * 4, cudaMemcpyHostToDevice, st));
    B200_CUDA(cudaStreamSynchronize(st));
    M.step = 0;
}
// One fused forward + backward pass over n rows into the gradient accumulators.
float accumulate_gradients(SurrogateModel& M, const float* features, const float* labels, size_t n, cudaStream_t st) {
    if (!features || !labels || !n || n > (size_t(1) << 31)) throw Failure(BLITZ_INVALID_ARGUMENT, "bad training batch");
    B200_CUDA(cudaMemsetAsync(M.loss.p, 0, 4, st));
    B200_CUDA(cudaMemsetAsync(M.error.p, 0, 4, st));
    B200_CUDA(launch_mlp(M.dev(), features, uint32_t(n), nullptr, labels, float(1.0 / double(n)), M.loss.p,
                         M.error.p, 148, st));
    float loss = 0;
    uint32_t err = 0;
    B200_CUDA(cudaMemcpyAsync(&loss, M.loss.p, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaMemcpyAsync(&err, M.error.p, 4, cudaMemcpyDeviceToHost, st));
    B200_CUDA(cudaStreamSynchronize(st));
    if (err) throw Failure(BLITZ_INTERNAL_ERROR, "surrogate tensor-core wait timed out");
    return loss / float(n);
}
} // namespace

blitz_status blitz_surrogate_create(int device, uint32_t seed, blitz_surrogate** out, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!out) throw Failure(BLITZ_INVALID_ARGUMENT, "null output");
        *out = nullptr;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
            cudaGetLastError();
            throw Failure(BLITZ_UNAVAILABLE, "no CUDA device for the surrogate");
        }
        auto h = std::make_unique<blitz_surrogate>();
        SurrogateModel& M = h->m;
        M.device = device;
        M.pool.limit = size_t(64) << 20;
        DeviceScope scope(device);
        B200_CUDA(cudaStreamCreateWithFlags(&M.stream, cudaStreamNonBlocking));
        M.master = Buf<float>(M.pool, kParams);
        M.grads = Buf<float>(M.pool, kParams);
        M.m = Buf<float>(M.pool, kParams);
        M.v = Buf<float>(M.pool, kParams);
        M.wb = Buf<__nv_bfloat16>(M.pool, kParams);
        M.norm = Buf<float>(M.pool, 2 * kSurrogateIn);
        M.loss = Buf<float>(M.pool, 1);
        M.error = Buf<uint32_t>(M.pool, 1);
        M.mask = Buf<uint8_t>(M.pool, kParams);
        std::vector<uint8_t> mask(kParams);
        for (uint32_t i = 0; i < kParams; ++i) mask[i] = surrogate_param_live(i);
        B200_CUDA(cudaMemcpyAsync(M.mask.p, mask.data(), kParams, cudaMemcpyHostToDevice, M.stream));
        B200_CUDA(cudaMemsetAsync(M.error.p, 0, 4, M.stream));
        // He-uniform weights (fan-in 48, 128, 128), zero biases.
        std::vector<float> p(kParams, 0.f);
        uint64_t state = seed;
        auto uni = [&](float bound) {
            return float((double(mix64(state) >> 11) * 0x1.0p-53 * 2 - 1) * bound);
        };
        for (uint32_t i = 0; i < 8192; ++i) p[kOffW1 + i] = uni(std::sqrt(6.f / kSurrogateIn));
        for (uint32_t i = 0; i < 16384; ++i) p[kOffW2 + i] = uni(std::sqrt(6.f / 128));
        for (uint32_t i = 0; i < 2048; ++i) p[kOffW3 + i] = uni(std::sqrt(6.f / 128));
        std::vector<float> mean(kSurrogateIn, 0.f), inv(kSurrogateIn, 1.f);
        upload_params(M, p.data(), mean.data(), inv.data());
        *out = h.release();
    });
}

void blitz_surrogate_destroy(blitz_surrogate* h) {
    if (!h) return;
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(h->m.device);
    delete h;
    cudaSetDevice(previous);
}

blitz_status blitz_surrogate_load(blitz_surrogate* h, const float* params, size_t count, const float* mean,
                                  const float* inv_std, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!h || !params || count != kParams) throw Failure(BLITZ_INVALID_ARGUMENT, "bad surrogate parameters");
        DeviceScope scope(h->m.device);
        upload_params(h->m, params, mean, inv_std);
    });
}

blitz_status blitz_surrogate_save(const blitz_surrogate* h, float* params, size_t capacity, float* mean,
                                  float* inv_std, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!h || (params && capacity < kParams)) throw Failure(BLITZ_INVALID_ARGUMENT, "bad surrogate output");
        const SurrogateModel& M = h->m;
        DeviceScope scope(M.device);
        if (params) B200_CUDA(cudaMemcpyAsync(params, M.master.p, kParams * 4, cudaMemcpyDeviceToHost, M.stream));
        if (mean) B200_CUDA(cudaMemcpyAsync(mean, M.norm.p, kSurrogateIn * 4, cudaMemcpyDeviceToHost, M.stream));
        if (inv_std)
            B200_CUDA(cudaMemcpyAsync(inv_std, M.norm.p + kSurrogateIn, kSurrogateIn * 4, cudaMemcpyDeviceToHost,
                                      M.stream));
        B200_CUDA(cudaStreamSynchronize(M.stream));
    });
}

blitz_status blitz_surrogate_score(blitz_surrogate* h, const float* features, size_t n, float* out, void* stream,
                                   char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!h || (n && (!features || !out)) || n > (size_t(1) << 31))
            throw Failure(BLITZ_INVALID_ARGUMENT, "bad surrogate scoring arguments");
        SurrogateModel& M = h->m;
        DeviceScope scope(M.device);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : M.stream;
        B200_CUDA(cudaMemsetAsync(M.error.p, 0, 4, st));
        B200_CUDA(launch_mlp(M.dev(), features, uint32_t(n), out, nullptr, 0.f, nullptr, M.error.p, 148, st));
        uint32_t err = 0;
        B200_CUDA(cudaMemcpyAsync(&err, M.error.p, 4, cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaStreamSynchronize(st));
        if (err) throw Failure(BLITZ_INTERNAL_ERROR, "surrogate tensor-core wait timed out");
    });
}

blitz_status blitz_surrogate_gradients(blitz_surrogate* h, const float* features, const float* labels, size_t n,
                                       float* gradients, size_t capacity, float* loss, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!h || !gradients || capacity < kParams) throw Failure(BLITZ_INVALID_ARGUMENT, "bad gradient output");
        SurrogateModel& M = h->m;
        DeviceScope scope(M.device);
        B200_CUDA(cudaMemsetAsync(M.grads.p, 0, kParams * 4, M.stream));
        const float l = accumulate_gradients(M, features, labels, n, M.stream);
        B200_CUDA(cudaMemcpyAsync(gradients, M.grads.p, kParams * 4, cudaMemcpyDeviceToHost, M.stream));
        B200_CUDA(cudaMemsetAsync(M.grads.p, 0, kParams * 4, M.stream));
        B200_CUDA(cudaStreamSynchronize(M.stream));
        if (loss) *loss = l;
    });
}

blitz_status blitz_surrogate_train_step(blitz_surrogate* h, const float* features, const float* labels, size_t n,
                                        float lr, float* loss, void* stream, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!h || !(lr > 0)) throw Failure(BLITZ_INVALID_ARGUMENT, "bad training step");
        SurrogateModel& M = h->m;
        DeviceScope scope(M.device);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : M.stream;
        const float l = accumulate_gradients(M, features, labels, n, st);
        ++M.step;
        launch_adam(M.master.p, M.grads.p, M.m.p, M.v.p, M.wb.p, kParams, lr, 0.9f, 0.999f, 1e-8f, M.step, M.mask.p,
                    st);
        B200_CUDA(cudaGetLastError());
        if (loss) *loss = l;
    });
}

blitz_status blitz_audit_surrogate_features(blitz_audit_session* s, double screen, double screen2, float* features,
                                            blitz_collapse* collapses, size_t capacity, size_t* count, char* error,
                                            size_t cap) {
    return guarded(error, cap, [&] {
        if (!s || !count || !(screen > 0) || !(screen2 > 0))
            throw Failure(BLITZ_INVALID_ARGUMENT, "bad feature arguments");
        Session& S = s->s;
        DeviceScope scope(S.device);
        Topology& t = S.topo;
        *count = t.actions;
        if (!features || capacity < t.actions) return;
        const float px = float(screen / std::max(1e-20, 2 * S.bounds.radius));
        const float px2 = float(screen2 / std::max(1e-20, 2 * S.bounds.radius));
        launch_features(S.state.view, t.view, t.edits.p, t.offsets.p + t.total_nbrs, t.actions, px, px2, features,
                        S.stream);
        if (collapses && t.actions) {
            S.order.ensure(S.pool, t.actions);
            std::vector<uint32_t> iota(t.actions);
            for (uint32_t i = 0; i < t.actions; ++i) iota[i] = i;
            B200_CUDA(cudaMemcpyAsync(S.order.p, iota.data(), t.actions * 4, cudaMemcpyHostToDevice, S.stream));
            S.collapse_dev.ensure(S.pool, t.actions);
            launch_gather_window(t.edits.p, S.order.p, 0, t.actions, S.collapse_dev.p, S.stream);
            B200_CUDA(cudaMemcpyAsync(collapses, S.collapse_dev.p, t.actions * sizeof(blitz_collapse),
                                      cudaMemcpyDeviceToHost, S.stream));
        }
        B200_CUDA(cudaStreamSynchronize(S.stream));
        B200_CUDA(cudaGetLastError());
    });
}

blitz_status blitz_audit_attach_surrogate(blitz_audit_session* s, blitz_surrogate* h, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s) throw Failure(BLITZ_INVALID_ARGUMENT, "null session");
        if (h && h->m.device != s->s.device) throw Failure(BLITZ_INVALID_ARGUMENT, "surrogate on another device");
        s->s.surrogate = h ? &h->m : nullptr;
    });
}

// ---------------------------------------------------------------------------
// Batched audit of several sessions' candidates in one persistent launch.
struct blitz_audit_batch {
    std::vector<blitz_audit_session*> sessions;
    int device = 0;
    cudaStream_t stream = nullptr;
    Pool pool;
    Buf<CandidateRecord> records;
    Buf<blitz_collapse> host_cands;         // device copies for the host entry point
    Buf<blitz_candidate_verdict> host_out;
    std::vector<Buf<AuditEntry>> entries; // per plan slot
    std::vector<uint32_t> nentries;
    std::vector<uint64_t> units;
    Buf<uint32_t> queue, spill, spill_huge, spill_giant, spill_far, exact;
    cudaEvent_t giant_fork = nullptr, giant_join = nullptr;
    Buf<unsigned char> huge, giant;
    uint32_t huge_blocks = 0;
    int variant = kAuditTierSmall;
    bool tuned = false;
    float tune_ms[4] = {0, 0, 0, 0};
    // captured launch sequence and the inputs it was captured for
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint8_t> signature;
    uint64_t graph_launches = 0, exact_candidates = 0;
    // profile of the last call with BLITZ_BATCH_PROFILE
    Buf<unsigned long long> stats;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> marks; // per plan slot, 4 (launch_audit)
    float audit_ms = 0, tier_ms[3] = {0, 0, 0};
    unsigned long long prof[kAuditStats] = {};
    // Side streams that run the sessions' small per-candidate launches
    // (records, verdicts) side by side, forked from and joined to the
    // batch's stream by events (captured into the graph as parallel
    // branches).
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> side_done;
    cudaEvent_t fork = nullptr;
    void ensure_side(size_t n) {
        if (!fork) B200_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        while (side.size() < n) {
            cudaStream_t s;
            cudaEvent_t e;
            B200_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            side.push_back(s);
            B200_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            side_done.push_back(e);
        }
    }
    // Runs launch(i, stream) for i < n spread over the side streams; `st`
    // waits for all of them.
    template <class F> void side_by_side(size_t n, cudaStream_t st, F&& launch) {
        const size_t k = std::min(side.size(), n);
        B200_CUDA(cudaEventRecord(fork, st));
        for (size_t j = 0; j < k; ++j) B200_CUDA(cudaStreamWaitEvent(side[j], fork, 0));
        for (size_t i = 0; i < n; ++i) launch(i, side[i % k]);
        for (size_t j = 0; j < k; ++j) {
            B200_CUDA(cudaEventRecord(side_done[j], side[j]));
            B200_CUDA(cudaStreamWaitEvent(st, side_done[j], 0));
        }
    }
    ~blitz_audit_batch() {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
        for (auto e : side_done) cudaEventDestroy(e);
        for (auto e : marks) cudaEventDestroy(e);
        if (giant_fork) cudaEventDestroy(giant_fork);
        if (giant_join) cudaEventDestroy(giant_join);
        for (auto s_ : side) cudaStreamDestroy(s_);
        if (fork) cudaEventDestroy(fork);
        stats.release();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        records.release(), queue.release(), spill.release(), spill_huge.release(), exact.release(), huge.release();
        host_cands.release(), host_out.release();
        spill_giant.release(), spill_far.release(), giant.release();
        entries.clear();
        if (stream) cudaStreamDestroy(stream);
    }
};

blitz_status blitz_audit_batch_create(blitz_audit_session* const* sessions, size_t count, blitz_audit_batch** out,
                                      char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!out || !sessions || !count) throw Failure(BLITZ_INVALID_ARGUMENT, "no sessions");
        *out = nullptr;
        auto b = std::make_unique<blitz_audit_batch>();
        for (size_t i = 0; i < count; ++i) {
            if (!sessions[i]) throw Failure(BLITZ_INVALID_ARGUMENT, "null session");
            if (sessions[i]->s.device != sessions[0]->s.device)
                throw Failure(BLITZ_INVALID_ARGUMENT, "sessions on different devices");
            b->sessions.push_back(sessions[i]);
        }
        b->device = sessions[0]->s.device;
        b->pool.limit = size_t(1) << 40;
        DeviceScope scope(b->device);
        B200_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        *out = b.release();
    });
}

void blitz_audit_batch_destroy(blitz_audit_batch* b) {
    if (!b) return;
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(b->device);
    delete b;
    cudaSetDevice(previous);
}

// One batched audit of device candidates into device verdicts on `st`
// (blitz_audit_batch_candidates without the status wrapper); synchronises.
static void batch_candidates(blitz_audit_batch* b, const blitz_collapse* cands, const size_t* counts,
                             const blitz_eval_settings gates_in[4], blitz_candidate_verdict* out, uint32_t flags,
                             cudaStream_t st) {
    {
        if (!b || !counts || !gates_in || flags > 15) throw Failure(BLITZ_INVALID_ARGUMENT, "bad batch arguments");
        const bool counting = (flags & 4u) != 0, profile = counting || (flags & 8u) != 0;
        if (profile && (flags & 1u)) throw Failure(BLITZ_INVALID_ARGUMENT, "profiling runs without graph replay");
        const size_t ns = b->sessions.size();
        std::vector<uint64_t> off(ns + 1, 0);
        for (size_t i = 0; i < ns; ++i) {
            if (counts[i] > UINT32_MAX / 2) throw Failure(BLITZ_INVALID_ARGUMENT, "too many candidates");
            off[i + 1] = off[i] + counts[i];
        }
        if (off[ns] && (!cands || !out)) throw Failure(BLITZ_INVALID_ARGUMENT, "null candidate or verdict array");
        if (off[ns] > UINT32_MAX) throw Failure(BLITZ_INVALID_ARGUMENT, "too many candidates");
        for (int g = 0; g < 4; ++g) gate_of(&gates_in[g], b->sessions[0]->s.bounds);
        // Plans (built or refreshed on each session's own stream) and tables.
        std::vector<AuditSetup> setup(ns);
        size_t slots = 0;
        bool big = false, giant = false;
        for (size_t i = 0; i < ns; ++i) {
            Session& S = b->sessions[i]->s;
            setup_audit(S, gates_in, setup[i], true);
            if (upload_verdict_tables(S, setup[i], uint32_t(counts[i]), S.stream))
                B200_CUDA(cudaStreamSynchronize(S.stream));
            slots = std::max(slots, setup[i].plans.size());
            for (Plan* p : setup[i].plans) big |= p->size > 256, giant |= p->size > 1024;
        }
        b->records.ensure(b->pool, std::max<uint64_t>(1, off[ns]));
        b->entries.resize(slots);
        b->nentries.assign(slots, 0);
        b->units.assign(slots, 0);
        uint64_t max_units = 0;
        for (size_t j = 0; j < slots; ++j) {
            std::vector<AuditEntry> e;
            uint64_t first = 0;
            for (size_t i = 0; i < ns; ++i) {
                if (j >= setup[i].plans.size() || !counts[i]) continue;
                Plan& p = *setup[i].plans[j];
                e.push_back(AuditEntry{p.dev, b->records.p + off[i], p.records.p, first});
                first += uint64_t(counts[i]) * p.views;
            }
            if (first > UINT32_MAX) throw Failure(BLITZ_INVALID_ARGUMENT, "too many (candidate, view) units");
            b->entries[j].ensure(b->pool, std::max<size_t>(1, e.size()));
            if (!e.empty())
                B200_CUDA(cudaMemcpyAsync(b->entries[j].p, e.data(), e.size() * sizeof(AuditEntry),
                                          cudaMemcpyHostToDevice, st));
            b->nentries[j] = uint32_t(e.size());
            b->units[j] = first;
            max_units = std::max(max_units, first);
        }
        b->queue.ensure(b->pool, 8);
        b->spill.ensure(b->pool, max_units + 1);
        b->exact.ensure(b->pool, ns);
        if (big && !b->huge.p) {
            int sms = 148;
            B200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
            b->huge_blocks = uint32_t(std::max(1, 3 * sms));
            b->huge = Buf<unsigned char>(b->pool, audit_huge_scratch_bytes(b->huge_blocks));
        }
        if (big) b->spill_huge.ensure(b->pool, max_units + 1);
        if (giant && !b->giant.p) b->giant = Buf<unsigned char>(b->pool, audit_giant_scratch_bytes(kGiantBlocks));
        if (giant) b->spill_giant.ensure(b->pool, max_units + 1), b->spill_far.ensure(b->pool, max_units + 1);
        GiantTier giant_tier{b->spill_giant.p, b->giant.p, kGiantBlocks};
        B200_CUDA(cudaStreamSynchronize(st));
        // The launch sequence: per-session records, one audit job per plan
        // slot over all sessions, per-session verdicts.
        if (profile && !b->stats.p) {
            b->stats = Buf<unsigned long long>(b->pool, kAuditStats);
            B200_CUDA(cudaEventCreate(&b->ev[0]));
            B200_CUDA(cudaEventCreate(&b->ev[1]));
        }
        while (profile && b->marks.size() < 4 * slots) {
            cudaEvent_t e;
            B200_CUDA(cudaEventCreate(&e));
            b->marks.push_back(e);
        }
        b->ensure_side(std::min<size_t>(ns, 16));
        if (giant) {
            // units beyond the huge tier's regions: the giant tier beside the
            // huge tier, on the first side stream
            if (!b->giant_fork) {
                B200_CUDA(cudaEventCreateWithFlags(&b->giant_fork, cudaEventDisableTiming));
                B200_CUDA(cudaEventCreateWithFlags(&b->giant_join, cudaEventDisableTiming));
            }
            giant_tier.far = b->spill_far.p;
            giant_tier.side = b->side.empty() ? nullptr : b->side[0];
            giant_tier.fork = b->giant_fork, giant_tier.join = b->giant_join;
        }
        auto body = [&](int variant) {
            b->side_by_side(ns, st, [&](size_t i, cudaStream_t ss) {
                if (!counts[i]) return;
                Session& S = b->sessions[i]->s;
                Topology& t = S.topo;
                launch_prepare(S.state.view, t.view, S.state.view, t.view, cands + off[i], uint32_t(counts[i]),
                               t.positions.p, t.pos_cap, t.flat.p, S.options.preserve_uv != 0, b->records.p + off[i],
                               ss, t.uv());
            });
            if (profile) {
                cudaMemsetAsync(b->stats.p, 0, kAuditStats * 8, st);
                cudaEventRecord(b->ev[0], st);
            }
            for (size_t j = 0; j < slots; ++j) {
                if (!b->units[j]) continue;
                AuditJob job{};
                job.entries = b->entries[j].p, job.nentries = b->nentries[j], job.total = b->units[j];
                launch_audit(job, counting ? b->stats.p : nullptr, b->queue.p, b->spill.p,
                             big ? b->spill_huge.p : nullptr, big ? b->huge.p : nullptr, big ? b->huge_blocks : 0,
                             st, variant, giant ? &giant_tier : nullptr, profile ? b->marks.data() + 4 * j : nullptr);
            }
            if (profile) cudaEventRecord(b->ev[1], st);
            cudaMemsetAsync(b->exact.p, 0, 4 * ns, st);
            b->side_by_side(ns, st, [&](size_t i, cudaStream_t ss) {
                if (!counts[i]) return;
                Session& S = b->sessions[i]->s;
                launch_verdicts(S.record_table.p, S.plan_views.p, S.plan_ss.p, S.gate_table.p, b->records.p + off[i],
                                uint32_t(counts[i]), out + off[i], nullptr, b->exact.p + i, ss);
            });
        };
        // Autotune: time both warp-tier variants on this call, keep the faster.
        if ((flags & 2u) && off[ns]) {
            cudaEvent_t e0, e1;
            B200_CUDA(cudaEventCreate(&e0));
            B200_CUDA(cudaEventCreate(&e1));
            float best_ms = 0;
            for (int v = 0; v < 4; ++v) {
                if ((v & kAuditSpillHeavy) && !big) continue;
                body(v); // warm
                B200_CUDA(cudaEventRecord(e0, st));
                body(v);
                B200_CUDA(cudaEventRecord(e1, st));
                B200_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                B200_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                b->tune_ms[v] = ms;
                if (v == 0 || ms < best_ms) best_ms = ms, b->variant = v;
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            b->tuned = true;
            if (b->exec) cudaGraphExecDestroy(b->exec), b->exec = nullptr;
            if (b->graph) cudaGraphDestroy(b->graph), b->graph = nullptr;
        }
        // Inputs a captured graph is bound to.
        std::vector<uint8_t> sig;
        auto put = [&](const void* p, size_t n) {
            const uint8_t* c = static_cast<const uint8_t*>(p);
            sig.insert(sig.end(), c, c + n);
        };
        put(&cands, sizeof cands), put(&out, sizeof out), put(&st, sizeof st), put(counts, ns * sizeof(size_t));
        put(gates_in, 4 * sizeof(blitz_eval_settings)), put(&b->variant, sizeof b->variant);
        for (size_t i = 0; i < ns; ++i) {
            Session& S = b->sessions[i]->s;
            put(&S.state_revision, sizeof(uint64_t));
            put(&S.record_table.p, sizeof(void*));
            for (Plan* p : setup[i].plans) put(&p->records.p, sizeof(void*)), put(&p->dviews.p, sizeof(void*));
        }
        for (auto& e : b->entries) put(&e.p, sizeof(void*));
        for (const void* q : {(const void*)b->records.p, (const void*)b->queue.p, (const void*)b->spill.p,
                              (const void*)b->spill_huge.p, (const void*)b->huge.p, (const void*)b->exact.p,
                              (const void*)b->spill_giant.p, (const void*)b->giant.p, (const void*)b->spill_far.p})
            put(&q, sizeof(q));
        if ((flags & 1u) && off[ns]) {
            if (b->exec && sig == b->signature) {
                B200_CUDA(cudaGraphLaunch(b->exec, st));
                ++b->graph_launches;
            } else {
                if (b->exec) cudaGraphExecDestroy(b->exec), b->exec = nullptr;
                if (b->graph) cudaGraphDestroy(b->graph), b->graph = nullptr;
                body(b->variant); // this call's results; the capture below records the same sequence
                B200_CUDA(cudaStreamSynchronize(st));
                B200_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                body(b->variant);
                cudaError_t e = cudaStreamEndCapture(st, &b->graph);
                if (e != cudaSuccess) throw Failure(BLITZ_INTERNAL_ERROR, "batch graph capture failed");
                B200_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
                b->signature = sig;
            }
        } else {
            body(b->variant);
        }
        std::vector<uint32_t> exact(ns, 0);
        B200_CUDA(cudaMemcpyAsync(exact.data(), b->exact.p, 4 * ns, cudaMemcpyDeviceToHost, st));
        B200_CUDA(cudaStreamSynchronize(st));
        B200_CUDA(cudaGetLastError());
        if (profile && off[ns]) {
            B200_CUDA(cudaEventElapsedTime(&b->audit_ms, b->ev[0], b->ev[1]));
            if (counting) B200_CUDA(cudaMemcpy(b->prof, b->stats.p, sizeof(b->prof), cudaMemcpyDeviceToHost));
            for (float& t : b->tier_ms) t = 0;
            for (size_t j = 0; j < slots; ++j) {
                if (!b->units[j]) continue;
                for (int k = 0; k < 3; ++k) {
                    float ms = 0;
                    B200_CUDA(cudaEventElapsedTime(&ms, b->marks[4 * j + k], b->marks[4 * j + k + 1]));
                    b->tier_ms[k] += ms;
                }
            }
        }
        for (size_t i = 0; i < ns; ++i) {
            if (!exact[i]) continue;
            b->exact_candidates += exact[i];
            resolve_exact(b->sessions[i]->s, setup[i], cands + off[i], uint32_t(counts[i]), out + off[i], nullptr,
                          st);
        }
        for (size_t i = 0; i < ns; ++i) b->sessions[i]->s.info.decoded += counts[i];
    }
}

blitz_status blitz_audit_batch_candidates(blitz_audit_batch* b, const blitz_collapse* cands, const size_t* counts,
                                          const blitz_eval_settings gates_in[4], blitz_candidate_verdict* out,
                                          uint32_t flags, void* stream, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!b) throw Failure(BLITZ_INVALID_ARGUMENT, "null batch");
        DeviceScope scope(b->device);
        batch_candidates(b, cands, counts, gates_in, out, flags, stream ? static_cast<cudaStream_t>(stream) : b->stream);
    });
}

blitz_status blitz_audit_batch_candidates_host(blitz_audit_batch* b, const blitz_collapse* cands,
                                               const size_t* counts, const blitz_eval_settings gates_in[4],
                                               blitz_candidate_verdict* out, uint32_t flags, char* error,
                                               size_t cap) {
    return guarded(error, cap, [&] {
        if (!b || !counts) throw Failure(BLITZ_INVALID_ARGUMENT, "bad batch arguments");
        DeviceScope scope(b->device);
        size_t n = 0;
        for (size_t i = 0; i < b->sessions.size(); ++i) n += counts[i];
        if (n && (!cands || !out)) throw Failure(BLITZ_INVALID_ARGUMENT, "null candidate or verdict array");
        // Batch-owned device buffers: their addresses stay fixed from call to
        // call, so a captured graph of the launch sequence keeps replaying.
        b->host_cands.ensure(b->pool, std::max<size_t>(1, n));
        b->host_out.ensure(b->pool, std::max<size_t>(1, n));
        cudaStream_t st = b->stream;
        if (n)
            B200_CUDA(cudaMemcpyAsync(b->host_cands.p, cands, n * sizeof(blitz_collapse), cudaMemcpyHostToDevice, st));
        batch_candidates(b, b->host_cands.p, counts, gates_in, b->host_out.p, flags, st);
        if (n)
            B200_CUDA(cudaMemcpyAsync(out, b->host_out.p, n * sizeof(blitz_candidate_verdict), cudaMemcpyDeviceToHost,
                                      st));
        B200_CUDA(cudaStreamSynchronize(st));
    });
}

blitz_status blitz_audit_batch_read_info(const blitz_audit_batch* b, blitz_audit_batch_info* out) {
    if (!b || !out || out->struct_size != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    out->sessions = uint32_t(b->sessions.size());
    out->tier = uint32_t(b->variant);
    out->tuned = b->tuned ? 1u : 0u;
    out->graph_captured = b->exec ? 1u : 0u;
    for (int v = 0; v < 4; ++v) out->tune_ms[v] = b->tune_ms[v];
    out->graph_launches = b->graph_launches;
    out->exact_candidates = b->exact_candidates;
    out->audit_ms = b->audit_ms;
    for (int k = 0; k < 3; ++k) out->tier_ms[k] = b->tier_ms[k];
    out->units = b->prof[0];
    out->region_samples = b->prof[1];
    out->changed_samples = b->prof[2];
    for (int k = 0; k < 4; ++k) out->tier_units[k] = b->prof[3 + k], out->tier_cycles[k] = b->prof[7 + k];
    for (int k = 0; k < 3; ++k) out->phase_cycles[k] = b->prof[11 + k];
    out->flipped_samples = b->prof[14];
    for (int k = 0; k < 15; ++k) out->region_split[k] = b->prof[15 + k];
    out->face_samples = b->prof[30];
    for (int k = 0; k < 4; ++k) out->tier_max_cycles[k] = b->prof[31 + k];
    return BLITZ_OK;
}

// Per-view records of the session's state against a plan's reference, read
// from the plan's resident state data (popcounts, clip counts, tile maxima;
// the plan is refreshed first if the state moved on), for evaluate_full: the
// confirmation of a level redraws no raster. Views with clipping or a
// distance of 2^24 or more carry a flag, so evaluate_full redraws them.
static std::vector<ViewRecord> plan_state_records(Session& S, Plan& p) {
    std::vector<ViewRecord> recs(p.views);
    std::vector<int32_t> maxima(2 * size_t(p.views), -1);
    if (!p.state_is_ref && p.t1.p) {
        const uint32_t tiles = ((p.size + 31) / 32) * ((p.size + 31) / 32);
        S.view_maxima.ensure(S.pool, 2 * size_t(p.views));
        launch_view_maxima(p.t1.p, p.t2.p, tiles, p.views, S.view_maxima.p, S.stream);
        B200_CUDA(cudaMemcpyAsync(maxima.data(), S.view_maxima.p, maxima.size() * 4, cudaMemcpyDeviceToHost,
                                  S.stream));
        B200_CUDA(cudaStreamSynchronize(S.stream));
    }
    for (uint32_t v = 0; v < p.views; ++v) {
        ViewRecord& r = recs[v];
        r = ViewRecord{};
        r.changed = uint32_t(p.hpop[4 * v]);
        r.total = uint32_t(p.hpop[4 * v + 1]);
        r.ca = p.hpop[4 * v + 2] > 0;
        r.cb = p.hpop[4 * v + 3] > 0;
        r.flags = uint8_t((p.hviews[v].clipped_ref ? kRecClippedRef : 0) | (p.hstate[4 * v + 2] ? kRecClippedCand : 0));
        const int32_t m = std::max(std::max(maxima[2 * v], maxima[2 * v + 1]), 0);
        if (r.changed && r.ca && r.cb) r.max_d2 = uint32_t(m);
        if (r.max_d2 >= kExactLimit) r.flags |= kRecLarge;
    }
    return recs;
}

// ---------------------------------------------------------------------------
// LOD chain: schedule, per-level executor and confirmation.
namespace {
// Curve::at (chain.cpp:25-36).
double curve_at(const blitz_chain_settings& c, double t) {
    const float* xy = c.transition_curve;
    const uint32_t n = c.transition_points;
    if (t <= xy[0]) return xy[1];
    for (uint32_t i = 1; i < n; ++i)
        if (t <= xy[2 * i]) {
            const double u = (t - xy[2 * i - 2]) / (double(xy[2 * i]) - xy[2 * i - 2]);
            return xy[2 * i - 1] * (1 - u) + xy[2 * i + 1] * u;
        }
    return xy[2 * n - 1];
}
// The schedule's part of the settings checks (levels, pixels, curve).
void check_schedule(const blitz_chain_settings* c) {
    if (!c || c->struct_size != sizeof(*c)) throw Failure(BLITZ_INVALID_ARGUMENT, "bad chain settings");
    if (c->levels < 2 || c->levels > 32) throw Failure(BLITZ_INVALID_ARGUMENT, "level count must be 2..32");
    if (!(c->base_pixels >= c->last_pixels) || !(c->last_pixels > 0) || c->base_pixels > 16384)
        throw Failure(BLITZ_INVALID_ARGUMENT, "base pixels must be >= last pixels and <= 16384");
    if (c->transition_points < 1 || c->transition_points > 8)
        throw Failure(BLITZ_INVALID_ARGUMENT, "transition curve needs 1..8 points");
    if (!(c->max_lod0_delta_px >= 0) || !std::isfinite(c->max_lod0_delta_px))
        throw Failure(BLITZ_INVALID_ARGUMENT, "invalid optional pixel limit");
    // The curve rules of the reference's settings validation (chain.cpp:67-77).
    const float* xy = c->transition_curve;
    const uint32_t n = c->transition_points;
    if (xy[0] != 0 || xy[2 * (n - 1)] != 1) throw Failure(BLITZ_INVALID_ARGUMENT, "curves must span [0,1]");
    double last = -1;
    for (uint32_t i = 0; i < n; ++i) {
        const float x = xy[2 * i], y = xy[2 * i + 1];
        if (!std::isfinite(x) || !std::isfinite(y) || x <= last || x > 1 || y < 0 || y > 1e6)
            throw Failure(BLITZ_INVALID_ARGUMENT, "curve points must be ordered, finite and in 0..1e6");
        last = x;
    }
}
// schedule (chain.cpp:101-118): for levels 1..levels-1 the audited screen
// size S_i = S_0 (S_last / S_0)^(i / (levels - 1)), the transition bound
// delta_i = curve(t_i), and the LOD0 bound B_i = B_(i-1) S_i / S_(i-1) +
// delta_i, capped at max_lod0_delta_px when that is positive. Index 0 is the
// source: base pixels, bounds 0.
void chain_schedule(const blitz_chain_settings& c, double* pixels, double* transition, double* source) {
    pixels[0] = c.base_pixels, transition[0] = source[0] = 0;
    double cumulative = 0;
    for (uint32_t level = 1; level < c.levels; ++level) {
        const double p = c.base_pixels * std::pow(c.last_pixels / c.base_pixels, double(level) / (c.levels - 1));
        const double delta = curve_at(c, c.levels == 2 ? 0 : double(level - 1) / (c.levels - 2));
        cumulative = cumulative * p / pixels[level - 1] + delta;
        pixels[level] = p;
        transition[level] = delta;
        source[level] = c.max_lod0_delta_px > 0 ? std::min(cumulative, c.max_lod0_delta_px) : cumulative;
    }
}
blitz_eval_settings chain_gate(const blitz_chain_settings& c, double pixels, double limit, bool audit) {
    blitz_eval_settings e;
    std::memset(&e, 0, sizeof e);
    e.struct_size = sizeof e;
    e.profile = 0;
    e.supersample = audit ? c.audit_supersample : c.search_supersample;
    e.max_supersample = c.max_supersample;
    e.force_two_sided = c.force_two_sided;
    e.conservative_screen = 0;
    e.views_orthographic = audit ? c.audit_orthographic : c.search_orthographic;
    e.views_perspective = audit ? c.audit_perspective : c.search_perspective;
    e.views_seed = audit ? c.audit_seed : c.search_seed;
    e.screen_size = pixels;
    e.limit = limit;
    e.max_changed_area = audit ? c.max_changed_area : 1.0;
    return e;
}
} // namespace

void blitz_chain_settings_init(blitz_chain_settings* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->struct_size = sizeof(*c);
    c->levels = 2;
    c->base_pixels = c->last_pixels = 24;
    c->max_lod0_delta_px = 2;
    // the reference's default transition curve {(0, 2), (1, 3)} (remesher.hpp:12-13)
    c->transition_curve[0] = 0, c->transition_curve[1] = 2, c->transition_curve[2] = 1, c->transition_curve[3] = 3;
    c->transition_points = 2;
    c->search_orthographic = 42, c->search_perspective = 12, c->search_seed = 0xB1172024u;
    c->audit_orthographic = 642, c->audit_perspective = 64, c->audit_seed = 0xB1172026u;
    c->search_supersample = 4, c->audit_supersample = 8, c->max_supersample = 32;
    c->max_changed_area = 1.0;
    c->batch = 64;
    c->trial_budget = 1u << 30;
    c->min_faces = 1;
    c->ranking = 3;
}

blitz_status blitz_mesh_bounds(const blitz_mesh* mesh, float center[3], double* radius, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!mesh || !center || !radius) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        const HostMesh h = import_mesh(mesh);
        const Bounds b = bounds_of(h);
        for (int k = 0; k < 3; ++k) center[k] = b.center[k];
        *radius = b.radius;
    });
}

blitz_status blitz_view_cameras(const float center[3], double radius, double screen, uint16_t ortho, uint16_t persp,
                                uint32_t seed, blitz_view_camera* out, size_t capacity, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!center || !out) throw Failure(BLITZ_INVALID_ARGUMENT, "null argument");
        if (capacity < size_t(ortho) + persp) throw Failure(BLITZ_INVALID_ARGUMENT, "camera output too small");
        if (!(screen > 0) || !std::isfinite(screen) || !(radius > 0) || !std::isfinite(radius))
            throw Failure(BLITZ_INVALID_ARGUMENT, "screen and radius must be positive and finite");
        Bounds b{};
        for (int k = 0; k < 3; ++k) b.center[k] = center[k];
        b.radius = radius;
        const std::vector<Camera> cams = make_cameras(b, screen, ortho, persp, seed);
        static_assert(sizeof(blitz_view_camera) == sizeof(Camera), "camera layouts");
        for (size_t i = 0; i < cams.size(); ++i) {
            blitz_view_camera& o = out[i];
            std::memcpy(o.right, cams[i].right, 12), std::memcpy(o.up, cams[i].up, 12);
            std::memcpy(o.forward, cams[i].forward, 12);
            o.distance = cams[i].distance, o.focal = cams[i].focal, o.scale = cams[i].scale;
            o.perspective = cams[i].perspective, o.pad = 0;
        }
    });
}

blitz_status blitz_chain_schedule(const blitz_chain_settings* c, double* pixels, double* transition,
                                  double* source_bound, size_t capacity, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        check_schedule(c);
        if (!pixels || !transition || !source_bound || capacity < c->levels)
            throw Failure(BLITZ_INVALID_ARGUMENT, "schedule output needs `levels` entries");
        chain_schedule(*c, pixels, transition, source_bound);
    });
}

blitz_status blitz_audit_chain(blitz_audit_session* s, const blitz_chain_settings* c, blitz_chain_level* out,
                               size_t capacity, blitz_chain_emit emit, void* user, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!s) throw Failure(BLITZ_INVALID_ARGUMENT, "null session");
        check_schedule(c);
        if (c->batch < 1 || c->batch > 64) throw Failure(BLITZ_INVALID_ARGUMENT, "action batch outside 1..64");
        if (c->ranking != 0 && c->ranking != 1 && c->ranking != 3 && c->ranking != 4)
            throw Failure(BLITZ_INVALID_ARGUMENT, "unknown ranking");
        if (c->ranking == 0 && !s->s.surrogate) throw Failure(BLITZ_INVALID_ARGUMENT, "learned ranking needs a surrogate");
        if (out && capacity < c->levels - 1) throw Failure(BLITZ_INVALID_ARGUMENT, "level output too small");
        Session& S = s->s;
        DeviceScope scope(S.device);
        if (c->keep_permille && !S.surrogate) throw Failure(BLITZ_INVALID_ARGUMENT, "no surrogate attached");
        reset_state(S);
        auto bind_previous_source = [&] {
            S.previous_is_source = true;
            S.previous = DeviceMesh{};
            S.previous_h = HostMesh{};
            for (auto it = S.plans.begin(); it != S.plans.end();)
                it = it->first.reference == 1 ? S.plans.erase(it) : std::next(it);
        };
        bind_previous_source();
        double sched_pixels[32], sched_delta[32], sched_bound[32];
        chain_schedule(*c, sched_pixels, sched_delta, sched_bound);
        std::vector<uint32_t> idx;
        std::vector<float> pos;
        for (uint32_t level = 1; level < c->levels; ++level) {
            const uint64_t t0 = now_ns();
            const double pixels = sched_pixels[level], delta = sched_delta[level], bound = sched_bound[level];
            blitz_eval_settings gates[4] = {chain_gate(*c, pixels, bound, false), chain_gate(*c, pixels, delta, false),
                                            chain_gate(*c, pixels, bound, true), chain_gate(*c, pixels, delta, true)};
            for (int g = 0; g < 4; ++g) gate_of(&gates[g], S.bounds);
            // Plans of earlier levels' screen sizes are not used again.
            for (auto it = S.plans.begin(); it != S.plans.end();)
                it = it->first.screen != pixels ? S.plans.erase(it) : std::next(it);
            // previous level = the state now (the source for level 1)
            if (level >= 2) {
                HostMesh h;
                const DevMesh& m = S.state.view;
                h.idx.resize(size_t(S.state_faces) * 3);
                h.pos.resize(size_t(m.nv) * 3);
                B200_CUDA(cudaMemcpyAsync(h.idx.data(), m.idx, h.idx.size() * 4, cudaMemcpyDeviceToHost, S.stream));
                B200_CUDA(cudaMemcpyAsync(h.pos.data(), m.pos, h.pos.size() * 4, cudaMemcpyDeviceToHost, S.stream));
                if (m.mat) {
                    h.mat.resize(S.state_faces);
                    B200_CUDA(cudaMemcpyAsync(h.mat.data(), m.mat, h.mat.size() * 2, cudaMemcpyDeviceToHost, S.stream));
                }
                h.sided = S.source_h.sided;
                B200_CUDA(cudaStreamSynchronize(S.stream));
                S.previous_h = std::move(h);
                S.previous.upload(S.pool, S.previous_h, S.stream);
                S.previous_is_source = false;
                for (auto it = S.plans.begin(); it != S.plans.end();)
                    it = it->first.reference == 1 ? S.plans.erase(it) : std::next(it);
            }
            blitz_audit_execution r{};
            r.struct_size = sizeof(r);
            if (c->batch == 1 && !c->keep_permille)
                execute(S, c->min_faces, c->trial_budget, gates, nullptr, 0, r, int(c->ranking));
            else
                execute_batched(S, c->min_faces, c->trial_budget, gates, c->batch, c->keep_permille, nullptr, 0, r,
                                int(c->ranking));
            // confirmation at the audit views (generate.cpp:456-562)
            GateRef refs[4];
            PlanKey keys[4];
            resolve_gates(S, gates, refs, keys);
            DevMesh state = S.state.view;
            state.nf = S.state_faces;
            const DevMesh& prev = S.previous_is_source ? S.source.view : S.previous.view;
            // the audit plans hold the state's data against both references
            auto records = [&](int gi) {
                Plan& p = plan_for(S, keys[gi]);
                return p.resource_limited || !p.tiled ? std::vector<ViewRecord>() : plan_state_records(S, p);
            };
            const std::vector<ViewRecord> rs = records(2), rt = records(3);
            const Measurement ms = evaluate_full(S, S.source.view, state, &gates[2], refs[2].g,
                                                 rs.empty() ? nullptr : rs.data());
            const Measurement mt = evaluate_full(S, prev, state, &gates[3], refs[3].g, rt.empty() ? nullptr : rt.data());
            B200_CUDA(cudaStreamSynchronize(S.stream));
            if (out) {
                blitz_chain_level& l = out[level - 1];
                std::memset(&l, 0, sizeof l);
                l.struct_size = sizeof l;
                l.level = level;
                l.pixels = pixels, l.transition = delta, l.source_bound = bound;
                l.faces = S.state_faces, l.commits = r.commits, l.trials = r.trials;
                l.stop_reason = r.stop_reason;
                l.confirmed = measurement_accepted(ms) && measurement_accepted(mt);
                std::memcpy(&l.source_audit, &ms, sizeof ms);
                std::memcpy(&l.transition_audit, &mt, sizeof mt);
                l.seconds = double(now_ns() - t0) * 1e-9;
            }
            if (emit) {
                const DevMesh& m = S.state.view;
                idx.resize(size_t(S.state_faces) * 3);
                pos.resize(size_t(m.nv) * 3);
                B200_CUDA(cudaMemcpyAsync(idx.data(), m.idx, idx.size() * 4, cudaMemcpyDeviceToHost, S.stream));
                B200_CUDA(cudaMemcpyAsync(pos.data(), m.pos, pos.size() * 4, cudaMemcpyDeviceToHost, S.stream));
                B200_CUDA(cudaStreamSynchronize(S.stream));
                emit(user, level, idx.data(), S.state_faces, pos.data(), m.nv);
            }
        }
        bind_previous_source();
    });
}
