// The generation surface of blitz.h over the audit engine: settings and
// neural option defaults, BLZNET policy files, blitz_generate_neural and the
// result queries.
//
// blitz_generate_neural (c_api.cpp:294-304, neural/generate.cpp:127-562)
// runs the LOD chain of blitz_audit_chain: the schedule of blitz::schedule
// (chain.cpp:101-118), per level the four gates of eval_config / the gate
// hook (chain.cpp:179-199, generate.cpp:365-388) against the source and the
// previous level, the batched executor over midpoint collapses (the action
// proposals of GpuActionState::execute, action_gpu.cu:1947-2086) and the
// confirmation of the emitted level at the audit views (generate.cpp:456-562).
// Host code only: every audit runs in the engine's kernels.
#include "../../include/blitz_audit.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// ---- SHA-256 (FIPS 180-4, section 6.2) ----
class Sha256 {
  public:
    Sha256() {
        static const uint32_t init[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                                         0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
        std::memcpy(h_, init, sizeof h_);
    }
    void update(const uint8_t* p, size_t n) {
        bits_ += uint64_t(n) * 8;
        while (n) {
            const size_t take = std::min(n, size_t(64) - fill_);
            std::memcpy(block_ + fill_, p, take);
            fill_ += take, p += take, n -= take;
            if (fill_ == 64) compress(), fill_ = 0;
        }
    }
    std::string hex() {
        const uint64_t bits = bits_;
        const uint8_t one = 0x80, zero = 0;
        update(&one, 1);
        while (fill_ != 56) update(&zero, 1);
        uint8_t len[8];
        for (int i = 0; i < 8; ++i) len[i] = uint8_t(bits >> (56 - 8 * i));
        update(len, 8);
        static const char digits[] = "0123456789abcdef";
        std::string out;
        for (uint32_t w : h_)
            for (int i = 28; i >= 0; i -= 4) out.push_back(digits[(w >> i) & 15u]);
        return out;
    }

  private:
    static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
    void compress() {
        static const uint32_t k[64] = {
            0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
            0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
            0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
            0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
            0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
            0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
            0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
            0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
        uint32_t w[64];
        for (int i = 0; i < 16; ++i)
            w[i] = uint32_t(block_[4 * i]) << 24 | uint32_t(block_[4 * i + 1]) << 16 | uint32_t(block_[4 * i + 2]) << 8 |
                   uint32_t(block_[4 * i + 3]);
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h_[0], b = h_[1], c = h_[2], d = h_[3], e = h_[4], f = h_[5], g = h_[6], hh = h_[7];
        for (int i = 0; i < 64; ++i) {
            const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
            hh = g, g = f, f = e, e = d + t1, d = c, c = b, b = a, a = t1 + t2;
        }
        h_[0] += a, h_[1] += b, h_[2] += c, h_[3] += d, h_[4] += e, h_[5] += f, h_[6] += g, h_[7] += hh;
    }
    uint32_t h_[8];
    uint8_t block_[64];
    size_t fill_ = 0;
    uint64_t bits_ = 0;
};

std::string sha256_hex(const uint8_t* p, size_t n) {
    Sha256 s;
    s.update(p, n);
    return s.hex();
}

struct Failure {
    blitz_status status;
    std::string text;
};

void message(char* out, size_t n, const std::string& text) {
    if (out && n) {
        const size_t k = std::min(text.size(), n - 1);
        std::memcpy(out, text.data(), k);
        out[k] = 0;
    }
}

template <class F> blitz_status guarded(char* error, size_t cap, F f) {
    message(error, cap, "");
    try {
        f();
        return BLITZ_OK;
    } catch (const Failure& e) {
        message(error, cap, e.text);
        return e.status;
    } catch (const std::bad_alloc&) {
        message(error, cap, "allocation failed");
        return BLITZ_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        message(error, cap, e.what());
        return BLITZ_INTERNAL_ERROR;
    } catch (...) {
        message(error, cap, "unknown exception");
        return BLITZ_INTERNAL_ERROR;
    }
}

uint32_t le32(const std::vector<uint8_t>& d, size_t at) {
    return uint32_t(d[at]) | uint32_t(d[at + 1]) << 8 | uint32_t(d[at + 2]) << 16 | uint32_t(d[at + 3]) << 24;
}

// Weights of a policy network (placement.hpp:27-32 and internal.hpp:54-62):
// architecture 1 (graph encoder, width 64 only), 2 (action scorer, 80 -> 3),
// 3 and 4 (placement policies, 128 -> 12), hidden widths 64, 128 or 256.
size_t policy_weight_count(uint32_t architecture, uint32_t width) {
    if (architecture == 1) {
        if (width != 64) return 0;
        const uint32_t in[5] = {48, 128, 128, 72, 64}, out[5] = {64, 64, 64, 64, 4};
        size_t n = 0;
        for (int i = 0; i < 5; ++i) n += size_t(out[i]) * (in[i] + 1);
        return n;
    }
    uint32_t inputs = 0, outputs = 0;
    if (architecture == 2) inputs = 80, outputs = 3;
    if (architecture == 3 || architecture == 4) inputs = 128, outputs = 12;
    if (!inputs || (width != 64 && width != 128 && width != 256)) return 0;
    return size_t(width) * (inputs + 1) + size_t(width) * (width + 1) + size_t(outputs) * (width + 1);
}

} // namespace

struct blitz_neural_model {
    blitz_neural_options_v2 options{};
    uint32_t architecture = 0, width = 0, use = 0;
    std::string provenance, sha256;
    std::vector<float> weights;
};

namespace {

// Reads and checks a BLZNET01/02/03 file (model_io.cpp:59-107): magic,
// architecture, weight count, provenance length, width (02/03), use scope
// (03: endpoint reuse only, architecture 4), provenance, little-endian FP32
// weights (finite), and the lowercase hex SHA-256 of everything before it.
void load_policy(const char* path, blitz_neural_model& m) {
    if (!path || !path[0]) throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural model path"};
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw Failure{BLITZ_INVALID_ARGUMENT, std::string("cannot open neural model: ") + path};
    const std::streamoff size = f.tellg();
    const size_t largest = 92 + policy_weight_count(4, 256) * 4 + 65536;
    if (size < 84 || size_t(size) > largest) throw Failure{BLITZ_INVALID_ARGUMENT, "neural model size invalid"};
    std::vector<uint8_t> d(static_cast<size_t>(size));
    f.seekg(0);
    if (!f.read(reinterpret_cast<char*>(d.data()), size)) throw Failure{BLITZ_INVALID_ARGUMENT, "truncated neural model"};
    const bool v3 = !std::memcmp(d.data(), "BLZNET03", 8), v2 = !std::memcmp(d.data(), "BLZNET02", 8);
    const bool v1 = !std::memcmp(d.data(), "BLZNET01", 8);
    if (!v1 && !v2 && !v3) throw Failure{BLITZ_INVALID_ARGUMENT, "incompatible neural model schema/architecture"};
    const uint32_t architecture = le32(d, 8), count = le32(d, 12), provenance = le32(d, 16);
    const uint32_t width = (v2 || v3) ? le32(d, 20) : 64u;
    const size_t header = v3 ? 28 : (v2 ? 24 : 20);
    const uint32_t use = v3 ? le32(d, 24) : 0u;
    if (v3 && (use != 1 || architecture != 4))
        throw Failure{BLITZ_INVALID_ARGUMENT, "incompatible neural model use scope"};
    const size_t expected_count = policy_weight_count(architecture, width);
    if (!expected_count || count != expected_count)
        throw Failure{BLITZ_INVALID_ARGUMENT, "incompatible neural model schema/architecture"};
    if (provenance > 65536 || d.size() != header + provenance + size_t(count) * 4 + 64)
        throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural model payload"};
    const std::string sum = sha256_hex(d.data(), d.size() - 64);
    if (std::memcmp(sum.data(), d.data() + d.size() - 64, 64))
        throw Failure{BLITZ_INVALID_ARGUMENT, "neural model checksum mismatch"};
    m.architecture = architecture, m.width = width, m.use = use;
    m.provenance.assign(reinterpret_cast<const char*>(d.data() + header), provenance);
    m.weights.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t bits = le32(d, header + provenance + size_t(i) * 4);
        std::memcpy(&m.weights[i], &bits, 4);
        if (!std::isfinite(m.weights[i])) throw Failure{BLITZ_INVALID_ARGUMENT, "nonfinite model weights"};
    }
    m.sha256 = sha256_hex(d.data(), d.size());
}

// Option checks of NeuralModel (generate.cpp:18-55) that apply here.
void check_options(const blitz_neural_options_v2& o, const blitz_neural_model& m) {
    if (o.device < 0 || o.memory_mib < 128 || o.memory_mib > 65536 || !o.action_trials || o.action_trials > 65536 ||
        o.ranking > 4)
        throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural model options"};
    if (!o.action_batch || o.action_batch > 64) throw Failure{BLITZ_INVALID_ARGUMENT, "action batch outside 1..64"};
    if (o.exact_position_bps > 10000 || o.view_batch < 1 || o.view_batch > 4 ||
        (o.candidate_batch != 1 && o.candidate_batch != 2 && o.candidate_batch != 4 && o.candidate_batch != 8))
        throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural precision or audit batch"};
    if (o.confirmation > 2) throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural confirmation backend"};
    if (o.origin > 2) throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural proposal origin"};
    if (o.raster_backend > 1 || o.vertex_storage > 3)
        throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural raster or storage selection"};
    if (m.architecture == 1 && o.ranking != 0)
        throw Failure{BLITZ_INVALID_ARGUMENT, "action ranking controls require an action policy"};
    if (m.architecture == 1 && o.origin != 0)
        throw Failure{BLITZ_INVALID_ARGUMENT, "predecessor origins require an action policy"};
    if (!o.preserve_uv && m.architecture != 4)
        throw Failure{BLITZ_INVALID_ARGUMENT, "UV relaxation requires a UV-conditioned v4 policy"};
}

} // namespace

struct blitz_result {
    struct Level {
        std::vector<uint32_t> idx;
        std::vector<float> pos, uv;
        std::vector<uint16_t> mat;
        blitz_chain_level rec{};
        bool shared = true; // vertex positions are the source's (no referenced slot moved)
        uint64_t added_bytes = 0;
    };
    blitz_mesh source{};
    std::vector<Level> lods; // lods[0] = the source
    std::vector<size_t> runtime;
    uint64_t vertex_bytes = 0, source_vertex_bytes = 0;
    uint32_t max_added_bps = UINT32_MAX;
    blitz_neural_info info{};
    std::vector<blitz_neural_action_proposal> proposals;
};

namespace {

blitz_mesh exported(const blitz_result& r, size_t i) {
    const blitz_result::Level& l = r.lods[i];
    blitz_mesh m = r.source;
    if (i == 0) return m;
    if (!l.shared) m.positions = blitz_stream{l.pos.data(), l.pos.size() / 3, 12};
    if (!l.uv.empty()) m.uv = blitz_stream{l.uv.data(), l.uv.size() / 2, 8};
    m.indices = l.idx.data();
    m.index_count = l.idx.size();
    m.materials = l.mat.empty() ? nullptr : l.mat.data();
    m.material_count = l.mat.size();
    return m;
}

// Bytes one vertex takes in the source's streams (FP32 positions, normals,
// uv, tangents; RGBA8 colours).
uint64_t vertex_bytes(const blitz_mesh& m) {
    uint64_t b = 12;
    if (m.normals.data) b += 12;
    if (m.uv.data) b += 8;
    if (m.colors.data) b += 4;
    if (m.tangents.data) b += 16;
    return b;
}

struct EmitContext {
    blitz_result* result;
    blitz_audit_session* session;
    bool with_uv, with_mat;
    std::string error;
};

void on_level(void* user, uint32_t, const uint32_t* indices, uint32_t faces, const float* positions,
              uint32_t vertices) {
    EmitContext& c = *static_cast<EmitContext*>(user);
    try {
        blitz_result::Level l;
        l.idx.assign(indices, indices + size_t(faces) * 3);
        l.pos.assign(positions, positions + size_t(vertices) * 3);
        char err[256];
        if (c.with_uv) {
            l.uv.resize(size_t(vertices) * 2);
            if (blitz_audit_state_uv(c.session, l.uv.data(), l.uv.size(), err, sizeof err) != BLITZ_OK) c.error = err;
        }
        if (c.with_mat) {
            l.mat.resize(faces);
            uint32_t n = 0;
            if (blitz_audit_state_materials(c.session, l.mat.data(), l.mat.size(), &n, err, sizeof err) != BLITZ_OK)
                c.error = err;
        }
        c.result->lods.push_back(std::move(l));
    } catch (...) {
        c.error = "level copy failed";
    }
}

} // namespace

extern "C" {

blitz_status blitz_settings_init(blitz_settings* out, size_t n) {
    if (!out || n != sizeof(blitz_settings)) return BLITZ_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    out->struct_size = sizeof *out;
    out->abi_version = BLITZ_ABI_VERSION;
    // blitz::Settings defaults (remesher.hpp:31-56; ViewSet evaluate.hpp:8)
    out->levels = 8;
    out->profile = 1; // normals
    out->max_added_vertex_bytes_bps = 2000;
    out->beam_width = 8;
    out->candidate_budget = 64;
    out->search_supersample = 4, out->audit_supersample = 8, out->max_supersample = 32;
    out->search_ortho = 42, out->search_perspective = 12, out->search_seed = 0xB1172024u;
    out->audit_ortho = 642, out->audit_perspective = 64, out->audit_seed = 0xB1172026u;
    out->pixels_per_meter = 512, out->meters_per_unit = 1, out->last_pixels = 16;
    out->max_changed_area = 1.0;
    out->prune = 1, out->coupled_wedges = 1;
    return BLITZ_OK;
}

blitz_status blitz_generate(const blitz_mesh*, const blitz_settings*, blitz_result** out, char* error, size_t cap) {
    if (out) *out = nullptr;
    message(error, cap, "the classical reducer is not part of this engine; use blitz_generate_neural");
    return BLITZ_UNAVAILABLE;
}

blitz_status blitz_neural_options_init(blitz_neural_options* out, size_t n) {
    if (!out || n != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    *out = blitz_neural_options{sizeof(*out), 1, 0, 6144, 1, {0, 0, 0}};
    return BLITZ_OK;
}

blitz_status blitz_neural_model_load(const char* path, const blitz_neural_options* o, blitz_neural_model** out,
                                     char* error, size_t cap) {
    if (out) *out = nullptr;
    return guarded(error, cap, [&] {
        if (!out || !o || o->struct_size != sizeof(*o) || o->version != 1 || o->overdraw_tiebreak > 1 ||
            o->reserved[0] || o->reserved[1] || o->reserved[2])
            throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural descriptor"};
        auto m = std::make_unique<blitz_neural_model>();
        blitz_neural_options_v2_init(&m->options, sizeof m->options);
        m->options.device = o->device;
        m->options.memory_mib = o->memory_mib;
        m->options.overdraw_tiebreak = o->overdraw_tiebreak;
        load_policy(path, *m);
        check_options(m->options, *m);
        *out = m.release();
    });
}

blitz_status blitz_neural_model_load_v2(const char* path, const blitz_neural_options_v2* o, blitz_neural_model** out,
                                        char* error, size_t cap) {
    if (out) *out = nullptr;
    return guarded(error, cap, [&] {
        if (!out || !o || o->struct_size != sizeof(*o) || o->version != 2 || o->reserved[0] || o->reserved[1] ||
            o->reserved[2] || o->preserve_uv > 1 || o->overdraw_tiebreak > 1 || o->cache_rasters > 1 ||
            o->mask_only_coverage > 1 || o->direct_targets > 1)
            throw Failure{BLITZ_INVALID_ARGUMENT, "invalid neural v2 descriptor"};
        auto m = std::make_unique<blitz_neural_model>();
        m->options = *o;
        load_policy(path, *m);
        check_options(m->options, *m);
        *out = m.release();
    });
}

void blitz_neural_model_destroy(blitz_neural_model* m) { delete m; }

const char* blitz_neural_model_sha256(const blitz_neural_model* m) { return m ? m->sha256.c_str() : nullptr; }

blitz_status blitz_generate_neural(const blitz_mesh* mesh, const blitz_settings* c, const blitz_neural_model* model,
                                   blitz_result** out, char* error, size_t cap) {
    if (out) *out = nullptr;
    if (!model) {
        message(error, cap, "neural model is required");
        return BLITZ_INVALID_ARGUMENT;
    }
    bool cancelled = false;
    const blitz_status st = guarded(error, cap, [&] {
        if (!mesh || !c || !out || mesh->struct_size != sizeof(*mesh) || c->struct_size != sizeof(*c) ||
            mesh->abi_version != BLITZ_ABI_VERSION || c->abi_version != BLITZ_ABI_VERSION)
            throw Failure{BLITZ_INVALID_ARGUMENT, "null pointer, descriptor size or ABI version mismatch"};
        const blitz_neural_options_v2& o = model->options;
        if (c->profile != 0) throw Failure{BLITZ_UNAVAILABLE, "only the coverage profile is audited by this engine"};
        if (o.ranking == 0 || o.ranking == 2)
            throw Failure{BLITZ_UNAVAILABLE, "learned and shuffled rankings (policy network scores) are not built"};
        if (o.raster_backend != 0) throw Failure{BLITZ_UNAVAILABLE, "the Vulkan raster backend is not built"};
        if (c->cancelled && c->cancelled(c->user_data)) {
            cancelled = true;
            throw Failure{BLITZ_CANCELLED, "cancelled"};
        }
        // Chain settings (c_api.cpp:146-177, chain.cpp:101-118, 179-199).
        blitz_chain_settings cs;
        blitz_chain_settings_init(&cs);
        cs.levels = c->levels;
        cs.last_pixels = c->last_pixels;
        cs.max_lod0_delta_px = c->max_lod0_delta_px;
        if (c->base_pixels != 0) {
            cs.base_pixels = c->base_pixels;
        } else { // first = diameter x meters_per_unit x pixels_per_meter (chain.cpp:104)
            float center[3];
            double radius = 0;
            char err[256];
            if (blitz_mesh_bounds(mesh, center, &radius, err, sizeof err) != BLITZ_OK)
                throw Failure{BLITZ_INVALID_ARGUMENT, err};
            cs.base_pixels = 2 * radius * c->meters_per_unit * c->pixels_per_meter;
        }
        if (c->transition_count) {
            if (!c->transition) throw Failure{BLITZ_INVALID_ARGUMENT, "null transition curve"};
            if (c->transition_count > 8) throw Failure{BLITZ_INVALID_ARGUMENT, "more than 8 transition points"};
            for (size_t i = 0; i < c->transition_count; ++i)
                cs.transition_curve[2 * i] = c->transition[i].x, cs.transition_curve[2 * i + 1] = c->transition[i].y;
            cs.transition_points = uint32_t(c->transition_count);
        }
        cs.search_orthographic = c->search_ortho, cs.search_perspective = c->search_perspective;
        cs.search_seed = c->search_seed;
        cs.audit_orthographic = c->audit_ortho, cs.audit_perspective = c->audit_perspective;
        cs.audit_seed = c->audit_seed;
        cs.search_supersample = c->search_supersample, cs.audit_supersample = c->audit_supersample;
        cs.max_supersample = c->max_supersample;
        cs.max_changed_area = c->max_changed_area;
        cs.batch = o.action_batch;
        cs.trial_budget = o.action_trials;
        cs.min_faces = 1;
        cs.ranking = o.ranking; // 1 Constant, 3 ShortestEdge, 4 CurrentPlane
        char err[512];
        double p[32], t[32], b[32];
        if (blitz_chain_schedule(&cs, p, t, b, 32, err, sizeof err) != BLITZ_OK)
            throw Failure{BLITZ_INVALID_ARGUMENT, err};
        blitz_neural_options_v2 so = o;
        blitz_audit_session* session = nullptr;
        blitz_status s = blitz_audit_session_create(mesh, &so, &session, err, sizeof err);
        if (s != BLITZ_OK) throw Failure{s, err};
        std::unique_ptr<blitz_audit_session, void (*)(blitz_audit_session*)> hold(session, blitz_audit_session_destroy);
        auto r = std::make_unique<blitz_result>();
        r->source = *mesh;
        r->vertex_bytes = vertex_bytes(*mesh);
        r->source_vertex_bytes = r->vertex_bytes * mesh->positions.count;
        r->max_added_bps = c->max_added_vertex_bytes_bps;
        blitz_result::Level zero;
        zero.rec.pixels = p[0];
        zero.rec.confirmed = 1;
        zero.rec.faces = uint32_t(mesh->index_count / 3);
        zero.idx.assign(mesh->indices, mesh->indices + mesh->index_count);
        r->lods.push_back(std::move(zero));
        EmitContext ctx{r.get(), session, mesh->uv.data != nullptr, mesh->materials != nullptr, {}};
        std::vector<blitz_chain_level> levels(cs.levels - 1);
        s = blitz_audit_chain(session, &cs, levels.data(), levels.size(), on_level, &ctx, err, sizeof err);
        if (s != BLITZ_OK) throw Failure{s, err};
        if (!ctx.error.empty()) throw Failure{BLITZ_INTERNAL_ERROR, ctx.error};
        if (r->lods.size() != cs.levels) throw Failure{BLITZ_INTERNAL_ERROR, "chain emitted a wrong level count"};
        // Moved slots referenced by a level are new vertices.
        const uint8_t* src = static_cast<const uint8_t*>(mesh->positions.data);
        const size_t stride = mesh->positions.stride ? mesh->positions.stride : 12;
        uint32_t previous_faces = uint32_t(mesh->index_count / 3);
        uint64_t audit_ns = 0;
        for (size_t i = 1; i < r->lods.size(); ++i) {
            blitz_result::Level& l = r->lods[i];
            l.rec = levels[i - 1];
            std::vector<uint8_t> used(l.pos.size() / 3, 0);
            for (uint32_t v : l.idx) used[v] = 1;
            uint64_t moved = 0;
            for (size_t v = 0; v < used.size(); ++v)
                if (used[v] && std::memcmp(&l.pos[3 * v], src + v * stride, 12) != 0) ++moved;
            l.shared = moved == 0;
            l.added_bytes = moved * r->vertex_bytes;
            audit_ns += uint64_t(l.rec.seconds * 1e9);
            blitz_neural_action_proposal a{};
            a.struct_size = sizeof a, a.version = 1;
            a.start_triangles = previous_faces, a.target_triangles = cs.min_faces, a.final_triangles = l.rec.faces;
            a.trial_budget = cs.trial_budget, a.trials = l.rec.trials, a.accepted_batches = l.rec.commits;
            a.screen_pixels = l.rec.pixels;
            a.origin = i == 1 ? BLITZ_NEURAL_SOURCE : BLITZ_NEURAL_PREVIOUS;
            a.output = 0; // rebuilt: placed vertices
            a.stop_reason = l.rec.stop_reason;
            r->proposals.push_back(a);
            previous_faces = l.rec.faces;
        }
        // Runtime levels: consecutive identical levels share one (chain.cpp:16-24).
        for (size_t i = 0; i < r->lods.size(); ++i) {
            const blitz_result::Level &a = r->lods[i], *b = i ? &r->lods[i - 1] : nullptr;
            const bool same_vertices = b && (a.shared ? b->shared : (!b->shared && a.pos == b->pos));
            if (b && a.idx == b->idx && same_vertices) continue;
            r->runtime.push_back(i);
        }
        blitz_neural_info si{};
        si.struct_size = sizeof si;
        blitz_audit_session_info(session, &si);
        r->info = si;
        r->info.gpu_audit_ns = audit_ns;
        r->info.legal_collapses = 0;
        r->info.fallback_levels = 0;
        for (const blitz_chain_level& l : levels) {
            r->info.legal_collapses += l.commits;
            r->info.fallback_levels += l.confirmed ? 0u : 1u;
        }
        if (c->cancelled && c->cancelled(c->user_data)) cancelled = true;
        *out = r.release();
    });
    if (st == BLITZ_OK && cancelled) return BLITZ_CANCELLED;
    return st;
}

size_t blitz_result_lod_count(const blitz_result* r) { return r ? r->lods.size() : 0; }
size_t blitz_result_runtime_lod_count(const blitz_result* r) { return r ? r->runtime.size() : 0; }
size_t blitz_result_runtime_lod_index(const blitz_result* r, size_t i) {
    return r && i < r->runtime.size() ? r->runtime[i] : SIZE_MAX;
}

blitz_status blitz_result_lod(const blitz_result* r, size_t i, blitz_lod_info* out) {
    if (!r || !out || out->struct_size != sizeof(*out) || i >= r->lods.size()) return BLITZ_INVALID_ARGUMENT;
    const blitz_result::Level& l = r->lods[i];
    blitz_lod_info o{};
    o.struct_size = sizeof o;
    o.mesh = exported(*r, i);
    o.screen_pixels = l.rec.pixels;
    o.transition_limit = i ? l.rec.transition : 0;
    o.source_limit = i ? l.rec.source_bound : 0;
    o.transition_error = i ? l.rec.transition_audit.error : 0;
    o.source_error = i ? l.rec.source_audit.error : 0;
    o.transition_worst_view = i ? l.rec.transition_audit.worst_view : 0;
    o.source_worst_view = i ? l.rec.source_audit.worst_view : 0;
    o.shared_vertices = l.shared;
    o.passed = i ? l.rec.confirmed : 1;
    o.reference_triangles = l.rec.faces;
    o.transition_changed_area = i ? l.rec.transition_audit.changed_area : 0;
    o.source_changed_area = i ? l.rec.source_audit.changed_area : 0;
    o.transition_changed_area_worst_view = i ? l.rec.transition_audit.changed_area_worst_view : 0;
    o.source_changed_area_worst_view = i ? l.rec.source_audit.changed_area_worst_view : 0;
    *out = o;
    return BLITZ_OK;
}

blitz_status blitz_result_storage(const blitz_result* r, blitz_storage_info* out) {
    if (!r || !out || out->struct_size != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    uint64_t added = 0, index = 0;
    for (size_t i : r->runtime) {
        added += r->lods[i].added_bytes;
        index += r->lods[i].idx.size() * 4;
    }
    blitz_storage_info o{};
    o.struct_size = sizeof o;
    o.source_vertex_bytes = r->source_vertex_bytes;
    o.added_vertex_bytes = added;
    o.index_bytes = index;
    o.total_bytes = r->source_vertex_bytes + added + index;
    o.max_added_vertex_bytes_bps = r->max_added_bps;
    o.added_vertex_budget_bytes =
        r->max_added_bps == UINT32_MAX ? UINT64_MAX : r->source_vertex_bytes * r->max_added_bps / 10000;
    *out = o;
    return BLITZ_OK;
}

blitz_status blitz_result_runtime_lod_storage(const blitz_result* r, size_t i, blitz_runtime_lod_storage_info* out) {
    if (!r || !out || out->struct_size != sizeof(*out) || i >= r->runtime.size()) return BLITZ_INVALID_ARGUMENT;
    uint64_t cumulative = 0;
    for (size_t k = 0; k <= i; ++k) cumulative += r->lods[r->runtime[k]].added_bytes;
    const size_t s = r->runtime[i];
    blitz_runtime_lod_storage_info o{};
    o.struct_size = sizeof o;
    o.scheduled_index = uint8_t(s);
    o.added_vertex_bytes = r->lods[s].added_bytes;
    o.index_bytes = r->lods[s].idx.size() * 4;
    o.cumulative_added_vertex_bytes = cumulative;
    *out = o;
    return BLITZ_OK;
}

void blitz_result_destroy(blitz_result* r) { delete r; }

blitz_status blitz_result_neural_info(const blitz_result* r, blitz_neural_info* out) {
    if (!r || !out || out->struct_size != sizeof(*out)) return BLITZ_INVALID_ARGUMENT;
    *out = r->info;
    out->struct_size = sizeof(*out);
    return BLITZ_OK;
}

size_t blitz_result_neural_action_proposal_count(const blitz_result* r) { return r ? r->proposals.size() : 0; }

blitz_status blitz_result_neural_action_proposal(const blitz_result* r, size_t i, blitz_neural_action_proposal* out) {
    if (!r || !out || out->struct_size != sizeof(*out) || out->version != 1 || i >= r->proposals.size())
        return BLITZ_INVALID_ARGUMENT;
    *out = r->proposals[i];
    return BLITZ_OK;
}

} // extern "C"
