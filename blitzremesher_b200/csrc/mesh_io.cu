// Mesh files in and LOD chains out (host code): OBJ, PLY and STL import into
// blitz_mesh descriptors, PLY export of a mesh, and a chain's export as one
// glTF 2.0 scene (chain.gltf + chain.bin) with a lods.json manifest.
//
// The readers follow the reference's import rules (src/io.cpp:118-229): OBJ
// corners deduplicated by their (position, normal, uv) index triple,
// polygons fanned into triangles, material ids 1 + the material's place in the
// OBJ's material library (0 without one), non-opaque materials refused;
// PLY ascii and binary in either byte order with x/y/z, nx/ny/nz, u/v (or
// s/t), red/green/blue/alpha and a per-face material_index, faces triangles
// only; STL binary when its size is 84 + 50 x count bytes, else ascii, corners
// welded on exact position bits; a 1 GiB input cap and the reference's mesh
// validation (mesh.cpp:27-41). glTF import is not built. The chain export
// follows save_chain (io.cpp:298-359): one glTF mesh per runtime level with
// one primitive per material, one node per scheduled level, and a manifest
// of the levels, their limits, audits and storage.
#include "../../include/blitz_audit.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace fs = std::filesystem;

struct blitz_mesh_file {
    std::vector<float> positions, normals, uv, tangents;
    std::vector<blitz_color_rgba8> colors;
    std::vector<uint32_t> indices;
    std::vector<uint16_t> materials;
};

namespace {

struct Failure {
    blitz_status status;
    std::string text;
};
[[noreturn]] void fail(const std::string& text) { throw Failure{BLITZ_INVALID_ARGUMENT, text}; }

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
    }
}

// Linear RGBA8 channel of a value in [0, 1] (mesh.cpp:5-11).
uint8_t color_channel(double v) {
    if (!std::isfinite(v) || v < 0 || v > 1) fail("color channels must be finite and in [0,1]");
    return uint8_t(std::floor(v * 255 + .5));
}

std::string lower(std::string s) {
    for (char& c : s) c = char(std::tolower(static_cast<unsigned char>(c)));
    return s;
}

// ---- OBJ ----
struct ObjLibrary {
    std::vector<std::string> names;
};
ObjLibrary read_mtl(const fs::path& path) {
    ObjLibrary lib;
    std::ifstream f(path);
    if (!f) return lib; // a missing library leaves the ids at their first-use order
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream s(line);
        std::string word;
        s >> word;
        if (word == "newmtl") {
            std::string name;
            s >> name;
            lib.names.push_back(name);
        } else if (word == "d") {
            double d = 1;
            if (s >> d && d < 1) fail("nonopaque OBJ material");
        } else if (word == "Tr") {
            double t = 0;
            if (s >> t && t > 0) fail("nonopaque OBJ material");
        } else if (word == "map_d") {
            fail("nonopaque OBJ material");
        }
    }
    return lib;
}

void read_obj(const fs::path& path, blitz_mesh_file& m) {
    std::ifstream f(path);
    if (!f) fail("cannot open OBJ: " + path.string());
    std::vector<float> v, vn, vt, vc;
    bool colors = false, normals = false, uv = false;
    struct Key {
        long long v, n, t;
        bool operator==(const Key& o) const { return v == o.v && n == o.n && t == o.t; }
    };
    struct Hash {
        size_t operator()(const Key& k) const {
            return size_t(k.v) * 73856093u ^ size_t(k.n) * 19349663u ^ size_t(k.t) * 83492791u;
        }
    };
    std::unordered_map<Key, uint32_t, Hash> corners;
    std::vector<std::string> library, used;
    int material = 0;
    std::string line;
    auto resolve = [](long long i, size_t count) -> long long {
        if (i > 0) return i - 1;
        if (i < 0) return (long long)count + i;
        fail("invalid OBJ index 0");
    };
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream s(line);
        std::string word;
        if (!(s >> word) || word[0] == '#') continue;
        if (word == "v") {
            double x, y, z;
            if (!(s >> x >> y >> z)) fail("invalid OBJ vertex");
            v.insert(v.end(), {float(x), float(y), float(z)});
            double r, g, b;
            if (s >> r >> g >> b) {
                vc.insert(vc.end(), {float(r), float(g), float(b)});
                colors = true;
            } else {
                vc.insert(vc.end(), {1.f, 1.f, 1.f});
            }
        } else if (word == "vn") {
            double x, y, z;
            if (!(s >> x >> y >> z)) fail("invalid OBJ normal");
            vn.insert(vn.end(), {float(x), float(y), float(z)});
        } else if (word == "vt") {
            double x, y = 0;
            if (!(s >> x)) fail("invalid OBJ uv");
            s >> y;
            vt.insert(vt.end(), {float(x), float(y)});
        } else if (word == "mtllib") {
            std::string name;
            s >> name;
            for (auto& n : read_mtl(path.parent_path() / name).names) library.push_back(n);
        } else if (word == "usemtl") {
            std::string name;
            s >> name;
            auto it = std::find(library.begin(), library.end(), name);
            if (it != library.end()) {
                material = int(it - library.begin()) + 1;
            } else {
                auto u = std::find(used.begin(), used.end(), name);
                if (u == used.end()) used.push_back(name), u = used.end() - 1;
                material = int(library.size() + (u - used.begin())) + 1;
            }
            if (material >= 65535) fail("too many OBJ materials");
        } else if (word == "f") {
            std::vector<uint32_t> poly;
            std::string corner;
            while (s >> corner) {
                long long ids[3] = {0, 0, 0};
                bool has[3] = {false, false, false};
                size_t at = 0;
                for (int k = 0; k < 3 && at <= corner.size(); ++k) {
                    const size_t slash = corner.find('/', at);
                    const std::string part = corner.substr(at, slash == std::string::npos ? std::string::npos : slash - at);
                    if (!part.empty()) ids[k] = std::stoll(part), has[k] = true;
                    if (slash == std::string::npos) break;
                    at = slash + 1;
                }
                if (!has[0]) fail("invalid OBJ face corner");
                const Key key{resolve(ids[0], v.size() / 3), has[2] ? resolve(ids[2], vn.size() / 3) : -1,
                              has[1] ? resolve(ids[1], vt.size() / 2) : -1};
                auto [it, inserted] = corners.emplace(key, uint32_t(m.positions.size() / 3));
                if (inserted) {
                    if (key.v < 0 || size_t(key.v) * 3 + 2 >= v.size()) fail("invalid OBJ position index");
                    if (key.n >= 0 && size_t(key.n) * 3 + 2 >= vn.size()) fail("invalid OBJ normal index");
                    if (key.t >= 0 && size_t(key.t) * 2 + 1 >= vt.size()) fail("invalid OBJ UV index");
                    m.positions.insert(m.positions.end(), &v[3 * key.v], &v[3 * key.v] + 3);
                    if (key.n >= 0) m.normals.insert(m.normals.end(), &vn[3 * key.n], &vn[3 * key.n] + 3);
                    else m.normals.insert(m.normals.end(), {0.f, 0.f, 0.f});
                    if (key.t >= 0) m.uv.insert(m.uv.end(), &vt[2 * key.t], &vt[2 * key.t] + 2);
                    else m.uv.insert(m.uv.end(), {0.f, 0.f});
                    m.colors.push_back(blitz_color_rgba8{color_channel(vc[3 * key.v]), color_channel(vc[3 * key.v + 1]),
                                                         color_channel(vc[3 * key.v + 2]), 255});
                    normals |= key.n >= 0;
                    uv |= key.t >= 0;
                }
                poly.push_back(it->second);
            }
            if (poly.size() < 3) fail("OBJ face with fewer than three corners");
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                m.indices.insert(m.indices.end(), {poly[0], poly[k], poly[k + 1]});
                m.materials.push_back(uint16_t(material));
            }
        }
    }
    if (!normals) m.normals.clear();
    if (!uv) m.uv.clear();
    if (!colors) m.colors.clear();
}

// ---- PLY ----
void read_ply(const fs::path& path, blitz_mesh_file& m) {
    std::ifstream f(path, std::ios::binary);
    if (!f) fail("cannot open PLY: " + path.string());
    std::string line;
    std::getline(f, line);
    if (line != "ply" && line != "ply\r") fail("invalid PLY magic");
    struct Prop {
        std::string name, type, count;
    };
    struct Element {
        std::string name;
        size_t count = 0;
        std::vector<Prop> props;
    };
    std::vector<Element> elements;
    bool ascii = true, big = false, ended = false;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream s(line);
        std::string word;
        s >> word;
        if (word == "end_header") {
            ended = true;
            break;
        }
        if (word == "format") {
            s >> word;
            if (word == "binary_little_endian") ascii = false;
            else if (word == "binary_big_endian") ascii = false, big = true;
            else if (word != "ascii") fail("unknown PLY format");
        } else if (word == "element") {
            Element e;
            s >> e.name >> e.count;
            if (!s || e.count >= UINT32_MAX) fail("oversized PLY element");
            elements.push_back(e);
        } else if (word == "property") {
            if (elements.empty()) fail("PLY property without element");
            Prop p;
            s >> p.type;
            if (p.type == "list") s >> p.count >> p.type;
            s >> p.name;
            elements.back().props.push_back(p);
        }
    }
    if (!ended) fail("missing PLY end_header");
    auto scalar = [&](const std::string& type) -> double {
        if (ascii) {
            double v;
            if (!(f >> v) || !std::isfinite(v)) fail("bad PLY value");
            return v;
        }
        auto take = [&](size_t n, uint8_t* out) {
            if (!f.read(reinterpret_cast<char*>(out), std::streamsize(n))) fail("truncated PLY");
            if (big) std::reverse(out, out + n);
        };
        uint8_t b[8];
        if (type == "float" || type == "float32") { float v; take(4, b); std::memcpy(&v, b, 4); return v; }
        if (type == "double" || type == "float64") { double v; take(8, b); std::memcpy(&v, b, 8); return v; }
        if (type == "uchar" || type == "uint8") { take(1, b); return b[0]; }
        if (type == "char" || type == "int8") { take(1, b); return int8_t(b[0]); }
        if (type == "ushort" || type == "uint16") { uint16_t v; take(2, b); std::memcpy(&v, b, 2); return v; }
        if (type == "short" || type == "int16") { int16_t v; take(2, b); std::memcpy(&v, b, 2); return v; }
        if (type == "uint" || type == "uint32") { uint32_t v; take(4, b); std::memcpy(&v, b, 4); return v; }
        if (type == "int" || type == "int32") { int32_t v; take(4, b); std::memcpy(&v, b, 4); return v; }
        fail("unknown PLY scalar type");
    };
    bool normals = false, uv = false, colors = false;
    for (const Element& e : elements)
        for (size_t i = 0; i < e.count; ++i) {
            float p[3] = {0, 0, 0}, n[3] = {0, 0, 0}, t[2] = {0, 0};
            blitz_color_rgba8 c{255, 255, 255, 255};
            uint16_t mat = 0;
            for (const Prop& prop : e.props) {
                if (!prop.count.empty()) {
                    const double raw = scalar(prop.count);
                    if (raw < 0 || raw > 1000000 || std::floor(raw) != raw) fail("bad PLY list length");
                    const bool corners = e.name == "face" && (prop.name == "vertex_indices" || prop.name == "vertex_index");
                    if (corners && raw != 3) fail("PLY requires triangulated faces");
                    for (size_t k = 0; k < size_t(raw); ++k) {
                        const double v = scalar(prop.type);
                        if (!corners) continue;
                        if (v < 0 || v >= double(UINT32_MAX) || std::floor(v) != v) fail("bad PLY index");
                        m.indices.push_back(uint32_t(v));
                    }
                    continue;
                }
                const double v = scalar(prop.type);
                const std::string& nm = prop.name;
                if (e.name == "vertex") {
                    if (nm == "x") p[0] = float(v);
                    if (nm == "y") p[1] = float(v);
                    if (nm == "z") p[2] = float(v);
                    if (nm == "nx") n[0] = float(v), normals = true;
                    if (nm == "ny") n[1] = float(v);
                    if (nm == "nz") n[2] = float(v);
                    if (nm == "u" || nm == "s") t[0] = float(v), uv = true;
                    if (nm == "v" || nm == "t") t[1] = float(v);
                    if (nm == "red" || nm == "green" || nm == "blue" || nm == "alpha") {
                        const double top = (prop.type == "uchar" || prop.type == "uint8")     ? 255
                                           : (prop.type == "ushort" || prop.type == "uint16") ? 65535
                                                                                              : 1;
                        if (top != 1 && std::floor(v) != v) fail("nonintegral PLY integer color");
                        const uint8_t ch = color_channel(v / top);
                        if (nm == "red") c.r = ch;
                        if (nm == "green") c.g = ch;
                        if (nm == "blue") c.b = ch;
                        if (nm == "alpha") c.a = ch;
                        colors = true;
                    }
                } else if (e.name == "face" && nm == "material_index") {
                    if (v < 0 || v > 65535 || std::floor(v) != v) fail("invalid material index");
                    mat = uint16_t(v);
                }
            }
            if (e.name == "vertex") {
                m.positions.insert(m.positions.end(), p, p + 3);
                m.normals.insert(m.normals.end(), n, n + 3);
                m.uv.insert(m.uv.end(), t, t + 2);
                m.colors.push_back(c);
            }
            if (e.name == "face") m.materials.push_back(mat);
        }
    if (!normals) m.normals.clear();
    if (!uv) m.uv.clear();
    if (!colors) m.colors.clear();
}

// ---- STL ----
void read_stl(const fs::path& path, blitz_mesh_file& m) {
    std::ifstream f(path, std::ios::binary);
    if (!f) fail("cannot open STL: " + path.string());
    const uint64_t bytes = fs::file_size(path);
    uint32_t count = 0;
    if (bytes >= 84) {
        f.seekg(80);
        f.read(reinterpret_cast<char*>(&count), 4);
    }
    const bool binary = bytes >= 84 && bytes == 84ull + 50ull * count;
    std::unordered_map<std::string, uint32_t> welded;
    auto add = [&](const float* p) {
        const std::string key(reinterpret_cast<const char*>(p), 12);
        auto [it, inserted] = welded.emplace(key, uint32_t(m.positions.size() / 3));
        if (inserted) m.positions.insert(m.positions.end(), p, p + 3);
        m.indices.push_back(it->second);
    };
    if (binary) {
        for (uint32_t i = 0; i < count; ++i) {
            float rec[12];
            uint16_t attribute;
            if (!f.read(reinterpret_cast<char*>(rec), 48) || !f.read(reinterpret_cast<char*>(&attribute), 2))
                fail("truncated STL");
            for (int j = 0; j < 3; ++j) add(rec + 3 + 3 * j);
        }
    } else {
        f.clear();
        f.seekg(0);
        std::string word;
        while (f >> word)
            if (word == "vertex") {
                float p[3];
                if (!(f >> p[0] >> p[1] >> p[2])) fail("invalid ASCII STL");
                add(p);
            }
    }
}

// The reference's mesh validation (mesh.cpp:27-41).
void validate(const blitz_mesh_file& m) {
    const size_t n = m.positions.size() / 3;
    if (!n || n >= UINT32_MAX || m.indices.empty() || m.indices.size() % 3 || m.indices.size() >= UINT32_MAX)
        fail("mesh requires nonempty triangle indices and 32-bit representable counts");
    if (!m.materials.empty() && m.materials.size() != m.indices.size() / 3)
        fail("material count differs from triangle count");
    for (uint32_t i : m.indices)
        if (i >= n) fail("index outside vertex stream");
    for (float x : m.positions)
        if (!std::isfinite(x)) fail("nonfinite position or normal");
    for (float x : m.normals)
        if (!std::isfinite(x)) fail("nonfinite position or normal");
    for (float x : m.uv)
        if (!std::isfinite(x)) fail("nonfinite UV");
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) lo[k] = hi[k] = m.positions[k];
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], double(m.positions[3 * i + k])),
                                    hi[k] = std::max(hi[k], double(m.positions[3 * i + k]));
    if (!(hi[0] > lo[0] || hi[1] > lo[1] || hi[2] > lo[2])) fail("zero or invalid source extent");
}

blitz_mesh describe(const blitz_mesh_file& m) {
    blitz_mesh d{};
    d.struct_size = sizeof d;
    d.abi_version = BLITZ_ABI_VERSION;
    const size_t n = m.positions.size() / 3;
    d.positions = blitz_stream{m.positions.data(), n, 12};
    if (!m.normals.empty()) d.normals = blitz_stream{m.normals.data(), n, 12};
    if (!m.uv.empty()) d.uv = blitz_stream{m.uv.data(), n, 8};
    if (!m.colors.empty()) d.colors = blitz_stream{m.colors.data(), n, 4};
    if (!m.tangents.empty()) d.tangents = blitz_stream{m.tangents.data(), n, 16};
    d.indices = m.indices.data();
    d.index_count = m.indices.size();
    if (!m.materials.empty()) d.materials = m.materials.data(), d.material_count = m.materials.size();
    return d;
}

template <class T> const T* element(const blitz_stream& s, size_t i) {
    return reinterpret_cast<const T*>(static_cast<const uint8_t*>(s.data) + i * (s.stride ? s.stride : sizeof(T)));
}

template <class T> void put(std::vector<uint8_t>& out, const T& v) {
    const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
    out.insert(out.end(), p, p + sizeof(T));
}

std::string number(double v) {
    if (!std::isfinite(v)) return "null";
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return buf;
}

} // namespace

extern "C" {

blitz_status blitz_mesh_file_load(const char* path, blitz_mesh_file** out, blitz_mesh* mesh, char* error,
                                  size_t cap) {
    if (out) *out = nullptr;
    return guarded(error, cap, [&] {
        if (!path || !out || !mesh) fail("null argument");
        const fs::path p(path);
        std::error_code ec;
        const uint64_t size = fs::file_size(p, ec);
        if (ec) fail("cannot open mesh file: " + p.string());
        if (size > (1ull << 30)) fail("input exceeds 1 GiB import cap");
        const std::string ext = lower(p.extension().string());
        auto m = std::make_unique<blitz_mesh_file>();
        if (ext == ".obj") read_obj(p, *m);
        else if (ext == ".ply") read_ply(p, *m);
        else if (ext == ".stl") read_stl(p, *m);
        else if (ext == ".gltf" || ext == ".glb") throw Failure{BLITZ_UNAVAILABLE, "glTF import is not built"};
        else fail("unsupported mesh extension");
        try {
            validate(*m);
        } catch (const Failure& e) {
            fail(p.string() + ": " + e.text);
        }
        *mesh = describe(*m);
        *out = m.release();
    });
}

void blitz_mesh_file_destroy(blitz_mesh_file* m) { delete m; }

blitz_status blitz_mesh_save_ply(const blitz_mesh* m, const char* path, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!m || !path || m->struct_size != sizeof(*m) || !m->positions.data || !m->indices || m->index_count % 3)
            fail("invalid mesh or path");
        const size_t n = m->positions.count, faces = m->index_count / 3;
        std::ofstream f(path, std::ios::binary);
        if (!f) fail(std::string("cannot write PLY: ") + path);
        f << "ply\nformat binary_little_endian 1.0\nelement vertex " << n
          << "\nproperty float x\nproperty float y\nproperty float z\n";
        if (m->normals.data) f << "property float nx\nproperty float ny\nproperty float nz\n";
        if (m->uv.data) f << "property float u\nproperty float v\n";
        if (m->colors.data) f << "property uchar red\nproperty uchar green\nproperty uchar blue\nproperty uchar alpha\n";
        f << "element face " << faces << "\nproperty list uchar uint vertex_indices\nproperty ushort material_index\n"
          << "end_header\n";
        std::vector<uint8_t> row;
        for (size_t i = 0; i < n; ++i) {
            row.clear();
            for (int k = 0; k < 3; ++k) put(row, element<float>(m->positions, i)[k]);
            if (m->normals.data)
                for (int k = 0; k < 3; ++k) put(row, element<float>(m->normals, i)[k]);
            if (m->uv.data)
                for (int k = 0; k < 2; ++k) put(row, element<float>(m->uv, i)[k]);
            if (m->colors.data) put(row, *element<blitz_color_rgba8>(m->colors, i));
            f.write(reinterpret_cast<const char*>(row.data()), std::streamsize(row.size()));
        }
        for (size_t t = 0; t < faces; ++t) {
            row.clear();
            put(row, uint8_t(3));
            for (int k = 0; k < 3; ++k) put(row, m->indices[3 * t + k]);
            put(row, uint16_t(m->materials ? m->materials[t] : 0));
            f.write(reinterpret_cast<const char*>(row.data()), std::streamsize(row.size()));
        }
        if (!f) fail(std::string("cannot write PLY: ") + path);
    });
}

blitz_status blitz_result_save_chain(const blitz_result* r, const char* directory, char* error, size_t cap) {
    return guarded(error, cap, [&] {
        if (!r || !directory) fail("null argument");
        const size_t levels = blitz_result_lod_count(r), runtime_count = blitz_result_runtime_lod_count(r);
        if (!levels || !runtime_count) fail("empty result");
        std::vector<blitz_lod_info> info(levels);
        for (size_t i = 0; i < levels; ++i) {
            info[i].struct_size = sizeof(blitz_lod_info);
            if (blitz_result_lod(r, i, &info[i]) != BLITZ_OK) fail("result level query failed");
        }
        std::vector<size_t> runtime(runtime_count);
        for (size_t i = 0; i < runtime_count; ++i) runtime[i] = blitz_result_runtime_lod_index(r, i);
        std::vector<uint8_t> bin;
        std::ostringstream views, accessors, meshes, nodes, materials;
        size_t nviews = 0, naccessors = 0;
        auto accessor = [&](size_t offset, size_t count, int components, int type, const char* shape,
                            const std::string& extra) {
            if (nviews) views << ",";
            views << "{\"buffer\":0,\"byteOffset\":" << offset << ",\"byteLength\":"
                  << count * components * (type == 5121 ? 1 : 4) << "}";
            if (naccessors) accessors << ",";
            accessors << "{\"bufferView\":" << nviews << ",\"componentType\":" << type << ",\"count\":" << count
                      << ",\"type\":\"" << shape << "\"" << extra << "}";
            ++nviews;
            return naccessors++;
        };
        // Vertex attributes of one level's mesh descriptor: a JSON attribute map.
        auto attributes = [&](const blitz_mesh& m) {
            std::ostringstream a;
            const size_t n = m.positions.count;
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            size_t start = bin.size();
            for (size_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) {
                    const float v = element<float>(m.positions, i)[k];
                    put(bin, v);
                    lo[k] = std::min(lo[k], double(v)), hi[k] = std::max(hi[k], double(v));
                }
            std::string bounds = ",\"min\":[" + number(lo[0]) + "," + number(lo[1]) + "," + number(lo[2]) +
                                 "],\"max\":[" + number(hi[0]) + "," + number(hi[1]) + "," + number(hi[2]) + "]";
            a << "{\"POSITION\":" << accessor(start, n, 3, 5126, "VEC3", bounds);
            auto floats = [&](const blitz_stream& s, int k, const char* name, const char* shape) {
                if (!s.data) return;
                const size_t at = bin.size();
                for (size_t i = 0; i < n; ++i)
                    for (int c = 0; c < k; ++c) put(bin, element<float>(s, i)[c]);
                a << ",\"" << name << "\":" << accessor(at, n, k, 5126, shape, "");
            };
            floats(m.normals, 3, "NORMAL", "VEC3");
            floats(m.uv, 2, "TEXCOORD_0", "VEC2");
            if (m.colors.data) {
                const size_t at = bin.size();
                for (size_t i = 0; i < n; ++i) put(bin, *element<blitz_color_rgba8>(m.colors, i));
                a << ",\"COLOR_0\":" << accessor(at, n, 4, 5121, "VEC4", ",\"normalized\":true");
            }
            floats(m.tangents, 4, "TANGENT", "VEC4");
            a << "}";
            return a.str();
        };
        uint16_t top = 0;
        for (size_t i : runtime) {
            const blitz_mesh& m = info[i].mesh;
            for (size_t t = 0; m.materials && t < m.index_count / 3; ++t) top = std::max(top, m.materials[t]);
        }
        const blitz_mesh& source = info[0].mesh;
        for (unsigned i = 0; i <= top; ++i) {
            const bool two = i < source.double_sided_count && source.double_sided && source.double_sided[i];
            materials << (i ? "," : "") << "{\"name\":\"material_" << i << "\",\"doubleSided\":"
                      << (two ? "true" : "false") << "}";
        }
        const std::string shared = attributes(source);
        for (size_t k = 0; k < runtime.size(); ++k) {
            const blitz_mesh& m = info[runtime[k]].mesh;
            const std::string a = info[runtime[k]].shared_vertices ? shared : attributes(m);
            std::map<uint16_t, std::vector<uint32_t>> groups;
            for (size_t t = 0; t < m.index_count / 3; ++t)
                for (int c = 0; c < 3; ++c) groups[m.materials ? m.materials[t] : 0].push_back(m.indices[3 * t + c]);
            meshes << (k ? "," : "") << "{\"name\":\"LOD" << runtime[k] << "\",\"primitives\":[";
            bool first = true;
            for (auto& [mat, ids] : groups) {
                const size_t at = bin.size();
                for (uint32_t i : ids) put(bin, i);
                meshes << (first ? "" : ",") << "{\"attributes\":" << a << ",\"indices\":"
                       << accessor(at, ids.size(), 1, 5125, "SCALAR", "") << ",\"material\":" << mat << ",\"mode\":4}";
                first = false;
            }
            meshes << "]}";
        }
        std::vector<size_t> mesh_of(levels, 0);
        for (size_t i = 0, k = 0; i < levels; ++i) {
            if (k + 1 < runtime.size() && i == runtime[k + 1]) ++k;
            mesh_of[i] = k;
            nodes << (i ? "," : "") << "{\"mesh\":" << k << ",\"name\":\"LOD" << i << "\"}";
        }
        const fs::path dir(directory);
        fs::create_directories(dir);
        {
            std::ofstream b(dir / "chain.bin", std::ios::binary);
            b.write(reinterpret_cast<const char*>(bin.data()), std::streamsize(bin.size()));
            if (!b) fail("cannot write glTF buffer");
        }
        std::ostringstream g;
        g << "{\"asset\":{\"version\":\"2.0\",\"generator\":\"blitzremesher_b200\"},\"scene\":0,"
          << "\"scenes\":[{\"nodes\":[0]}],\"nodes\":[" << nodes.str() << "],\"meshes\":[" << meshes.str()
          << "],\"accessors\":[" << accessors.str() << "],\"bufferViews\":[" << views.str() << "],\"materials\":["
          << materials.str() << "],\"buffers\":[{\"uri\":\"chain.bin\",\"byteLength\":" << bin.size() << "}]}\n";
        std::ofstream(dir / "chain.gltf") << g.str();
        // Manifest: levels with their limits and audits, runtime meshes, storage.
        blitz_storage_info st{};
        st.struct_size = sizeof st;
        blitz_result_storage(r, &st);
        std::ostringstream j;
        j << "{\"version\":3,\"gltf\":\"chain.gltf\",\"storage\":{\"source_vertex_bytes\":" << st.source_vertex_bytes
          << ",\"added_vertex_bytes\":" << st.added_vertex_bytes << ",\"index_bytes\":" << st.index_bytes
          << ",\"total_bytes\":" << st.total_bytes << "},\"runtime_levels\":[";
        for (size_t k = 0; k < runtime.size(); ++k) j << (k ? "," : "") << runtime[k];
        j << "],\"runtime_lod_count\":" << runtime.size() << ",\"lods\":[";
        for (size_t i = 0; i < levels; ++i) {
            const blitz_lod_info& l = info[i];
            j << (i ? "," : "") << "{\"triangles\":" << l.mesh.index_count / 3 << ",\"vertices\":"
              << l.mesh.positions.count << ",\"reference_triangles\":" << l.reference_triangles
              << ",\"shared_vertices\":" << (l.shared_vertices ? "true" : "false")
              << ",\"screen_pixels\":" << number(l.screen_pixels) << ",\"transition_limit\":"
              << number(l.transition_limit) << ",\"source_limit\":" << number(l.source_limit)
              << ",\"adjacent\":{\"error_px\":" << number(l.transition_error) << ",\"worst_view\":"
              << l.transition_worst_view << ",\"changed_area\":" << number(l.transition_changed_area)
              << ",\"changed_area_worst_view\":" << l.transition_changed_area_worst_view
              << "},\"source\":{\"error_px\":" << number(l.source_error) << ",\"worst_view\":" << l.source_worst_view
              << ",\"changed_area\":" << number(l.source_changed_area) << ",\"changed_area_worst_view\":"
              << l.source_changed_area_worst_view << "},\"passed\":" << (l.passed ? "true" : "false")
              << ",\"gltf_mesh\":" << mesh_of[i] << ",\"gltf_node\":" << i << "}";
        }
        j << "],\"material_binding\":\"primitive.material is the input material ID\"}\n";
        std::ofstream(dir / "lods.json") << j.str();
    });
}

} // extern "C"
