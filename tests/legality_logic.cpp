// CPU check of the collapse-legality code the CUDA library runs
// (csrc/legality.cuh, compiled here for the host). A host build of the class
// topology with the layout the library's topology kernels produce (classes
// by position welding, ascending per-corner face lists, sorted unique
// neighbour rows with face counts, boundary and invalid flags, the single-fan
// rule) feeds single_fan and collapse_legal; the legal edits come out in the
// library's enumeration order (edges a < b ascending, a -> b then b -> a).
//
// Exported for ctypes:
//   int64_t legality_actions(const float* pos, uint32_t nv, const uint32_t* idx, uint32_t nf,
//                            const uint16_t* mat, uint32_t* out /* 7 words per edit */, uint64_t cap)
// Each edit: from, to, source0, source1, target0, target1, wedges | removed << 8.
#include "../blitzremesher_b200/csrc/legality.cuh"

#include <algorithm>
#include <cstring>
#include <unordered_map>
#include <vector>

using namespace b200;

namespace {
struct Key {
    uint32_t x, y, z;
    bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct KeyHash {
    size_t operator()(const Key& k) const { return hash_position(k.x, k.y, k.z); }
};
} // namespace

extern "C" int64_t legality_actions(const float* pos, uint32_t nv, const uint32_t* idx, uint32_t nf,
                                    const uint16_t* mat, uint32_t* out, uint64_t cap) {
    std::vector<uint32_t> geometry(nv);
    std::unordered_map<Key, uint32_t, KeyHash> first;
    for (uint32_t i = 0; i < nv; ++i) {
        const Key k{position_bits(pos[3 * i]), position_bits(pos[3 * i + 1]), position_bits(pos[3 * i + 2])};
        auto it = first.emplace(k, i).first;
        geometry[i] = it->second;
    }
    std::vector<std::vector<uint32_t>> faces_of(nv), entries(nv);
    std::vector<uint8_t> invalid(nv, 0), boundary(nv, 0);
    for (uint32_t f = 0; f < nf; ++f)
        for (int j = 0; j < 3; ++j) faces_of[geometry[idx[3 * f + j]]].push_back(f);
    for (uint32_t f = 0; f < nf; ++f)
        for (int j = 0; j < 3; ++j) {
            const uint32_t a = geometry[idx[3 * f + j]], b = geometry[idx[3 * f + (j + 1) % 3]];
            if (a == b) {
                for (int c = 0; c < 3; ++c) invalid[geometry[idx[3 * f + c]]] = 1;
                continue;
            }
            entries[a].push_back(b);
            entries[b].push_back(a);
        }
    std::vector<uint32_t> face_offsets(nv + 1, 0), faces, nbr_offsets(nv + 1, 0), neighbors;
    std::vector<uint8_t> nbr_count;
    for (uint32_t c = 0; c < nv; ++c) {
        std::sort(faces_of[c].begin(), faces_of[c].end());
        faces.insert(faces.end(), faces_of[c].begin(), faces_of[c].end());
        face_offsets[c + 1] = uint32_t(faces.size());
        std::vector<uint32_t>& e = entries[c];
        std::sort(e.begin(), e.end());
        for (size_t i = 0; i < e.size();) {
            size_t j = i + 1;
            while (j < e.size() && e[j] == e[i]) ++j;
            neighbors.push_back(e[i]);
            nbr_count.push_back(uint8_t(j - i < 3 ? j - i : 3));
            if (j - i == 1) boundary[c] = 1;
            if (j - i > 2) invalid[c] = 1;
            i = j;
        }
        nbr_offsets[c + 1] = uint32_t(neighbors.size());
    }
    neighbors.push_back(0);
    nbr_count.push_back(0);
    faces.push_back(0);
    ClassRing t{idx, mat, geometry.data(), face_offsets.data(), faces.data(), nbr_offsets.data(), neighbors.data(),
                nbr_count.data(), boundary.data(), invalid.data(), nv, nf};
    // Fans are decided on the flags before any fan result is written, as the
    // library's one-thread-per-class kernel reads them (a fan's own class
    // is the only flag it changes).
    std::vector<uint8_t> fan_bad(nv, 0);
    for (uint32_t u = 0; u < nv; ++u)
        if (!invalid[u]) fan_bad[u] = !single_fan(t, u);
    for (uint32_t u = 0; u < nv; ++u) invalid[u] |= fan_bad[u];
    uint64_t n = 0;
    for (uint32_t a = 0; a < nv; ++a)
        for (uint32_t k = nbr_offsets[a]; k < nbr_offsets[a + 1]; ++k) {
            const uint32_t b = neighbors[k];
            if (b <= a) continue;
            for (int dir = 0; dir < 2; ++dir) {
                Edit e{};
                e.from = dir ? b : a;
                e.to = dir ? a : b;
                if (!collapse_legal(t, e)) continue;
                if (n < cap) {
                    uint32_t* o = out + 7 * n;
                    o[0] = e.from, o[1] = e.to, o[2] = e.source[0], o[3] = e.source[1];
                    o[4] = e.target[0], o[5] = e.target[1], o[6] = uint32_t(e.wedges) | uint32_t(e.removed) << 8;
                }
                ++n;
            }
        }
    return int64_t(n);
}
