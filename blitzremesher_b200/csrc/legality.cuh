// Collapse legality on geometric classes, compiled for the host and the
// device alike: the library runs it one thread per directed edge, the CPU
// tests run the same code against the oracle's action sets.
//
// The predicate is the reference's legality with placement
// (src/neural/action_gpu.cu:487-624 with placement = true; the CPU statement
// is src/neural/action.cpp:146-256) and its single-fan rule
// (action_gpu.cu:288-344, action.cpp:109-144). It is written here as set
// operations on the class topology's sorted lists:
//   - the faces on the edge (u, v) are the intersection of the two classes'
//     ascending face lists, found by one merge;
//   - the link condition is one merge of the two sorted neighbour rows: the
//     classes adjacent to both must be exactly the apexes of the edge faces;
//   - the material rule compares the two classes' material sets;
//   - the faces that survive (u's faces off the edge), renamed by the wedge
//     map, must be proper triangles, pairwise distinct and distinct from
//     every face of v, compared as sorted class triples;
//   - a class's fan is one piece when a walk along its faces, entered at an
//     open end (a neighbour shared by one face) or anywhere on a closed
//     ring, crosses every face once.
#pragma once
#include "common.cuh"

namespace b200 {

// One directed collapse edit (action_gpu.cu:129-132): slot pairs (source of
// class `from`, target of class `to`) in ascending source order.
struct Edit {
    uint32_t from, to, source[2], target[2];
    uint8_t wedges, removed, valid, pad;
};

// Class topology of one mesh state, in host or device memory. Classes are
// named by their smallest vertex slot; face lists ascend; neighbour rows are
// sorted and unique with the number of faces each edge borders (capped at 3).
struct ClassRing {
    const uint32_t* idx;          // 3 slots per face
    const uint16_t* mat;          // per face or null
    const uint32_t* geometry;     // slot -> class
    const uint32_t* face_offsets; // class -> range in faces
    const uint32_t* faces;
    const uint32_t* nbr_offsets;  // class -> range in neighbors
    const uint32_t* neighbors;
    const uint8_t* nbr_count;
    const uint8_t* boundary;
    const uint8_t* invalid;
    uint32_t nv, nf;
};

BH uint32_t class_of(const ClassRing& t, uint32_t f, int j) { return t.geometry[t.idx[3 * f + j]]; }
BH uint16_t material_at(const ClassRing& t, uint32_t f) { return t.mat ? t.mat[f] : uint16_t(0); }

// Position of `key` in the sorted row [row, row + n), or kNone.
BH uint32_t row_position(const uint32_t* row, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (row[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && row[lo] == key ? lo : kNone;
}

// The two classes of face f other than u; false unless there are exactly two.
BH bool rim_of(const ClassRing& t, uint32_t f, uint32_t u, uint32_t& x, uint32_t& y) {
    uint32_t got[3], n = 0;
    for (int j = 0; j < 3; ++j) {
        const uint32_t c = class_of(t, f, j);
        if (c != u) got[n++] = c;
    }
    x = n > 0 ? got[0] : kNone;
    y = n > 1 ? got[1] : kNone;
    return n == 2;
}

// True when the faces around class u form one fan (an open or closed strip).
// Each face of u joins its two rim classes; with every rim class on at most
// two of u's faces (a valid class), the rims form paths and rings, and there
// is one piece exactly when a walk from an open end, or from any rim class
// when there is none, crosses all of u's faces.
BH bool single_fan(const ClassRing& t, uint32_t u) {
    const uint32_t f0 = t.face_offsets[u], f1 = t.face_offsets[u + 1];
    if (f0 == f1) return true;
    const uint32_t* row = t.neighbors + t.nbr_offsets[u];
    const uint32_t nrow = t.nbr_offsets[u + 1] - t.nbr_offsets[u];
    for (uint32_t k = f0; k < f1; ++k) {
        uint32_t x, y;
        if (!rim_of(t, t.faces[k], u, x, y)) return false;
        if (row_position(row, nrow, x) == kNone || row_position(row, nrow, y) == kNone) return false;
    }
    uint32_t start = kNone;
    for (uint32_t j = 0; j < nrow && start == kNone; ++j)
        if (t.nbr_count[t.nbr_offsets[u] + j] == 1) start = row[j];
    if (start == kNone) {
        uint32_t y;
        rim_of(t, t.faces[f0], u, start, y);
    }
    const uint32_t total = f1 - f0;
    uint32_t at = start, came = kNone, crossed = 0;
    while (crossed < total) {
        uint32_t through = kNone, next = kNone;
        for (uint32_t k = f0; k < f1 && through == kNone; ++k) {
            if (k == came) continue;
            uint32_t x, y;
            rim_of(t, t.faces[k], u, x, y);
            if (x == at) through = k, next = y;
            else if (y == at) through = k, next = x;
        }
        if (through == kNone) break;
        came = through;
        at = next;
        ++crossed;
        if (at == start) break;
    }
    return crossed == total;
}

BH void sort_triple(uint32_t& a, uint32_t& b, uint32_t& c) {
    if (a > b) { const uint32_t s = a; a = b; b = s; }
    if (b > c) { const uint32_t s = b; b = c; c = s; }
    if (a > b) { const uint32_t s = a; a = b; b = s; }
}

// Slot `id` after the collapse: the wedge target when id is a wedge source.
BH uint32_t renamed_slot(const Edit& e, uint32_t id) {
    for (uint32_t w = 0; w < e.wedges; ++w)
        if (e.source[w] == id) return e.target[w];
    return id;
}

// Sorted class triple of face f after the collapse (renamed) or before.
BH void face_key(const ClassRing& t, const Edit& e, uint32_t f, bool renamed, uint32_t key[3]) {
    for (int j = 0; j < 3; ++j) {
        const uint32_t id = t.idx[3 * f + j];
        key[j] = t.geometry[renamed ? renamed_slot(e, id) : id];
    }
    sort_triple(key[0], key[1], key[2]);
}

// Directed collapse e.from -> e.to; fills the wedge map (ascending sources)
// and the number of removed faces. Returns legality; e is unspecified when
// the collapse is illegal.
BH bool collapse_legal(const ClassRing& t, Edit& e) {
    const uint32_t u = e.from, v = e.to;
    e.wedges = 0;
    e.removed = 0;
    if (u >= t.nv || v >= t.nv || u == v || t.geometry[u] != u || t.geometry[v] != v) return false;
    if (t.invalid[u] || t.invalid[v]) return false;
    const uint32_t* ru = t.neighbors + t.nbr_offsets[u];
    const uint32_t* rv = t.neighbors + t.nbr_offsets[v];
    const uint32_t nu = t.nbr_offsets[u + 1] - t.nbr_offsets[u], nvr = t.nbr_offsets[v + 1] - t.nbr_offsets[v];
    if (row_position(ru, nu, v) == kNone) return false;

    // Faces on the edge: the merge of the two ascending face lists.
    const uint32_t* fu = t.faces + t.face_offsets[u];
    const uint32_t* fv = t.faces + t.face_offsets[v];
    const uint32_t cu = t.face_offsets[u + 1] - t.face_offsets[u], cv = t.face_offsets[v + 1] - t.face_offsets[v];
    uint32_t apex[2] = {kNone, kNone}, on_edge = 0;
    for (uint32_t i = 0, j = 0; i < cu && j < cv;) {
        if (fu[i] < fv[j]) { ++i; continue; }
        if (fv[j] < fu[i]) { ++j; continue; }
        const uint32_t f = fu[i];
        ++i, ++j;
        if (on_edge == 2) return false; // a third face on the edge
        uint32_t su = kNone, sv = kNone, third = kNone;
        for (int c = 0; c < 3; ++c) {
            const uint32_t id = t.idx[3 * f + c], g = t.geometry[id];
            if (g == u) su = id;
            else if (g == v) sv = id;
            else third = g;
        }
        if (third == kNone) return false; // degenerate face on the edge
        apex[on_edge++] = third;
        bool known = false;
        for (uint32_t w = 0; w < e.wedges; ++w) known |= e.source[w] == su && e.target[w] == sv;
        if (!known) {
            e.source[e.wedges] = su;
            e.target[e.wedges] = sv;
            ++e.wedges;
        }
    }
    if (on_edge == 0 || on_edge >= t.nf) return false;
    if (on_edge == 2 && apex[0] == apex[1]) return false;
    if (t.boundary[u] && (!t.boundary[v] || on_edge != 1)) return false;

    // Link condition: the common neighbours are exactly the apexes.
    uint32_t common = 0;
    for (uint32_t i = 0, j = 0; i < nu && j < nvr;) {
        if (ru[i] < rv[j]) { ++i; continue; }
        if (rv[j] < ru[i]) { ++j; continue; }
        const uint32_t w = ru[i];
        ++i, ++j;
        if (w != apex[0] && w != apex[1]) return false;
        ++common;
    }
    if (common != on_edge) return false;

    // Wedge map: two wedges need two distinct sources, kept in ascending order.
    if (e.wedges == 2) {
        if (e.source[0] == e.source[1]) return false;
        if (e.source[1] < e.source[0]) {
            uint32_t s = e.source[0];
            e.source[0] = e.source[1], e.source[1] = s;
            s = e.target[0];
            e.target[0] = e.target[1], e.target[1] = s;
        }
    }
    // Every corner of class u must be a wedge source.
    for (uint32_t i = 0; i < cu; ++i)
        for (int c = 0; c < 3; ++c) {
            const uint32_t id = t.idx[3 * fu[i] + c];
            if (t.geometry[id] == u && renamed_slot(e, id) == id) return false;
        }
    // Material junction: a multi-material fan needs equal material sets.
    bool mixed = false;
    for (uint32_t i = 1; i < cu; ++i) mixed |= material_at(t, fu[i]) != material_at(t, fu[0]);
    if (mixed) {
        for (int side = 0; side < 2; ++side) {
            const uint32_t* fa = side ? fv : fu;
            const uint32_t* fb = side ? fu : fv;
            const uint32_t ca = side ? cv : cu, cb = side ? cu : cv;
            for (uint32_t i = 0; i < ca; ++i) {
                const uint16_t want = material_at(t, fa[i]);
                bool seen = false;
                for (uint32_t j = 0; j < cb && !seen; ++j) seen = material_at(t, fb[j]) == want;
                if (!seen) return false;
            }
        }
    }
    // Surviving faces: proper, pairwise distinct, distinct from v's faces.
    auto on_v = [&](uint32_t f) {
        return class_of(t, f, 0) == v || class_of(t, f, 1) == v || class_of(t, f, 2) == v;
    };
    for (uint32_t i = 0; i < cu; ++i) {
        if (on_v(fu[i])) continue;
        uint32_t key[3];
        face_key(t, e, fu[i], true, key);
        if (key[0] == key[1] || key[1] == key[2]) return false;
        for (uint32_t j = i + 1; j < cu; ++j) {
            if (on_v(fu[j])) continue;
            uint32_t other[3];
            face_key(t, e, fu[j], true, other);
            if (other[0] == key[0] && other[1] == key[1] && other[2] == key[2]) return false;
        }
        for (uint32_t j = 0; j < cv; ++j) {
            uint32_t other[3];
            face_key(t, e, fv[j], false, other);
            if (other[0] == key[0] && other[1] == key[1] && other[2] == key[2]) return false;
        }
    }
    e.removed = uint8_t(on_edge);
    return true;
}

} // namespace b200
