// Full-raster path: coverage masks and sample counts of whole meshes, mask
// popcounts, and the exact squared distance transform used when a view is
// audited without the incremental path.
//
// Coverage semantics follow evaluate.cpp:125-189 (FP64 conservative test at
// sample centres, culling, clipping with the CPU's stop-at-first-clipped-face
// rule). Distances follow evaluate.cpp:33-70 and 196-209: the CPU float field
// equals the exact integer squared distance below 2^24; above it the float
// rounding of the two separable passes is reproduced.
#include "kernels.cuh"
#include "nearest.cuh"

namespace b200 {
namespace {
constexpr int kThreads = 256;
inline uint32_t blocks_for(uint64_t n, int threads = kThreads) { return uint32_t((n + threads - 1) / threads); }

struct RasterArgs {
    DevMesh m;
    Camera cam;
    float center[3];
    uint32_t ss, size, force_two, cpu_semantics;
};

__device__ FaceSetup face_setup(const RasterArgs& a, uint32_t f) {
    Proj p[3];
    for (int j = 0; j < 3; ++j) {
        uint32_t v = a.m.idx[3 * f + j];
        p[j] = project(a.m.pos[3 * v], a.m.pos[3 * v + 1], a.m.pos[3 * v + 2], a.center, a.cam, a.ss, a.size);
    }
    bool two = a.force_two;
    if (!two && a.m.sided) {
        uint16_t mat = a.m.mat ? a.m.mat[f] : 0;
        two = mat < a.m.nsided && a.m.sided[mat];
    }
    return setup_face(p[0], p[1], p[2], a.cam.perspective != 0, two, a.size);
}

__global__ void k_state_init(uint32_t* state) {
    if (threadIdx.x < 4) state[threadIdx.x] = threadIdx.x == 0 ? kNone : 0u;
}

// state[0]: first box-clipped face (min index), state[1]: any clip,
// state[2]: clipped face count, state[3]: count overflow.
__global__ void k_raster_clip(RasterArgs a, uint32_t* state) {
    uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.m.nf) return;
    FaceSetup s = face_setup(a, f);
    if (s.status == kFaceClipBox) atomicMin(state, f);
    if (s.status == kFaceClipBox || s.status == kFaceClipZ) {
        state[1] = 1;
        atomicAdd(state + 2, 1u);
    }
}

__device__ __forceinline__ void count_sample(uint8_t* counts, size_t i, uint32_t* state) {
    uint32_t* w = reinterpret_cast<uint32_t*>(counts) + (i >> 2);
    uint32_t shift = 8 * uint32_t(i & 3);
    uint32_t old = atomicAdd(w, 1u << shift);
    if (((old >> shift) & 0xffu) == 0xffu) state[3] = 1;
}
// The same count held at 255 ("255 or more"): exact for the audits, which
// compare a count with at most kMaxOk (< 255) changed faces, and for the
// coverage bits (count > 0); counts are always rebuilt from scratch.
__device__ __forceinline__ void count_sample_saturating(uint8_t* counts, size_t i) {
    uint32_t* w = reinterpret_cast<uint32_t*>(counts) + (i >> 2);
    const uint32_t shift = 8 * uint32_t(i & 3);
    uint32_t old = *w, seen;
    do {
        seen = old;
        if (((seen >> shift) & 0xffu) == 0xffu) return;
        old = atomicCAS(w, seen, seen + (1u << shift));
    } while (old != seen);
}

// One thread per face over its bounding box. bits: coverage (u64 LE layout as
// u32 words); counts: covering faces per sample (u8, packed in u32 words).
__global__ void k_raster_fill(RasterArgs a, uint32_t* bits, uint8_t* counts, uint32_t* state) {
    uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.m.nf) return;
    if (a.cpu_semantics && f > state[0]) return;
    FaceSetup s = face_setup(a, f);
    if (s.status != kFaceOk) return;
    for (int y = s.y0; y <= s.y1; ++y)
        for (int x = s.x0; x <= s.x1; ++x) {
            if (!face_covers(s, x, y)) continue;
            size_t i = size_t(y) * a.size + x;
            if (bits) atomicOr(bits + (i >> 5), 1u << (i & 31));
            if (counts) count_sample(counts, i, state);
        }
}

__global__ void k_popcounts(const uint32_t* a, const uint32_t* b, uint32_t words, uint64_t samples,
                            unsigned long long* out) {
    unsigned long long changed = 0, total = 0, ca = 0, cb = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) {
        uint32_t x = a[i], y = b[i];
        // samples != 0: bits at or past `samples` are not samples and do not count.
        if (samples && uint64_t(i + 1) * 32 > samples) {
            const uint64_t first = uint64_t(i) * 32;
            const uint32_t keep = samples > first ? uint32_t((1ull << (samples - first)) - 1) : 0u;
            x &= keep, y &= keep;
        }
        changed += __popc(x ^ y);
        total += __popc(x | y);
        ca += __popc(x);
        cb += __popc(y);
    }
    for (int o = 16; o; o >>= 1) {
        changed += __shfl_down_sync(0xffffffffu, changed, o);
        total += __shfl_down_sync(0xffffffffu, total, o);
        ca += __shfl_down_sync(0xffffffffu, ca, o);
        cb += __shfl_down_sync(0xffffffffu, cb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (changed) atomicAdd(out, changed);
        if (total) atomicAdd(out + 1, total);
        if (ca) atomicAdd(out + 2, ca);
        if (cb) atomicAdd(out + 3, cb);
    }
}

__device__ __forceinline__ bool bit_at(const uint32_t* bits, size_t i) { return (bits[i >> 5] >> (i & 31)) & 1u; }

// Horizontal distance to the nearest covered sample of row y (kNone when the
// row has none), one warp per row: per group of 32 samples each lane takes
// one sample, the group's coverage word is read once by all lanes, and the
// nearest covered sample at or after / at or before the lane comes from the
// word's bits or, when they hold none, from the groups already passed (the
// same for all lanes). Writes are 32 consecutive words per group.
__device__ void row_nearest_warp(const uint32_t* bits, uint32_t width, uint32_t y, uint32_t* g) {
    const uint32_t lane = threadIdx.x & 31;
    const size_t row = size_t(y) * width, row_end = row + width;
    const uint32_t groups = (width + 31) / 32;
    auto word_of = [&](uint32_t k) {
        const size_t b = row + size_t(k) * 32;
        const uint32_t sh = uint32_t(b & 31);
        const size_t w = b >> 5;
        uint32_t v = bits[w] >> sh;
        if (sh && (w + 1) * 32 < row_end) v |= bits[w + 1] << (32 - sh); // only words holding samples of the row
        const uint32_t rem = width - k * 32;
        return rem >= 32 ? v : (v & ((1u << rem) - 1u));
    };
    uint32_t next = kNone; // first covered sample after the groups to the right
    for (uint32_t k = groups; k-- > 0;) {
        const uint32_t w = word_of(k), x = k * 32 + lane;
        const uint32_t m = w & ~((1u << lane) - 1u); // covered samples at or after x in this group
        const uint32_t at = m ? k * 32 + uint32_t(__ffs(m)) - 1 : next;
        if (x < width) g[row + x] = at == kNone ? kNone : at - x;
        if (w) next = k * 32 + uint32_t(__ffs(w)) - 1;
    }
    uint32_t last = kNone; // last covered sample of the groups to the left
    for (uint32_t k = 0; k < groups; ++k) {
        const uint32_t w = word_of(k), x = k * 32 + lane;
        const uint32_t m = lane == 31 ? w : (w & ((2u << lane) - 1u)); // covered samples at or before x
        const uint32_t at = m ? k * 32 + 31 - uint32_t(__clz(m)) : last;
        if (x < width && at != kNone && x - at < g[row + x]) g[row + x] = x - at;
        if (w) last = k * 32 + 31 - uint32_t(__clz(w));
    }
}
__global__ void k_row_nearest(const uint32_t* to, uint32_t width, uint32_t height, uint32_t* g) {
    const uint32_t y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (y < height) row_nearest_warp(to, width, y, g);
}

// Lower envelope of the parabolas (y-q)^2 + g(x,q)^2 over rows q with a site
// (Felzenszwalb–Huttenlocher), in exact integer arithmetic: intersections are
// kept as fractions and compared by cross-multiplication.
__device__ void k_column_envelope_body(const uint32_t* g, uint32_t width, uint32_t height, uint32_t x, uint32_t* d2,
                                       int32_t* sv, long long* snum, long long* sden);
__global__ void k_column_envelope(const uint32_t* g, uint32_t width, uint32_t height, uint32_t* d2, int32_t* sv,
                                  long long* snum, long long* sden) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < width) k_column_envelope_body(g, width, height, x, d2, sv, snum, sden);
}
__device__ void k_column_envelope_body(const uint32_t* g, uint32_t width, uint32_t height, uint32_t x, uint32_t* d2,
                                       int32_t* sv, long long* snum, long long* sden) {
    const uint32_t size = width; // row stride of g and d2
    // Stack entry k of column x lives at k * width + x: neighbouring columns'
    // entries are neighbours in memory.
    struct Col {
        int32_t* p;
        size_t s;
        __device__ int32_t& operator[](int k) const { return p[size_t(k) * s]; }
    };
    struct ColL {
        long long* p;
        size_t s;
        __device__ long long& operator[](int k) const { return p[size_t(k) * s]; }
    };
    const Col v{sv + x, width};
    const ColL zn{snum + x, width}, zd{sden + x, width};
    int k = -1;
    for (uint32_t q = 0; q < height; ++q) {
        uint32_t gq = g[size_t(q) * size + x];
        if (gq == kNone) continue;
        long long fq = (long long)gq * gq + (long long)q * q;
        if (k < 0) {
            k = 0;
            v[0] = int32_t(q);
            continue;
        }
        long long num, den;
        for (;;) {
            int p = v[k];
            uint32_t gp = g[size_t(p) * size + x];
            long long fp = (long long)gp * gp + (long long)p * p;
            num = fq - fp;
            den = 2ll * ((long long)q - p);
            // s > z[k]  <=>  num/den > zn[k]/zd[k]
            if (k == 0 || num * zd[k] > zn[k] * den) break;
            --k;
        }
        ++k;
        v[k] = int32_t(q);
        zn[k] = num;
        zd[k] = den;
    }
    if (k < 0) {
        for (uint32_t y = 0; y < height; ++y) d2[size_t(y) * size + x] = kNone;
        return;
    }
    int top = k;
    k = 0;
    for (uint32_t y = 0; y < height; ++y) {
        while (k < top && zn[k + 1] < (long long)y * zd[k + 1]) ++k;
        long long dy = (long long)y - v[k];
        uint32_t gq = g[size_t(v[k]) * size + x];
        d2[size_t(y) * size + x] = uint32_t(dy * dy + (long long)gq * gq);
    }
}

// Max over samples covered by `from` and not by `to` of the field of `to`, as
// float bit patterns (non-negative floats order like their bits).
__global__ void k_directed_max(const uint32_t* from, const uint32_t* to, const uint32_t* d2, const uint32_t* g,
                               uint32_t width, uint32_t height, uint32_t* out) {
    size_t n = size_t(width) * height;
    uint32_t best = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        if (!bit_at(from, i) || bit_at(to, i)) continue;
        uint32_t d = d2[i];
        float val = d < kExactLimit ? float(d)
                                    : cpu_field_value(g, width, height, uint32_t(i % width), uint32_t(i / width));
        uint32_t b = __float_as_uint(val);
        best = b > best ? b : best;
    }
    for (int o = 16; o; o >>= 1) {
        uint32_t y = __shfl_down_sync(0xffffffffu, best, o);
        best = y > best ? y : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}
// Coverage words from the per-sample face counts (count > 0), u64 layout.
__global__ void k_counts_to_bits(const uint8_t* counts, size_t samples, uint32_t* bits, uint32_t words) {
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    uint32_t out = 0;
    size_t base = size_t(w) * 32;
    for (int k = 0; k < 32; ++k) {
        size_t i = base + k;
        if (i < samples && counts[i]) out |= 1u << k;
    }
    bits[w] = out;
}

// Per 32x32 tile: t1 = max reference field over samples covered by the state
// and not by the reference; t2 = max state field over samples covered by the
// reference and not by the state; -1 when the tile has no such sample.
__device__ void tile_maxima_body(const uint32_t* ref_bits, const uint32_t* state_bits, const uint32_t* ref_field,
                                 const uint32_t* state_field, uint32_t size, uint32_t tile, int32_t* t1, int32_t* t2);
__global__ void k_tile_maxima(const uint32_t* ref_bits, const uint32_t* state_bits, const uint32_t* ref_field,
                              const uint32_t* state_field, uint32_t size, int32_t* t1, int32_t* t2) {
    tile_maxima_body(ref_bits, state_bits, ref_field, state_field, size, blockIdx.x, t1, t2);
}
__device__ void tile_maxima_body(const uint32_t* ref_bits, const uint32_t* state_bits, const uint32_t* ref_field,
                                 const uint32_t* state_field, uint32_t size, uint32_t tile, int32_t* t1, int32_t* t2) {
    const uint32_t tiles_x = (size + 31) / 32;
    const uint32_t lane = threadIdx.x;
    const uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
    const uint32_t x = tx * 32 + lane;
    int32_t m1 = -1, m2 = -1;
    if (x < size)
        for (uint32_t r = 0; r < 32; ++r) {
            uint32_t y = ty * 32 + r;
            if (y >= size) break;
            size_t i = size_t(y) * size + x;
            bool p = bit_at(state_bits, i), q = bit_at(ref_bits, i);
            if (p && !q) m1 = max(m1, int32_t(min(ref_field[i], 0x7fffffffu)));
            if (q && !p) m2 = max(m2, int32_t(min(state_field[i], 0x7fffffffu)));
        }
    for (int o = 16; o; o >>= 1) {
        m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    if (lane == 0) t1[tile] = m1, t2[tile] = m2;
}
// A packed coverage mask (bit i = sample i = y * size + x of a linear bit
// stream) read 32 columns at a time, for nearest_d2.
struct StreamMask {
    const uint32_t* bits;
    uint32_t size;
    __device__ uint32_t chunk(uint32_t row, uint32_t c) const {
        const size_t b = size_t(row) * size + size_t(c) * 32;
        const uint32_t sh = uint32_t(b & 31);
        const size_t w = b >> 5;
        uint32_t v = bits[w];
        if (sh) v = (v >> sh) | (bits[w + 1] << (32 - sh)); // the mask's padding word keeps this in bounds
        const uint32_t rem = size - c * 32;
        return rem >= 32 ? v : v & ((1u << rem) - 1u);
    }
};
// tile_maxima_body without the state's field: t2 takes each reference-only
// sample's exact squared distance to the state's nearest covered sample by
// the outward search (the value the field holds there; kNone, as the field's
// empty value, clamps the same way).
__device__ void tile_maxima_search_body(const uint32_t* ref_bits, const uint32_t* state_bits,
                                        const uint32_t* ref_field, uint32_t size, uint32_t tile, int32_t* t1,
                                        int32_t* t2) {
    const uint32_t tiles_x = (size + 31) / 32;
    const uint32_t lane = threadIdx.x;
    const uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
    const uint32_t x = tx * 32 + lane;
    const StreamMask state{state_bits, size};
    int32_t m1 = -1, m2 = -1;
    if (x < size)
        for (uint32_t r = 0; r < 32; ++r) {
            const uint32_t y = ty * 32 + r;
            if (y >= size) break;
            const size_t i = size_t(y) * size + x;
            const bool p = bit_at(state_bits, i), q = bit_at(ref_bits, i);
            if (p && !q) m1 = max(m1, int32_t(min(ref_field[i], 0x7fffffffu)));
            if (q && !p) m2 = max(m2, int32_t(min(nearest_d2(state, x, y), 0x7fffffffu)));
        }
    for (int o = 16; o; o >>= 1) {
        m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    if (lane == 0) t1[tile] = m1, t2[tile] = m2;
}
// ---- all views of a plan in one launch (blockIdx.y = view) ----
struct ViewsArgs {
    DevMesh m;
    const Camera* cams;
    float center[3];
    uint32_t ss, size, force_two, pad;
};

__device__ FaceSetup face_setup_view(const ViewsArgs& a, const Camera& cam, uint32_t f) {
    Proj p[3];
    for (int j = 0; j < 3; ++j) {
        uint32_t v = a.m.idx[3 * f + j];
        p[j] = project(a.m.pos[3 * v], a.m.pos[3 * v + 1], a.m.pos[3 * v + 2], a.center, cam, a.ss, a.size);
    }
    bool two = a.force_two;
    if (!two && a.m.sided) {
        uint16_t mat = a.m.mat ? a.m.mat[f] : 0;
        two = mat < a.m.nsided && a.m.sided[mat];
    }
    return setup_face(p[0], p[1], p[2], cam.perspective != 0, two, a.size);
}

// Face counts of every view: state[4v+2] clipped faces, state[4v+3] overflow
// (kSaturate: counts held at 255 instead, no overflow).
template <bool kSaturate>
__global__ void k_count_views(ViewsArgs a, uint8_t* counts, size_t stride, uint32_t* state) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (f >= a.m.nf) return;
    const Camera cam = a.cams[v];
    FaceSetup s = face_setup_view(a, cam, f);
    uint32_t* st = state + 4 * v;
    if (s.status == kFaceClipBox || s.status == kFaceClipZ) {
        atomicAdd(st + 2, 1u);
        return;
    }
    if (s.status != kFaceOk) return;
    uint8_t* c = counts + stride * v;
    for (int y = s.y0; y <= s.y1; ++y)
        for (int x = s.x0; x <= s.x1; ++x)
            if (face_covers(s, x, y)) {
                if constexpr (kSaturate) count_sample_saturating(c, size_t(y) * a.size + x);
                else count_sample(c, size_t(y) * a.size + x, st);
            }
}
// Changed faces of a combined trial, all views: the state's face leaves its
// samples (-1; every covered sample counts it, so no count goes below zero),
// the trial's face, when it survives, enters (+1; passing 255 sets the view's
// overflow flag, and the caller counts afresh).
__global__ void k_count_delta_views(ViewsArgs a, TrialDelta d, uint8_t* counts, size_t stride, uint32_t* state) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (f >= a.m.nf) return;
    bool changed = false;
    for (int j = 0; j < 3; ++j) {
        const uint32_t id = a.m.idx[3 * f + j];
        changed |= d.remap[id] != kNone || d.owner[d.geometry[id]] != kNone;
    }
    if (!changed) return;
    const Camera cam = a.cams[v];
    uint32_t* st = state + 4 * v;
    uint8_t* c = counts + stride * v;
    const FaceSetup s = face_setup_view(a, cam, f);
    if (s.status == kFaceClipBox || s.status == kFaceClipZ) {
        atomicSub(st + 2, 1u);
    } else if (s.status == kFaceOk) {
        for (int y = s.y0; y <= s.y1; ++y)
            for (int x = s.x0; x <= s.x1; ++x)
                if (face_covers(s, x, y)) {
                    const size_t i = size_t(y) * a.size + x;
                    atomicSub(reinterpret_cast<uint32_t*>(c) + (i >> 2), 1u << (8 * uint32_t(i & 3)));
                }
    }
    if (!d.keep[f]) return;
    ViewsArgs b = a;
    b.m = d.trial;
    const FaceSetup t = face_setup_view(b, cam, d.offsets[f]);
    if (t.status == kFaceClipBox || t.status == kFaceClipZ) {
        atomicAdd(st + 2, 1u);
        return;
    }
    if (t.status != kFaceOk) return;
    for (int y = t.y0; y <= t.y1; ++y)
        for (int x = t.x0; x <= t.x1; ++x)
            if (face_covers(t, x, y)) count_sample(c, size_t(y) * a.size + x, st);
}
// Face counts of every view into 32-bit counters (`wide`, samples per view;
// no overflow, for the deep overlaps of small screens), then narrowed to
// counts held at 255 by k_narrow_counts_views: far fewer retries than the
// compare-and-swap counts where hundreds of faces cover a sample.
__global__ void k_count_views_wide(ViewsArgs a, uint32_t* wide, uint32_t* state) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (f >= a.m.nf) return;
    const Camera cam = a.cams[v];
    FaceSetup s = face_setup_view(a, cam, f);
    if (s.status == kFaceClipBox || s.status == kFaceClipZ) {
        atomicAdd(state + 4 * v + 2, 1u);
        return;
    }
    if (s.status != kFaceOk) return;
    uint32_t* c = wide + size_t(a.size) * a.size * v;
    for (int y = s.y0; y <= s.y1; ++y)
        for (int x = s.x0; x <= s.x1; ++x)
            if (face_covers(s, x, y)) atomicAdd(c + size_t(y) * a.size + x, 1u);
}
__global__ void k_narrow_counts_views(const uint32_t* wide, size_t samples, uint8_t* counts, size_t cstride) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t v = blockIdx.y;
    if (i < samples) counts[cstride * v + i] = uint8_t(min(wide[samples * v + i], 255u));
}
__global__ void k_counts_to_bits_views(const uint8_t* counts, size_t cstride, size_t samples, uint32_t* bits,
                                       uint32_t wstride, uint32_t words) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (w >= words) return;
    const uint8_t* c = counts + cstride * v;
    uint32_t out = 0;
    const size_t base = size_t(w) * 32;
    for (int k = 0; k < 32; ++k) {
        size_t i = base + k;
        if (i < samples && c[i]) out |= 1u << k;
    }
    bits[size_t(wstride) * v + w] = out;
}
__global__ void k_row_nearest_views(const uint32_t* bits, uint32_t wstride, uint32_t size, uint32_t* g) {
    const uint32_t y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, v = blockIdx.y;
    if (y >= size) return;
    const size_t samples = size_t(size) * size;
    row_nearest_warp(bits + size_t(wstride) * v, size, y, g + samples * v);
}
__global__ void k_column_envelope_views(const uint32_t* g, uint32_t size, uint32_t* d2, int32_t* sv, long long* sn,
                                        long long* sd) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (x >= size) return;
    const size_t samples = size_t(size) * size;
    k_column_envelope_body(g + samples * v, size, size, x, d2 + samples * v, sv + samples * v, sn + samples * v,
                           sd + samples * v);
}
__global__ void k_tile_maxima_views(const uint32_t* ref_bits, const uint32_t* state_bits, uint32_t wstride,
                                    const uint32_t* ref_field, const uint32_t* state_field, uint32_t size, int32_t* t1,
                                    int32_t* t2) {
    const uint32_t v = blockIdx.y, tiles_x = (size + 31) / 32, tiles = tiles_x * tiles_x;
    const size_t samples = size_t(size) * size;
    tile_maxima_body(ref_bits + size_t(wstride) * v, state_bits + size_t(wstride) * v, ref_field + samples * v,
                     state_field + samples * v, size, blockIdx.x, t1 + size_t(tiles) * v, t2 + size_t(tiles) * v);
}
__global__ void k_tile_maxima_search_views(const uint32_t* ref_bits, const uint32_t* state_bits, uint32_t wstride,
                                           const uint32_t* ref_field, uint32_t size, int32_t* t1, int32_t* t2) {
    const uint32_t v = blockIdx.y, tiles_x = (size + 31) / 32, tiles = tiles_x * tiles_x;
    const size_t samples = size_t(size) * size;
    tile_maxima_search_body(ref_bits + size_t(wstride) * v, state_bits + size_t(wstride) * v, ref_field + samples * v,
                            size, blockIdx.x, t1 + size_t(tiles) * v, t2 + size_t(tiles) * v);
}
__global__ void k_popcounts_views(const uint32_t* a, const uint32_t* b, uint32_t wstride, uint32_t words,
                                  unsigned long long* out) {
    const uint32_t v = blockIdx.y;
    unsigned long long changed = 0, total = 0, ca = 0, cb = 0;
    const uint32_t* av = a + size_t(wstride) * v;
    const uint32_t* bv = b + size_t(wstride) * v;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) {
        uint32_t x = av[i], y = bv[i];
        changed += __popc(x ^ y);
        total += __popc(x | y);
        ca += __popc(x);
        cb += __popc(y);
    }
    for (int o = 16; o; o >>= 1) {
        changed += __shfl_down_sync(0xffffffffu, changed, o);
        total += __shfl_down_sync(0xffffffffu, total, o);
        ca += __shfl_down_sync(0xffffffffu, ca, o);
        cb += __shfl_down_sync(0xffffffffu, cb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        unsigned long long* o = out + 4 * v;
        if (changed) atomicAdd(o, changed);
        if (total) atomicAdd(o + 1, total);
        if (ca) atomicAdd(o + 2, ca);
        if (cb) atomicAdd(o + 3, cb);
    }
}
} // namespace

// The state data of all views of a plan, refreshed in a handful of launches:
// counts (and clipped/overflow counters), coverage words, popcounts against the
// reference and, when fields are kept, the tile maxima: from the state field
// when `state_field` is given, else (ref_field, t1, t2 given) by searches
// from the reference-only samples. `saturate`: counts held at 255, through
// 32-bit counters in `wide` (samples * nviews) when given. `recount` false:
// `counts` and `state` already hold the views' counts (launch_count_delta_views).
void launch_refresh_views(const DevMesh& m, const Camera* cams_dev, uint32_t nviews, const float* center, uint32_t ss,
                          uint32_t size, bool force_two, uint8_t* counts, size_t cstride, uint32_t* state,
                          uint32_t* state_bits, const uint32_t* ref_bits, uint32_t wstride,
                          unsigned long long* pop, const uint32_t* ref_field, uint32_t* state_field, uint32_t* g,
                          int32_t* sv, long long* sn, long long* sd, int32_t* t1, int32_t* t2, bool saturate,
                          cudaStream_t s, uint32_t* wide, bool recount) {
    ViewsArgs a;
    a.m = m;
    a.cams = cams_dev;
    a.center[0] = center[0], a.center[1] = center[1], a.center[2] = center[2];
    a.ss = ss, a.size = size, a.force_two = force_two, a.pad = 0;
    const size_t samples = size_t(size) * size;
    if (recount) cudaMemsetAsync(counts, 0, cstride * nviews, s);
    if (recount) cudaMemsetAsync(state, 0, 16 * size_t(nviews), s);
    if (m.nf && recount) {
        const dim3 grid(blocks_for(m.nf, 128), nviews);
        if (saturate && wide) {
            cudaMemsetAsync(wide, 0, samples * nviews * 4, s);
            k_count_views_wide<<<grid, 128, 0, s>>>(a, wide, state);
            k_narrow_counts_views<<<dim3(uint32_t((samples + 255) / 256), nviews), 256, 0, s>>>(wide, samples, counts,
                                                                                                 cstride);
        } else if (saturate) {
            k_count_views<true><<<grid, 128, 0, s>>>(a, counts, cstride, state);
        } else {
            k_count_views<false><<<grid, 128, 0, s>>>(a, counts, cstride, state);
        }
    }
    const uint32_t words = uint32_t((samples + 63) / 64) * 2;
    if (state_bits) {
        k_counts_to_bits_views<<<dim3(blocks_for(words), nviews), kThreads, 0, s>>>(counts, cstride, samples,
                                                                                     state_bits, wstride, words);
        if (state_field) {
            k_row_nearest_views<<<dim3(blocks_for(uint64_t(size) * 32, 128), nviews), 128, 0, s>>>(state_bits, wstride,
                                                                                                 size, g);
            k_column_envelope_views<<<dim3(blocks_for(size, 64), nviews), 64, 0, s>>>(g, size, state_field, sv, sn,
                                                                                       sd);
            const uint32_t tiles = ((size + 31) / 32) * ((size + 31) / 32);
            k_tile_maxima_views<<<dim3(tiles, nviews), 32, 0, s>>>(ref_bits, state_bits, wstride, ref_field,
                                                                   state_field, size, t1, t2);
        } else if (ref_field && t1 && t2) {
            // no state field: t2 by searches from the reference-only samples
            const uint32_t tiles = ((size + 31) / 32) * ((size + 31) / 32);
            k_tile_maxima_search_views<<<dim3(tiles, nviews), 32, 0, s>>>(ref_bits, state_bits, wstride, ref_field,
                                                                          size, t1, t2);
        }
    }
    cudaMemsetAsync(pop, 0, 32 * size_t(nviews), s);
    uint32_t grid = blocks_for(words);
    if (grid > 64) grid = 64;
    k_popcounts_views<<<dim3(grid, nviews), kThreads, 0, s>>>(ref_bits, state_bits ? state_bits : ref_bits, wstride,
                                                               words, pop);
}

void launch_count_delta_views(const DevMesh& m, const TrialDelta& d, const Camera* cams_dev, uint32_t nviews,
                              const float* center, uint32_t ss, uint32_t size, bool force_two, uint8_t* counts,
                              size_t cstride, uint32_t* state, cudaStream_t s) {
    if (!m.nf) return;
    ViewsArgs a;
    a.m = m;
    a.cams = cams_dev;
    a.center[0] = center[0], a.center[1] = center[1], a.center[2] = center[2];
    a.ss = ss, a.size = size, a.force_two = force_two, a.pad = 0;
    k_count_delta_views<<<dim3(blocks_for(m.nf, 128), nviews), 128, 0, s>>>(a, d, counts, cstride, state);
}

// Exact squared distance fields of `nviews` masks (view v's coverage at
// bits + wstride * v, its field at field + size^2 * v): the row pass and the
// column envelope of launch_field for all of them in two launches.
void launch_fields_views(const uint32_t* bits, uint32_t wstride, uint32_t nviews, uint32_t size, uint32_t* g,
                         uint32_t* field, int32_t* sv, long long* sn, long long* sd, cudaStream_t s) {
    k_row_nearest_views<<<dim3(blocks_for(uint64_t(size) * 32, 128), nviews), 128, 0, s>>>(bits, wstride, size, g);
    k_column_envelope_views<<<dim3(blocks_for(size, 64), nviews), 64, 0, s>>>(g, size, field, sv, sn, sd);
}

// The last stages of launch_refresh_views against another reference, for
// views whose state coverage (state_bits) and, optionally, field
// (state_field; null: t2 by searches) are already computed: tile maxima and
// popcounts.
void launch_compare_views(uint32_t nviews, uint32_t size, const uint32_t* state_bits, const uint32_t* ref_bits,
                          uint32_t wstride, const uint32_t* ref_field, const uint32_t* state_field, int32_t* t1,
                          int32_t* t2, unsigned long long* pop, cudaStream_t s) {
    const size_t samples = size_t(size) * size;
    const uint32_t words = uint32_t((samples + 63) / 64) * 2;
    const uint32_t tiles = ((size + 31) / 32) * ((size + 31) / 32);
    if (state_field)
        k_tile_maxima_views<<<dim3(tiles, nviews), 32, 0, s>>>(ref_bits, state_bits, wstride, ref_field, state_field,
                                                               size, t1, t2);
    else
        k_tile_maxima_search_views<<<dim3(tiles, nviews), 32, 0, s>>>(ref_bits, state_bits, wstride, ref_field, size,
                                                                      t1, t2);
    cudaMemsetAsync(pop, 0, 32 * size_t(nviews), s);
    uint32_t grid = blocks_for(words);
    if (grid > 64) grid = 64;
    k_popcounts_views<<<dim3(grid, nviews), kThreads, 0, s>>>(ref_bits, state_bits, wstride, words, pop);
}

namespace {
// Per view: max over its 32x32 tiles of t1 and t2 (-1 when no tile has a sample).
__global__ void k_view_maxima(const int32_t* t1, const int32_t* t2, uint32_t tiles, int32_t* out) {
    const uint32_t v = blockIdx.x;
    int32_t m1 = -1, m2 = -1;
    for (uint32_t i = threadIdx.x; i < tiles; i += blockDim.x) {
        m1 = max(m1, t1[size_t(v) * tiles + i]);
        m2 = max(m2, t2[size_t(v) * tiles + i]);
    }
    for (int o = 16; o; o >>= 1) {
        m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    __shared__ int32_t r1[32], r2[32];
    const uint32_t w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) r1[w] = m1, r2[w] = m2;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t k = 1; k < blockDim.x / 32; ++k) m1 = max(m1, r1[k]), m2 = max(m2, r2[k]);
        out[2 * v] = m1;
        out[2 * v + 1] = m2;
    }
}
} // namespace

void launch_view_maxima(const int32_t* t1, const int32_t* t2, uint32_t tiles, uint32_t nviews, int32_t* out,
                        cudaStream_t s) {
    if (nviews) k_view_maxima<<<nviews, 256, 0, s>>>(t1, t2, tiles, out);
}

void launch_counts_to_bits(const uint8_t* counts, uint32_t size, uint32_t* bits, cudaStream_t s) {
    size_t samples = size_t(size) * size;
    uint32_t words = uint32_t((samples + 63) / 64) * 2;
    k_counts_to_bits<<<blocks_for(words), kThreads, 0, s>>>(counts, samples, bits, words);
}

void launch_tile_maxima(const uint32_t* ref_bits, const uint32_t* state_bits, const uint32_t* ref_field,
                        const uint32_t* state_field, uint32_t size, int32_t* t1, int32_t* t2, cudaStream_t s) {
    uint32_t tiles = ((size + 31) / 32) * ((size + 31) / 32);
    k_tile_maxima<<<tiles, 32, 0, s>>>(ref_bits, state_bits, ref_field, state_field, size, t1, t2);
}

// Exact squared distance field of `bits` (d2 = kNone where the mask is empty).
void launch_field(const uint32_t* bits, uint32_t width, uint32_t height, uint32_t* g, uint32_t* d2, int32_t* stack_v,
                  long long* stack_num, long long* stack_den, cudaStream_t s) {
    k_row_nearest<<<blocks_for(uint64_t(height) * 32, 128), 128, 0, s>>>(bits, width, height, g);
    k_column_envelope<<<blocks_for(width, 64), 64, 0, s>>>(g, width, height, d2, stack_v, stack_num, stack_den);
}

void launch_raster(const DevMesh& m, const Camera* cam_host, const float* center, uint32_t ss, uint32_t size,
                   bool force_two, bool cpu_semantics, uint32_t* bits, uint8_t* counts, uint32_t* state,
                   cudaStream_t s) {
    RasterArgs a;
    a.m = m;
    a.cam = *cam_host;
    a.center[0] = center[0], a.center[1] = center[1], a.center[2] = center[2];
    a.ss = ss, a.size = size, a.force_two = force_two, a.cpu_semantics = cpu_semantics;
    k_state_init<<<1, 32, 0, s>>>(state);
    if (!m.nf) return;
    k_raster_clip<<<blocks_for(m.nf), kThreads, 0, s>>>(a, state);
    k_raster_fill<<<blocks_for(m.nf, 128), 128, 0, s>>>(a, bits, counts, state);
}

void launch_popcounts(const uint32_t* a, const uint32_t* b, uint32_t words, unsigned long long* out,
                      cudaStream_t s, uint64_t samples) {
    cudaMemsetAsync(out, 0, 4 * sizeof(unsigned long long), s);
    uint32_t grid = blocks_for(words);
    if (grid > 1184) grid = 1184;
    if (!grid) grid = 1;
    k_popcounts<<<grid, kThreads, 0, s>>>(a, b, words, samples, out);
}

// Field of `to`, max over from \ to (as float bits) into out_max.
void launch_distance(const uint32_t* from, const uint32_t* to, uint32_t width, uint32_t height, uint32_t* g,
                     uint32_t* d2, int32_t* stack_v, long long* stack_num, long long* stack_den, uint32_t* out_max,
                     cudaStream_t s) {
    k_row_nearest<<<blocks_for(uint64_t(height) * 32, 128), 128, 0, s>>>(to, width, height, g);
    k_column_envelope<<<blocks_for(width, 64), 64, 0, s>>>(g, width, height, d2, stack_v, stack_num, stack_den);
    size_t n = size_t(width) * height;
    uint32_t grid = uint32_t((n + kThreads - 1) / kThreads);
    if (grid > 148 * 16) grid = 148 * 16;
    k_directed_max<<<grid, kThreads, 0, s>>>(from, to, d2, g, width, height, out_max);
}

} // namespace b200
