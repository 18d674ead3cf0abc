// Incremental candidate audit and four-gate verdicts.
//
// A collapse changes coverage only where the faces of faces(from) U faces(to)
// land, before or after. One warp audits one (candidate, view) unit, pulled
// from a global work queue: it projects the candidate's distinct local
// vertices (plus the placement), sets up the old and the new faces, rasterizes
// them over their joint bounding box to derive the candidate's per-sample face
// count from the resident state counts (count - old + new), builds coverage
// words with __ballot_sync, updates the XOR/OR popcounts against the resident
// reference mask, and measures the exact squared distance of every changed
// sample by a row scan over coverage words. The result equals a full
// re-raster of the candidate (evaluate.cpp:125-209) sample for sample.
#include "kernels.cuh"
#include "nearest.cuh"

namespace b200 {
namespace {

constexpr int kAuditWarps = 8;
#ifndef B200_AUDIT_MIN_BLOCKS
#define B200_AUDIT_MIN_BLOCKS 3 // resident blocks per SM the register budget targets
#endif
constexpr int kMaxOk = 48;          // rasterized (unculled, unclipped) old + new faces
constexpr uint32_t kDirectTests = 4096; // bbox samples up to which phase 1 tests every sample
constexpr uint32_t kHeavyUnit = 512;    // changed samples above which a warp-tier unit may spill

// Per-warp limits of one (candidate, view) unit. The common tier keeps its
// scratch small so that many warps stay resident; units that overflow it are
// spilled to the large tier (few warps per SM, 256 x 256-sample regions).
struct LimitsSmall {
    static constexpr bool kWordRows = false; // region phase over coverage words
    static constexpr int kRegionWords = 4;     // region width <= 128 samples after 32-alignment
    static constexpr int kRegionRows = 64;     // region height
    static constexpr int kDeltaSamples = 2048; // region samples (unaligned bbox) with a count delta
    static constexpr int kQueue = 160;         // reference-only samples of affected tiles (>= 64)
    static constexpr int kAffected = 8;        // tiles outside the region whose distances may change
};
// A wider warp tier for workloads whose units often overflow the small one
// (one block of 8 warps per SM instead of three).
struct LimitsMedium {
    static constexpr bool kWordRows = true; // region phase over coverage words
    static constexpr int kRegionWords = 8;
    static constexpr int kRegionRows = 128;
    static constexpr int kDeltaSamples = 8192;
    static constexpr int kQueue = 640;
    static constexpr int kAffected = 16;
};
struct LimitsLarge {
    static constexpr bool kWordRows = true; // region phase over coverage words
    static constexpr int kRegionWords = 8;
    static constexpr int kRegionRows = 256;
    static constexpr int kDeltaSamples = 32768;
    static constexpr int kQueue = 4096;
    static constexpr int kAffected = 32;
};
constexpr int kLargeWarps = 3; // warps per block of the large tier
// The huge tier keeps its per-warp scratch in global memory (L2-resident
// working set per unit): regions up to 1024 x 1024 samples.
struct LimitsHuge {
    static constexpr bool kWordRows = true; // region phase over coverage words
    static constexpr int kRegionWords = 32;
    static constexpr int kRegionRows = 1024;
    static constexpr int kDeltaSamples = 16384; // direct-test units only
    static constexpr int kQueue = 65536;
    static constexpr int kAffected = 64;
};
constexpr int kHugeWarps = 8;
// The giant tier: any region of a raster up to 4160 x 4160 (512 px x ss 8),
// for the rare units beyond the huge tier; few warps, global scratch.
struct LimitsGiant {
    static constexpr bool kWordRows = true; // region phase over coverage words
    static constexpr int kRegionWords = 136;
    static constexpr int kRegionRows = 4160;
    static constexpr int kDeltaSamples = 16384;
    static constexpr int kQueue = 65536;
    static constexpr int kAffected = 64;
};
constexpr int kGiantWarps = 8;

template <class L> struct alignas(16) WarpScratch {
    double vx[32], vy[32], vz[32]; // projected local vertices; 31 = placement
    FaceSetup faces[kMaxOk];       // old faces carry pad = -1, new faces pad = +1
    uint32_t work[kMaxOk];         // exclusive prefix of bbox samples per face
    uint32_t affected[L::kAffected];
    uint32_t qcount[4];            // [0]: flipped samples queued
    uint32_t region[L::kRegionRows * L::kRegionWords]; // candidate XOR state coverage
    uint32_t delta[L::kDeltaSamples / 4]; // per-sample count delta + 128, one byte each
    uint32_t queue[L::kQueue];
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ uint32_t size_mask(uint32_t size, uint32_t chunk) {
    uint32_t rem = size - chunk * 32;
    return rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
}
// Columns [32*chunk, 32*chunk+32) of `row` from a linear bit stream (one
// padding word at the end of every mask keeps the second load in bounds).
__device__ __forceinline__ uint32_t chunk_global(const uint32_t* bits, uint32_t size, uint32_t row, uint32_t chunk) {
    size_t b = size_t(row) * size + size_t(chunk) * 32;
    uint32_t sh = uint32_t(b & 31);
    size_t w = b >> 5;
    uint32_t v = bits[w];
    if (sh) v = (v >> sh) | (bits[w + 1] << (32 - sh));
    return v & size_mask(size, chunk);
}

// The candidate's coverage: the state's, with the region's flipped samples
// (region words: candidate XOR state) applied.
struct CandMask {
    const uint32_t* state;
    const uint32_t* region;
    uint32_t size, y0, y1, c0, words;
    __device__ uint32_t chunk(uint32_t row, uint32_t c) const {
        const uint32_t w = chunk_global(state, size, row, c);
        if (row >= y0 && row <= y1 && c >= c0 && c < c0 + words) return w ^ region[(row - y0) * words + (c - c0)];
        return w;
    }
};
struct RefMask {
    const uint32_t* bits;
    uint32_t size;
    __device__ uint32_t chunk(uint32_t row, uint32_t c) const { return chunk_global(bits, size, row, c); }
};

__device__ __forceinline__ bool pv_ref_bit(const uint32_t* bits, size_t i) { return (bits[i >> 5] >> (i & 31)) & 1u; }

__device__ __forceinline__ void record_write(ViewRecord* out, const ViewRecord& r) {
    if (lane_id() == 0) *out = r;
}

// Rows of interval ends kept per pass of the word-row region phase.
constexpr int kPassRows = 8; // a pass's row fits 3 bits of the (row, face) item table
// Tables of region_word_rows after its interval ends (kPassRows * kMaxOk
// short2): the pass's (row, face) items (kPassRows * kMaxOk u16) and its
// word masks of the new and of the old faces (2 * kPassRows * 32 u32).
constexpr size_t kPassTableBytes = kPassRows * kMaxOk * 2 + 2 * kPassRows * 32 * 4;
// Shared memory of one warp of the global tiers: face setups, interval ends
// and the tables above.
constexpr size_t kGlobalTierWarpSmem = kMaxOk * sizeof(FaceSetup) + kPassRows * kMaxOk * 4 + kPassTableBytes;

// Region phase over coverage words (every tier but the small one),
// kPassRows rows at a time. Per (row, face) the covered samples are one
// interval (exact FP64 searches from a single-precision guess of each
// edge's crossing, face_interval_guess). A pass computes them for
// the (row, face) pairs whose row the face spans, spread evenly over the
// lanes (the pairs listed in `pairs`, face-major), and keeps them in `iv`
// (shared memory; empty for the other pairs). Each interval is then OR-ed
// into the pass's word masks in shared memory: the union of the new faces
// (B) and of the old faces (A); lanes own (row, word) cells, up to eight
// each. Because the state's count pc includes every old face (pc >= A), the
// candidate's count pc - A + B is positive wherever B > 0, and where B = 0
// it is pc - A. So a sample flips iff it is newly covered (B on a
// state-empty sample, from the state's coverage word alone) or it loses its
// last faces (A without B, and pc equal to the number of old faces covering
// it: the only samples whose state count is read, and whose old faces are
// counted from the intervals). The cells' coverage words are all loaded
// before any is used, and the next pass's rows are prefetched into L2 while
// this one runs. Flipped samples are written to the region words (candidate
// XOR state) and counted into the popcount deltas against the reference.
// `clk` (profiling only) accumulates SM cycles of the interval, mask and
// word steps and of the lane's lost-sample counts.
__device__ void region_word_rows(const FaceSetup* faces, uint32_t nok, int wx0, int ry0, int ry1, int words,
                                 const PlanView& pv, uint32_t size, bool same_ref, uint32_t* region, short2* iv,
                                 uint16_t* pairs, int& dchg, int& dtot, int& dcov, int& flips, bool& negative,
                                 long long* clk) {
    const uint32_t lane = lane_id();
    long long t0 = clk ? clock64() : 0;
    static_assert(kPassRows == 8 && kMaxOk < 8192, "item = face << 3 | row");
    uint32_t* const bn = reinterpret_cast<uint32_t*>(pairs + kPassRows * kMaxOk); // [kPassRows][32] new-face union
    uint32_t* const an = bn + kPassRows * 32;                                      // [kPassRows][32] old-face union
    // Prefetch (to L2) of the state and reference words of rows [y, y + 8):
    // lanes 0-15 the state's, 16-31 the reference's, two per row (the lines
    // of the region's first and last word in the row).
    auto prefetch_rows = [&](int y) {
        const int row = y + int((lane >> 1) & 7u);
        const bool ref = lane >= 16;
        if (row > ry1 || (ref && same_ref)) return;
        const uint32_t* bits = ref ? pv.ref_bits : pv.state_bits;
        const size_t first = (size_t(row) * size + size_t(wx0)) >> 5;
        const uint32_t* at = bits + first + ((lane & 1u) ? size_t(words - 1) : 0);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(at));
    };
    prefetch_rows(ry0);
    for (int ybase = ry0; ybase <= ry1; ybase += kPassRows) {
        const int ylast = min(ry1, ybase + kPassRows - 1);
        const uint32_t pass_rows = uint32_t(ylast - ybase + 1);
        if (ybase + kPassRows <= ry1) prefetch_rows(ybase + kPassRows);
        // Rows of the pass that faces lane and lane + 32 span; their
        // exclusive prefix over faces numbers the pass's (row, face) items.
        auto first_row = [&](uint32_t f) { return max(faces[f].y0, ybase); };
        auto span = [&](uint32_t f) {
            const int lo = first_row(f), hi = min(faces[f].y1, ylast);
            return lo <= hi ? uint32_t(hi - lo + 1) : 0u;
        };
        const uint32_t n0 = lane < nok ? span(lane) : 0u, n1 = lane + 32 < nok ? span(lane + 32) : 0u;
        uint32_t s0 = n0, s1 = n1;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t a = __shfl_up_sync(0xffffffffu, s0, o), b = __shfl_up_sync(0xffffffffu, s1, o);
            if (lane >= uint32_t(o)) s0 += a, s1 += b;
        }
        const uint32_t tot0 = __shfl_sync(0xffffffffu, s0, 31);
        const uint32_t items = tot0 + __shfl_sync(0xffffffffu, s1, 31);
        for (uint32_t f = lane; f < nok; f += 32) {
            const uint32_t at = f < 32 ? s0 - n0 : tot0 + s1 - n1, n = f < 32 ? n0 : n1;
            const uint32_t r0 = uint32_t(first_row(f) - ybase);
            for (uint32_t j = 0; j < n; ++j) pairs[at + j] = uint16_t(f << 3 | (r0 + j));
            for (uint32_t r = 0; r < pass_rows; ++r) iv[r * kMaxOk + f] = make_short2(1, 0);
        }
        __syncwarp();
        auto item = [&](uint32_t t, uint32_t& f, uint32_t& r) {
            const uint32_t p = pairs[t];
            f = p >> 3, r = p & 7u;
        };
        for (uint32_t t = lane; t < items; t += 32) {
            uint32_t f, r;
            item(t, f, r);
            int lo, hi;
            face_interval_guess(faces[f], double(ybase + int(r)) + .5, lo, hi);
            iv[r * kMaxOk + f] = make_short2(short(lo), short(hi));
        }
        __syncwarp();
        if (clk) {
            const long long t = clock64();
            clk[0] += t - t0, t0 = t;
        }
        for (int c0 = 0; c0 < words; c0 += 32) { // 32-word windows of wide regions
            const uint32_t cn = uint32_t(min(32, words - c0));
            const int xc0 = wx0 + 32 * c0;
            const uint32_t cells = pass_rows * cn;
            // The pass's word masks: every (row, face) interval OR-ed into
            // the words it spans; lanes then own (row, word) cells:
            // t = lane + 32k, up to eight.
            const int xc1 = wx0 + 32 * (c0 + int(cn)) - 1;
            for (uint32_t k = lane; k < 2 * kPassRows * 32; k += 32) bn[k] = 0;
            __syncwarp();
            for (uint32_t t = lane; t < items; t += 32) {
                uint32_t f, r;
                item(t, f, r);
                const short2 e = iv[r * kMaxOk + f];
                const int lo = max(int(e.x), xc0), hi = min(int(e.y), xc1);
                if (lo > hi) continue;
                uint32_t* dst = (faces[f].pad > 0 ? bn : an) + r * 32;
                for (int w = (lo - xc0) >> 5; w <= (hi - xc0) >> 5; ++w) {
                    const int xb = xc0 + 32 * w, a = max(lo, xb) - xb, z = min(hi, xb + 31) - xb;
                    atomicOr(dst + w, (z == 31 ? 0xffffffffu : ((2u << z) - 1u)) & ~((1u << a) - 1u));
                }
            }
            __syncwarp();
            if (clk) {
                const long long t = clock64();
                clk[1] += t - t0, t0 = t;
            }
            uint32_t S[8], R[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t t = lane + 32u * uint32_t(k);
                S[k] = R[k] = 0;
                if (t < cells) {
                    const uint32_t r = t / cn, w = t - r * cn;
                    if (bn[r * 32 + w] | an[r * 32 + w]) {
                        const uint32_t y = uint32_t(ybase) + r, cw = (uint32_t(xc0) >> 5) + w;
                        S[k] = chunk_global(pv.state_bits, size, y, cw);
                        R[k] = same_ref ? S[k] : chunk_global(pv.ref_bits, size, y, cw);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t t = lane + 32u * uint32_t(k);
                if (t >= cells) break;
                const uint32_t r = t / cn, w = t - r * cn;
                const uint32_t bnew = bn[r * 32 + w], aany = an[r * 32 + w];
                uint32_t* out = region + (uint32_t(ybase) + r - uint32_t(ry0)) * uint32_t(words) + uint32_t(c0) + w;
                if (!(bnew | aany)) {
                    *out = 0;
                    continue;
                }
                const int y = ybase + int(r), xb = xc0 + 32 * int(w);
                const uint32_t grown = bnew & ~S[k];   // newly covered
                uint32_t lost_cand = aany & ~bnew;     // covered only if other faces cover it
                negative |= (lost_cand & ~S[k]) != 0;  // pc >= A > 0 must hold
                lost_cand &= S[k];
                uint32_t lost = 0;
                const long long l0 = clk && lost_cand ? clock64() : 0;
                while (lost_cand) {
                    const int i = __ffs(lost_cand) - 1;
                    lost_cand &= lost_cand - 1;
                    const int x = xb + i;
                    uint32_t n_old = 0; // old faces covering (x, y)
                    for (uint32_t f = 0; f < nok; ++f) {
                        const short2 e = iv[r * kMaxOk + f];
                        n_old += faces[f].pad < 0 && int(e.x) <= x && x <= int(e.y);
                    }
                    const uint32_t pc = pv.state_count[size_t(y) * size + size_t(x)];
                    negative |= pc < n_old;
                    if (pc == n_old) lost |= 1u << i;
                }
                if (l0) clk[3] += clock64() - l0;
                const uint32_t fl = grown | lost;
                *out = fl;
                if (!fl) continue;
                flips += __popc(fl);
                dcov += __popc(grown) - __popc(lost);
                const uint32_t X = S[k] ^ R[k];
                dchg += __popc(fl & ~X) - __popc(fl & X);
                dtot += __popc(fl & ~R[k] & ~S[k]) - __popc(fl & ~R[k] & S[k]);
            }
            __syncwarp();
            if (clk) {
                const long long t = clock64();
                clk[2] += t - t0, t0 = t;
            }
        }
    }
}

// `spill` (small tier only): units that overflow the tier's limits append
// their unit index `u` there for the large tier instead of falling back, or
// to `far` (may be null) when their region is beyond the huge tier's.
template <class L>
__device__ void audit_unit(const CandidateRecord* __restrict__ rec, const PlanDev& plan, uint32_t v,
                           WarpScratch<L>& ws, ViewRecord* out, unsigned long long* stats, uint32_t u,
                           uint32_t* spill, uint32_t heavy = 0xffffffffu, FaceSetup* face_table = nullptr,
                           short2* iv_table = nullptr, uint16_t* pair_table = nullptr, uint32_t* far = nullptr) {
    // The face setups: in the warp's scratch, or in shared memory for the
    // tiers whose scratch is global (the row sweep reads them every row).
    FaceSetup* const faces = face_table ? face_table : ws.faces;
    // Every tier but the small one runs the region phase over coverage words
    // (region_word_rows; its interval and item tables in the warp's shared
    // memory: given by the global tiers, else the delta map's space) and the
    // distance phase walks the region words.
    constexpr bool word_rows = L::kWordRows;
    static_assert(!L::kWordRows || L::kDeltaSamples * sizeof(uint8_t) >= kPassRows * kMaxOk * 4 + kPassTableBytes,
                  "the delta map's space holds the word-row tables");
    short2* const iv_rows = iv_table ? iv_table : reinterpret_cast<short2*>(ws.delta);
    uint16_t* const pair_rows = pair_table ? pair_table : reinterpret_cast<uint16_t*>(ws.delta + kPassRows * kMaxOk);
    constexpr int kRegionWords = L::kRegionWords, kRegionRows = L::kRegionRows;
    constexpr int kDeltaSamples = L::kDeltaSamples, kQueue = L::kQueue, kAffected = L::kAffected;
    const uint32_t lane = lane_id();
    const long long t_start = stats ? clock64() : 0;
    const PlanView pv = plan.views[v];
    const uint32_t size = plan.size;
    ViewRecord r;
    r.pad = 0;
    r.flags = pv.clipped_ref ? kRecClippedRef : 0;
    r.ca = pv.cov_ref > 0;
    r.max_d2 = 0, r.changed = 0, r.total = 0, r.cb = 0;
    const bool same_ref = plan.state_is_ref != 0; // state words equal reference words
    if (!same_ref && !pv.tile_t1) {
        // Without tile maxima a state that differs from the reference needs
        // the full distance field.
        r.flags |= kRecFallback;
        record_write(out, r);
        return;
    }
    const Camera cam = plan.cameras[v];
    const uint32_t nverts = rec->nverts, nfaces = rec->nfaces;
    // Project the local vertices and the placement once.
    if (lane < nverts || lane == kPlacementLocal) {
        float px, py, pz;
        if (lane == kPlacementLocal) px = rec->placement[0], py = rec->placement[1], pz = rec->placement[2];
        else px = rec->verts[3 * lane], py = rec->verts[3 * lane + 1], pz = rec->verts[3 * lane + 2];
        Proj p = project(px, py, pz, plan.center, cam, plan.ss, size);
        ws.vx[lane] = p.x, ws.vy[lane] = p.y, ws.vz[lane] = p.z;
    }
    __syncwarp();
    // Face setups, old faces first, then the candidate's faces; the rasterized
    // ones are compacted into faces (old carry -1, new +1).
    const uint32_t below = (1u << lane) - 1u;
    const uint8_t fl = lane < nfaces ? rec->flags[lane] : 0;
    const bool two = plan.force_two || (fl & kFaceTwo);
    int x0 = 1 << 30, y0 = 1 << 30, x1 = -1, y1 = -1;
    uint32_t n_old, nok;
    int clip_delta;
    {
        bool ok = false, clip = false;
        FaceSetup s;
        if (lane < nfaces) {
            Proj a[3];
            for (int j = 0; j < 3; ++j) {
                uint32_t k = rec->old_face[3 * lane + j];
                a[j] = Proj{ws.vx[k], ws.vy[k], ws.vz[k]};
            }
            s = setup_face(a[0], a[1], a[2], cam.perspective != 0, two, size);
            ok = s.status == kFaceOk;
            clip = s.status == kFaceClipZ || s.status == kFaceClipBox;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        n_old = __popc(m);
        clip_delta = -__popc(__ballot_sync(0xffffffffu, clip));
        const uint32_t slot = __popc(m & below);
        if (ok && slot < uint32_t(kMaxOk)) {
            s.pad = -1;
            faces[slot] = s;
            x0 = s.x0, x1 = s.x1, y0 = s.y0, y1 = s.y1;
        }
    }
    {
        bool ok = false, clip = false;
        FaceSetup s;
        if (lane < nfaces && (fl & kFaceKept)) {
            Proj a[3];
            for (int j = 0; j < 3; ++j) {
                uint32_t k = rec->new_face[3 * lane + j];
                a[j] = Proj{ws.vx[k], ws.vy[k], ws.vz[k]};
            }
            s = setup_face(a[0], a[1], a[2], cam.perspective != 0, two, size);
            ok = s.status == kFaceOk;
            clip = s.status == kFaceClipZ || s.status == kFaceClipBox;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        nok = n_old + __popc(m);
        clip_delta += __popc(__ballot_sync(0xffffffffu, clip));
        const uint32_t slot = n_old + __popc(m & below);
        if (ok && slot < uint32_t(kMaxOk)) {
            s.pad = 1;
            faces[slot] = s;
            x0 = min(x0, s.x0), x1 = max(x1, s.x1), y0 = min(y0, s.y0), y1 = max(y1, s.y1);
        }
    }
    if (int64_t(pv.clip_state) + clip_delta > 0 || nok > uint32_t(kMaxOk)) {
        // A clipped candidate keeps the CPU's partial-raster values.
        r.flags |= kRecFallback | (int64_t(pv.clip_state) + clip_delta > 0 ? kRecClippedCand : 0);
        record_write(out, r);
        return;
    }
    for (int o = 16; o; o >>= 1) {
        x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    __syncwarp();
    const long long t_setup = stats ? clock64() : 0;
    // profiling only: region sub-phases (zeroing, direct path or row sweep,
    // the sweep's per-lane event and piece cycles, max over lanes)
    long long st_zero = 0, st_path = 0, st_events = 0, st_pieces = 0;
    int st_kind = -1, st_rows = 0;
    long long st_words = 0, st_lost = 0;
    int dchg = 0, dtot = 0, dcov = 0;
    uint32_t qn = 0, region_changed = 0, nflips = 0;
    int region_words = 0;
    bool fallback = false, beyond_huge = false;
    CandMask cmask;
    cmask.state = pv.state_bits;
    cmask.region = ws.region;
    cmask.size = size;
    uint64_t samples = 0, face_samples = 0;
    // The processed region: the changed faces' bbox widened to whole coverage
    // words; when the state differs from the reference, widened to whole
    // 32x32 tiles so every tile is either fully processed or fully outside.
    const int wx0 = x0 & ~31;
    const int ry0 = same_ref ? y0 : (y0 & ~31);
    const int ry1 = same_ref ? y1 : min(int(size) - 1, y1 | 31);
    const int words = x1 >= 0 ? ((x1 - wx0) >> 5) + 1 : 0;
    if (x1 >= 0) {
        const int rows = ry1 - ry0 + 1;
        cmask.y0 = uint32_t(ry0), cmask.y1 = uint32_t(ry1), cmask.c0 = uint32_t(wx0 >> 5), cmask.words = uint32_t(words);
        const int bw = x1 - x0 + 1, bh = y1 - y0 + 1;
        const int bws = (bw + 15) & ~15; // delta map row stride: whole 16-byte vectors
        // Sum of the faces' bbox areas: small units test every (face, sample
        // of its bbox) into a byte difference map; the others sweep rows.
        uint32_t area = 0;
        if (lane < nok) area += uint32_t(faces[lane].x1 - faces[lane].x0 + 1) * uint32_t(faces[lane].y1 - faces[lane].y0 + 1);
        if (lane + 32 < nok)
            area += uint32_t(faces[lane + 32].x1 - faces[lane + 32].x0 + 1) *
                    uint32_t(faces[lane + 32].y1 - faces[lane + 32].y0 + 1);
        for (int o = 16; o; o >>= 1) area += __shfl_xor_sync(0xffffffffu, area, o);
        face_samples = area;
        // The small tier (regions of at most 128 x 64 samples) always tests
        // every sample; a unit whose delta map does not fit goes on to the
        // next tier.
        constexpr bool kSweep = kDeltaSamples > 2048;
        const bool direct =
            !kSweep || (area <= kDirectTests && uint32_t(bws) * uint32_t(bh) <= uint32_t(kDeltaSamples));
        if (words > kRegionWords || rows > kRegionRows ||
            (!kSweep && uint32_t(bws) * uint32_t(bh) > uint32_t(kDeltaSamples))) {
            fallback = true;
            beyond_huge = words > LimitsHuge::kRegionWords || rows > LimitsHuge::kRegionRows;
        } else {
            samples = uint64_t(rows) * uint64_t(words) * 32;
            // ws.region holds the candidate's coverage words XOR the state's
            // over the region (its flipped samples). The word-row pass writes
            // every word itself; the other paths flip bits of zeroed words.
            const int nwords = rows * words;
            if (!word_rows)
                for (int k = int(lane); k < nwords; k += 32) ws.region[k] = 0;
            if (lane == 0) ws.qcount[0] = 0;
            __syncwarp();
            const long long t_zero = stats ? clock64() : 0;
            long long c_events = 0, c_pieces = 0;
            long long wr_clk[4] = {0, 0, 0, 0}; // word rows: intervals, masks, words, lost samples
            bool negative = false;
            int flips = 0;
            // A sample whose count changes by dv (state count pc): it flips
            // where covered-ness changes; each flip moves the popcounts
            // against the reference by one sample. With the state equal to
            // the reference every changed sample of the region is a flip, and
            // flips go to the queue for the distance phase (bit 31: covered by
            // the candidate).
            auto visit = [&](int x, int y, int dv, int pc, bool shared_rows) {
                const int cc = pc + dv;
                negative |= cc < 0;
                if ((cc > 0) == (pc > 0)) return;
                const bool P = pc > 0, C = !P;
                const bool R = same_ref ? P : pv_ref_bit(pv.ref_bits, size_t(y) * size + size_t(x));
                dcov += C ? 1 : -1;
                dchg += int(C != R) - int(P != R);
                dtot += int(C || R) - int(P || R);
                const uint32_t xr = uint32_t(x - wx0), yr = uint32_t(y - ry0);
                uint32_t* word = &ws.region[yr * uint32_t(words) + (xr >> 5)];
                if (shared_rows) atomicXor(word, 1u << (xr & 31));
                else *word ^= 1u << (xr & 31);
                ++flips;
                if (same_ref) {
                    const uint32_t pos = atomicAdd(&ws.qcount[0], 1u);
                    if (pos < uint32_t(kQueue)) ws.queue[pos] = xr | (yr << 15) | (C ? 0x80000000u : 0u);
                }
            };
            if constexpr (word_rows) {
                region_word_rows(faces, nok, wx0, ry0, ry1, words, pv, size, same_ref, ws.region, iv_rows, pair_rows,
                                 dchg, dtot, dcov, flips, negative, stats ? wr_clk : nullptr);
            } else if (direct) {
                const uint32_t delta_words = uint32_t(bws * bh) >> 2;
                for (uint32_t k = lane; k < delta_words; k += 32) ws.delta[k] = 0x80808080u;
                uint32_t c0 = 0, c1 = 0;
                if (lane < nok)
                    c0 = uint32_t(faces[lane].x1 - faces[lane].x0 + 1) * uint32_t(faces[lane].y1 - faces[lane].y0 + 1);
                if (lane + 32 < nok)
                    c1 = uint32_t(faces[lane + 32].x1 - faces[lane + 32].x0 + 1) *
                         uint32_t(faces[lane + 32].y1 - faces[lane + 32].y0 + 1);
                uint32_t i0 = c0, i1 = c1;
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t a = __shfl_up_sync(0xffffffffu, i0, o), b = __shfl_up_sync(0xffffffffu, i1, o);
                    if (lane >= uint32_t(o)) i0 += a, i1 += b;
                }
                const uint32_t tot0 = __shfl_sync(0xffffffffu, i0, 31);
                if (lane < nok) ws.work[lane] = i0 - c0;
                if (lane + 32 < nok) ws.work[lane + 32] = tot0 + i1 - c1;
                const uint32_t items = tot0 + __shfl_sync(0xffffffffu, i1, 31);
                __syncwarp();
                for (uint32_t t = lane; t < items; t += 32) {
                    uint32_t f = 0; // last face whose prefix is <= t
                    for (uint32_t step = 32; step; step >>= 1)
                        if (f + step < nok && ws.work[f + step] <= t) f += step;
                    const FaceSetup& s = faces[f];
                    const uint32_t fw = uint32_t(s.x1 - s.x0 + 1), r = t - ws.work[f];
                    const int fy = s.y0 + int(r / fw), fx = s.x0 + int(r % fw);
                    if (face_covers(s, fx, fy)) {
                        const uint32_t d = uint32_t(fy - y0) * uint32_t(bws) + uint32_t(fx - x0);
                        const uint32_t unit = 1u << (8 * (d & 3));
                        if (s.pad > 0) atomicAdd(&ws.delta[d >> 2], unit);
                        else atomicSub(&ws.delta[d >> 2], unit);
                    }
                }
                __syncwarp();
                const float inv_bws = 1.0f / float(bws);
                for (uint32_t k = lane; k < delta_words; k += 32) {
                    const uint32_t dw = ws.delta[k];
                    if (dw == 0x80808080u) continue;
                    for (uint32_t j = 0; j < 4; ++j) {
                        const int dv = int((dw >> (8 * j)) & 0xffu) - 128;
                        const uint32_t d = 4 * k + j;
                        if (!dv) continue;
                        uint32_t q = uint32_t(float(d) * inv_bws); // row in the bbox, corrected below
                        while (q * uint32_t(bws) > d) --q;
                        while ((q + 1) * uint32_t(bws) <= d) ++q;
                        if (d - q * uint32_t(bws) >= uint32_t(bw)) continue; // row padding
                        const int y = y0 + int(q), x = x0 + int(d - q * uint32_t(bws));
                        visit(x, y, dv, int(pv.state_count[size_t(y) * size + size_t(x)]), true);
                    }
                }
            } else if constexpr (kSweep) {
                // Row sweep, one bbox row per lane. Per face crossing the row
                // the covered samples form one interval: each edge term of
                // the reference's test is monotone in x (IEEE rounding is
                // monotone), so binary searches over the same FP64
                // expressions find its ends exactly. The sorted interval ends
                // (+1 at a new face's start and an old face's end, -1 at the
                // others) give the count delta piecewise; only samples of
                // pieces with a non-zero delta read their state count (four
                // per load).
                for (int y = y0 + int(lane); y <= y1; y += 32) {
                    const long long r0 = stats ? clock64() : 0;
                    uint32_t ev[2 * kMaxOk];
                    int n = 0;
                    auto insert = [&](uint32_t e) {
                        int i = n++;
                        while (i > 0 && ev[i - 1] > e) {
                            ev[i] = ev[i - 1];
                            --i;
                        }
                        ev[i] = e;
                    };
                    const double py = double(y) + .5;
                    for (uint32_t f = 0; f < nok; ++f) {
                        const FaceSetup& s = faces[f];
                        if (y < s.y0 || y > s.y1) continue;
                        int lo, hi;
                        face_interval(s, py, lo, hi);
                        if (lo > hi) continue;
                        const uint32_t up = s.pad > 0 ? 1u : 0u;
                        insert((uint32_t(lo) << 1) | up);
                        insert((uint32_t(hi + 1) << 1) | (up ^ 1u));
                    }
                    const long long r1 = stats ? clock64() : 0;
                    c_events += r1 - r0;
                    // Pieces with a non-zero delta go in groups of four: the
                    // groups' first count words are loaded together. A count
                    // word is the aligned 4-byte word holding x (view buffers
                    // start 4-aligned and are padded to 4).
                    const size_t row_at = size_t(y) * size;
                    auto count_word = [&](int x) {
                        return *reinterpret_cast<const uint32_t*>(pv.state_count + ((row_at + size_t(x)) & ~size_t(3)));
                    };
                    int pa[4], pb[4], pd[4], np = 0;
                    auto flush = [&]() {
                        uint32_t w[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) w[q] = q < np ? count_word(pa[q]) : 0u;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            if (q >= np) break;
                            uint32_t w4 = w[q];
                            for (int x = pa[q]; x < pb[q];) {
                                for (uint32_t j = uint32_t((row_at + size_t(x)) & 3); j < 4 && x < pb[q]; ++j, ++x)
                                    visit(x, y, pd[q], int((w4 >> (8 * j)) & 0xffu), false);
                                if (x < pb[q]) w4 = count_word(x);
                            }
                        }
                        np = 0;
                    };
                    int acc = 0;
                    for (int i = 0; i < n; ++i) {
                        acc += (ev[i] & 1u) ? 1 : -1;
                        if (!acc) continue;
                        const int xa = int(ev[i] >> 1), xb = i + 1 < n ? int(ev[i + 1] >> 1) : x1 + 1;
                        if (xa >= xb) continue;
                        pa[np] = xa, pb[np] = xb, pd[np] = acc;
                        if (++np == 4) flush();
                    }
                    flush();
                    if (stats) c_pieces += clock64() - r1;
                }
            }
            if (stats) {
                st_zero = t_zero - t_setup;
                st_path = clock64() - t_zero;
                st_kind = word_rows ? 2 : direct ? 0 : 1;
                st_rows = bh;
            }
            if (stats && word_rows) {
                for (int o = 16; o; o >>= 1) wr_clk[3] = max(wr_clk[3], __shfl_xor_sync(0xffffffffu, wr_clk[3], o));
                c_events = wr_clk[0], c_pieces = wr_clk[1], st_words = wr_clk[2], st_lost = wr_clk[3];
            }
            if (__any_sync(0xffffffffu, negative)) fallback = true;
            for (int o = 16; o; o >>= 1) {
                c_events = max(c_events, __shfl_xor_sync(0xffffffffu, c_events, o));
                c_pieces = max(c_pieces, __shfl_xor_sync(0xffffffffu, c_pieces, o));
            }
            st_events = c_events, st_pieces = c_pieces;
            for (int o = 16; o; o >>= 1) {
                dchg += __shfl_xor_sync(0xffffffffu, dchg, o);
                dtot += __shfl_xor_sync(0xffffffffu, dtot, o);
                dcov += __shfl_xor_sync(0xffffffffu, dcov, o);
                flips += __shfl_xor_sync(0xffffffffu, flips, o);
            }
            __syncwarp();
            region_words = nwords;
            nflips = uint32_t(flips);
            region_changed = nflips;
            // A unit with many changed samples goes to the next tier when
            // that one runs more warps per SM.
            if (spill && region_changed > heavy) fallback = true;
        }
    }
    __syncwarp();
    // Outside the region the candidate equals the state. State-only samples
    // keep their reference distance (tile maxima t1); reference-only samples
    // keep their state distance unless the region could hold their nearest
    // covered sample (a tile within sqrt(t2) of the changed bbox): those tiles
    // are searched again below.
    int32_t far1 = -1, far2 = -1;
    uint32_t naff = 0;
    if (!same_ref && !fallback) {
        const uint32_t tiles_x = (size + 31) / 32, ntiles = tiles_x * tiles_x;
        const uint32_t tc0 = uint32_t(wx0 >> 5), tc1 = tc0 + uint32_t(words) - 1;
        const uint32_t tr0 = uint32_t(ry0 >> 5), tr1 = uint32_t(ry1 >> 5);
        for (uint32_t base = 0; base < ntiles; base += 32) {
            const uint32_t k = base + lane;
            bool aff = false;
            if (k < ntiles) {
                const uint32_t tx = k % tiles_x, ty = k / tiles_x;
                const bool inside = words > 0 && tx >= tc0 && tx <= tc1 && ty >= tr0 && ty <= tr1;
                if (!inside) {
                    far1 = max(far1, pv.tile_t1[k]);
                    const int32_t t2 = pv.tile_t2[k];
                    if (t2 >= 0) {
                        if (x1 < 0) {
                            far2 = max(far2, t2);
                        } else {
                            const int64_t gx0 = int64_t(tx) * 32, gy0 = int64_t(ty) * 32;
                            const int64_t dx = max(int64_t(0), max(gx0 - x1, int64_t(x0) - (gx0 + 31)));
                            const int64_t dy = max(int64_t(0), max(gy0 - y1, int64_t(y0) - (gy0 + 31)));
                            if (dx * dx + dy * dy > int64_t(t2)) far2 = max(far2, t2);
                            else aff = true;
                        }
                    }
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, aff);
            const uint32_t pos = naff + __popc(m & below);
            if (aff && pos < uint32_t(kAffected)) ws.affected[pos] = k;
            naff += __popc(m);
        }
        for (int o = 16; o; o >>= 1) {
            far1 = max(far1, __shfl_xor_sync(0xffffffffu, far1, o));
            far2 = max(far2, __shfl_xor_sync(0xffffffffu, far2, o));
        }
        if (naff > uint32_t(kAffected)) fallback = true;
        __syncwarp();
        // Reference-only samples of affected tiles: one lane per tile row.
        for (uint32_t a = 0; a < naff && !fallback; ++a) {
            const uint32_t k = ws.affected[a], tx = k % tiles_x, ty = k / tiles_x;
            const uint32_t y = ty * 32 + lane;
            uint32_t bits = 0;
            if (y < size) bits = chunk_global(pv.ref_bits, size, y, tx) & ~cmask.chunk(y, tx);
            const uint32_t cnt = __popc(bits);
            uint32_t incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= uint32_t(o)) incl += t;
            }
            uint32_t pos = qn + incl - cnt;
            for (uint32_t b = bits; b; b &= b - 1, ++pos)
                if (pos < uint32_t(kQueue)) ws.queue[pos] = (tx * 32 + uint32_t(__ffs(b) - 1)) | (y << 15);
            qn += __shfl_sync(0xffffffffu, incl, 31);
            if (qn > uint32_t(kQueue)) fallback = true;
        }
        __syncwarp();
    }
    const long long t_region = stats ? clock64() : 0;
    r.changed = uint32_t(int64_t(pv.changed) + dchg);
    r.total = uint32_t(int64_t(pv.total) + dtot);
    r.cb = int64_t(pv.cov_state) + dcov > 0;
    uint32_t best = 0;
    if (!fallback && r.changed && r.ca && r.cb) {
        RefMask rmask{pv.ref_bits, size};
        // The running maximum (warp-wide after each round of 32 samples)
        // bounds every search: a sample whose nearest covered sample is
        // closer cannot raise it.
        best = uint32_t(max(max(far1, far2), 0));
        // Verdict-only calls (threshold predicate, evaluate.cu:1034-1169):
        // a sample nearer than `floor` cannot change any gate's verdict, so
        // its search may stop at any covered sample within it; a search
        // stops at `ceiling` (a farther nearest sample counts as ceiling + 1),
        // and once the maximum exceeds it every gate of the plan fails this
        // view and the view's searches stop. Exact calls: floor 0, ceiling
        // UINT32_MAX.
        const uint32_t floor_d2 = plan.d2_floor, ceiling_d2 = plan.d2_ceiling;
        // Reference-only samples of the affected tiles outside the region.
        for (uint32_t base = 0; base < qn && best <= ceiling_d2; base += 32) {
            const uint32_t k = base + lane;
            if (k < qn) {
                const uint32_t e = ws.queue[k];
                const uint32_t x = e & 0x7fffu, y = (e >> 15) & 0x7fffu;
                const uint32_t d = nearest_d2(cmask, x, y, max(best, floor_d2), ceiling_d2);
                best = d > best ? d : best;
            }
            for (int o = 16; o; o >>= 1) {
                const uint32_t y = __shfl_xor_sync(0xffffffffu, best, o);
                best = y > best ? y : best;
            }
        }
        __syncwarp();
        const uint32_t queued = same_ref ? nflips : 0;
        if (same_ref && !word_rows && queued <= uint32_t(kQueue)) {
            // The region's changed samples are its flips, queued in phase 2.
            // Candidate-only samples measure to the reference (resident field
            // or search), reference-only samples search the candidate.
            for (uint32_t base = 0; base < queued && best <= ceiling_d2; base += 32) {
                const uint32_t k = base + lane;
                if (k < queued) {
                    const uint32_t e = ws.queue[k];
                    const uint32_t x = uint32_t(wx0) + (e & 0x7fffu), y = uint32_t(ry0) + ((e >> 15) & 0x7fffu);
                    const uint32_t enough = max(best, floor_d2);
                    uint32_t d;
                    if (e >> 31)
                        d = pv.ref_field ? pv.ref_field[size_t(y) * size + x]
                                         : nearest_d2(rmask, x, y, enough, ceiling_d2);
                    else d = nearest_d2(cmask, x, y, enough, ceiling_d2);
                    best = d > best ? d : best;
                }
                for (int o = 16; o; o >>= 1) {
                    const uint32_t y = __shfl_xor_sync(0xffffffffu, best, o);
                    best = y > best ? y : best;
                }
            }
        } else {
            // Changed samples of the region from its coverage words, 32 words
            // per round: the round's masks and a prefix of their counts go to
            // shared memory and every lane takes samples by rank.
            const uint32_t cbase = uint32_t(wx0 >> 5);
            uint32_t* rmask_s = ws.queue;       // 32 xor masks (the queue is consumed)
            uint32_t* cmask_s = ws.queue + 32;  // 32 candidate words
            uint32_t* pre = ws.work;            // 33 prefix counts
            for (int base = 0; base < region_words && best <= ceiling_d2; base += 32) {
                const int k = base + int(lane);
                uint32_t xm = 0, Cw = 0;
                if (k < region_words) {
                    const uint32_t row = uint32_t(ry0 + k / words), cw = cbase + uint32_t(k % words);
                    const uint32_t Sw = chunk_global(pv.state_bits, size, row, cw);
                    Cw = Sw ^ ws.region[k];
                    xm = Cw ^ (same_ref ? Sw : chunk_global(pv.ref_bits, size, row, cw));
                }
                if (!__any_sync(0xffffffffu, xm != 0)) continue; // no changed sample in these 32 words
                const uint32_t cnt = __popc(xm);
                uint32_t incl = cnt;
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= uint32_t(o)) incl += t;
                }
                rmask_s[lane] = xm;
                cmask_s[lane] = Cw;
                pre[lane + 1] = incl;
                if (lane == 0) pre[0] = 0;
                const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                __syncwarp();
                for (uint32_t j = lane; j < total; j += 32) {
                    uint32_t w = 0; // last word whose prefix is <= j
                    for (uint32_t step = 16; step; step >>= 1)
                        if (pre[w + step] <= j) w += step;
                    const uint32_t m = rmask_s[w];
                    const uint32_t bit = __fns(m, 0, int(j - pre[w]) + 1);
                    const int kw = base + int(w);
                    const uint32_t ry = uint32_t(ry0 + kw / words), cw = uint32_t(kw % words);
                    const uint32_t x = uint32_t(wx0) + 32 * cw + bit;
                    const uint32_t enough = max(best, floor_d2);
                    uint32_t d;
                    if ((cmask_s[w] >> bit) & 1u)
                        d = pv.ref_field ? pv.ref_field[size_t(ry) * size + x]
                                         : nearest_d2(rmask, x, ry, enough, ceiling_d2);
                    else d = nearest_d2(cmask, x, ry, enough, ceiling_d2);
                    best = d > best ? d : best;
                }
                for (int o = 16; o; o >>= 1) {
                    const uint32_t y = __shfl_xor_sync(0xffffffffu, best, o);
                    best = y > best ? y : best;
                }
                __syncwarp();
            }
        }
    }
    r.max_d2 = best;
    if (fallback) r.flags |= kRecFallback;
    if (best >= kExactLimit) r.flags |= kRecLarge;
    if (lane == 0) {
        if (fallback && spill) {
            // a region beyond the huge tier's goes straight to the giant tier
            uint32_t* dst = far && beyond_huge ? far : spill;
            dst[1 + atomicAdd(dst, 1u)] = u;
        }
        *out = r;
        if (stats) {
            // profiling counters (kAuditStats slots): units, region samples,
            // searched samples; per tier units and SM cycles; SM cycles of the
            // face setup, the region phases and the distance phase; flips;
            // region sub-phases (zeroing; direct path cycles and units; row
            // sweep cycles and units, its event and piece cycles, rows; word
            // rows cycles and units, their interval, mask, word and
            // lost-sample cycles, rows); samples of the faces' bboxes (the
            // (face, sample) pairs a per-sample raster tests); per tier the
            // longest unit's SM cycles)
            const long long t_end = clock64();
            constexpr int tier = L::kRegionRows <= 128 ? 0 : L::kRegionRows <= 256 ? 1 : L::kRegionRows <= 1024 ? 2 : 3;
            atomicAdd(stats, 1ull);
            atomicAdd(stats + 1, (unsigned long long)samples);
            atomicAdd(stats + 2, (unsigned long long)(qn + region_changed));
            atomicAdd(stats + 3 + tier, 1ull);
            atomicAdd(stats + 7 + tier, (unsigned long long)(t_end - t_start));
            atomicMax(stats + 31 + tier, (unsigned long long)(t_end - t_start));
            atomicAdd(stats + 11, (unsigned long long)(t_setup - t_start));
            atomicAdd(stats + 12, (unsigned long long)(t_region - t_setup));
            atomicAdd(stats + 13, (unsigned long long)(t_end - t_region));
            atomicAdd(stats + 14, (unsigned long long)nflips);
            atomicAdd(stats + 15, (unsigned long long)st_zero);
            if (st_kind == 0) {
                atomicAdd(stats + 16, (unsigned long long)st_path);
                atomicAdd(stats + 17, 1ull);
            } else if (st_kind == 1) {
                atomicAdd(stats + 18, (unsigned long long)st_path);
                atomicAdd(stats + 19, 1ull);
                atomicAdd(stats + 20, (unsigned long long)st_events);
                atomicAdd(stats + 21, (unsigned long long)st_pieces);
                atomicAdd(stats + 22, (unsigned long long)st_rows);
            } else if (st_kind == 2) {
                atomicAdd(stats + 23, (unsigned long long)st_path);
                atomicAdd(stats + 24, 1ull);
                atomicAdd(stats + 25, (unsigned long long)st_events);
                atomicAdd(stats + 26, (unsigned long long)st_pieces);
                atomicAdd(stats + 27, (unsigned long long)st_words);
                atomicAdd(stats + 28, (unsigned long long)st_lost);
                atomicAdd(stats + 29, (unsigned long long)st_rows);
            }
            atomicAdd(stats + 30, (unsigned long long)face_samples);
        }
    }
    __syncwarp();
}

// Unit u of a job -> its plan, candidate record, output slot and local index.
// A job is one plan over one candidate array, or a table of entries (one per
// session of a batch) whose units are concatenated in entry order.
__device__ __forceinline__ void resolve_unit(const AuditJob& job, uint32_t u, const PlanDev*& plan,
                                             const CandidateRecord*& recs, ViewRecord*& out, uint32_t& local) {
    if (!job.entries) {
        plan = &job.plan, recs = job.recs, out = job.out, local = u;
        return;
    }
    uint32_t lo = 0, hi = job.nentries - 1;
    while (lo < hi) { // last entry whose first unit is <= u
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (job.entries[mid].first_unit <= u) lo = mid;
        else hi = mid - 1;
    }
    const AuditEntry& e = job.entries[lo];
    plan = &e.plan, recs = e.recs, out = e.out, local = u - uint32_t(e.first_unit);
}

// Persistent warps pull (candidate, view) units, candidate-major, from `queue`.
// kMulti = false: a single plan (kernel parameters only, no table lookup).
// L: the warp tier's limits; kMinBlocks: resident blocks the registers target.
template <bool kMulti, class L, int kMinBlocks>
__global__ void __launch_bounds__(kAuditWarps * 32, kMinBlocks)
    k_audit(const __grid_constant__ AuditJob job, unsigned long long* stats, uint32_t* queue, uint32_t* spill) {
    extern __shared__ __align__(16) unsigned char smem[];
    WarpScratch<L>& ws = reinterpret_cast<WarpScratch<L>*>(smem)[threadIdx.x >> 5];
    const uint32_t lane = lane_id();
    for (;;) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(queue, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= job.total) break;
        const PlanDev* plan = &job.plan;
        const CandidateRecord* recs = job.recs;
        ViewRecord* out = job.out;
        uint32_t lu = u;
        if (kMulti) resolve_unit(job, u, plan, recs, out, lu);
        const uint32_t c = lu / plan->nviews, v = lu - c * plan->nviews;
        const CandidateRecord* rec = recs + c;
        ViewRecord* slot = out + lu;
        if (!rec->valid || !rec->fast) {
            ViewRecord r{};
            r.flags = rec->valid ? kRecFallback : 0;
            record_write(slot, r);
            continue;
        }
        audit_unit(rec, *plan, v, ws, slot, stats, u, spill, job.heavy, nullptr, nullptr, nullptr, job.far);
    }
}

// The large tier: persistent warps over the spilled unit list {count,
// units}; what overflows it too is appended to `spill_next` (may be null).
__global__ void __launch_bounds__(kLargeWarps * 32, 1)
    k_audit_large(const __grid_constant__ AuditJob job, unsigned long long* stats, const uint32_t* spill,
                  uint32_t* cursor, uint32_t* spill_next) {
    extern __shared__ __align__(16) unsigned char smem[];
    WarpScratch<LimitsLarge>& ws = reinterpret_cast<WarpScratch<LimitsLarge>*>(smem)[threadIdx.x >> 5];
    const uint32_t lane = lane_id();
    const uint32_t count = spill[0];
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(cursor, 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= count) break;
        const uint32_t u = spill[1 + k];
        const PlanDev* plan;
        const CandidateRecord* recs;
        ViewRecord* out;
        uint32_t lu;
        resolve_unit(job, u, plan, recs, out, lu);
        const uint32_t c = lu / plan->nviews, v = lu - c * plan->nviews;
        audit_unit(recs + c, *plan, v, ws, out + lu, stats, u, spill_next);
    }
}

// The huge and giant tiers: the same over a spill list, each warp with its
// own slot of global scratch (`scratch`, one WarpScratch<L> per resident
// warp); what overflows goes to `spill_next` (may be null).
template <class L, int kWarps>
__global__ void __launch_bounds__(kWarps * 32, 3)
    k_audit_global(const __grid_constant__ AuditJob job, unsigned long long* stats, const uint32_t* spill,
                   uint32_t* cursor, unsigned char* scratch, uint32_t* spill_next) {
    // Dynamic shared memory, per warp: face setups, pass intervals, pass items.
    extern __shared__ __align__(16) unsigned char global_tier_smem[];
    const uint32_t wslot = threadIdx.x >> 5;
    unsigned char* mine = global_tier_smem + size_t(wslot) * kGlobalTierWarpSmem;
    FaceSetup* face_table = reinterpret_cast<FaceSetup*>(mine);
    short2* iv_table = reinterpret_cast<short2*>(mine + kMaxOk * sizeof(FaceSetup));
    uint16_t* pair_table = reinterpret_cast<uint16_t*>(mine + kMaxOk * sizeof(FaceSetup) + kPassRows * kMaxOk * 4);
    const uint32_t lane = lane_id();
    const uint32_t slot = blockIdx.x * kWarps + (threadIdx.x >> 5);
    WarpScratch<L>& ws = reinterpret_cast<WarpScratch<L>*>(scratch)[slot];
    const uint32_t count = spill[0];
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(cursor, 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= count) break;
        const uint32_t u = spill[1 + k];
        const PlanDev* plan;
        const CandidateRecord* recs;
        ViewRecord* out;
        uint32_t lu;
        resolve_unit(job, u, plan, recs, out, lu);
        const uint32_t c = lu / plan->nviews, v = lu - c * plan->nviews;
        audit_unit(recs + c, *plan, v, ws, out + lu, stats, u, spill_next, 0xffffffffu,
                   face_table, iv_table, pair_table);
    }
}

struct VerdictOut {
    uint8_t accepted, failed_gate, exact_path, resume_gate;
    uint32_t removed;
};

__global__ void k_verdicts(const ViewRecord* const* plan_records, const uint32_t* plan_views, const uint32_t* plan_ss,
                           const GateDev* gates, const CandidateRecord* recs, uint32_t n, VerdictOut* verdicts,
                           Measurement* measurements, uint32_t* exact_count) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const CandidateRecord& rec = recs[c];
    VerdictOut v{0, 0, 0, 0, rec.removed};
    Measurement* meas = measurements ? measurements + size_t(c) * 4 : nullptr;
    if (meas)
        for (int g = 0; g < 4; ++g) meas[g] = default_measurement();
    if (!rec.valid) {
        v.failed_gate = rec.failed;
        verdicts[c] = v;
        return;
    }
    bool accepted = true;
    for (int g = 0; g < 4 && accepted; ++g) {
        const GateDev gd = gates[g];
        const uint32_t views = plan_views[gd.plan], ss = plan_ss[gd.plan];
        const ViewRecord* rows = plan_records[gd.plan] + size_t(c) * views;
        Measurement m = default_measurement();
        m.supersample = gd.settings.supersample;
        bool exact = false;
        for (uint32_t vi = 0; vi < views; ++vi) {
            const ViewRecord r = rows[vi];
            if (r.flags & (kRecFallback | kRecLarge)) {
                exact = true;
                break;
            }
            Measurement cur = default_measurement();
            cur.worst_view = vi;
            finish_view(cur, r, gd.settings, ss, double(r.max_d2));
            if (!refinement_done(cur, gd.settings, ss)) {
                exact = true;
                break;
            }
            if (!aggregate_view(m, cur, vi)) break;
        }
        if (exact) {
            v.exact_path = 1;
            v.resume_gate = uint8_t(g);
            v.failed_gate = 0xff;
            atomicAdd(exact_count, 1u);
            accepted = false;
            break;
        }
        if (meas) meas[g] = m;
        if (!measurement_accepted(m)) {
            v.failed_gate = uint8_t(g + 1);
            accepted = false;
        }
    }
    v.accepted = accepted;
    verdicts[c] = v;
}
} // namespace

size_t audit_smem_bytes() { return kAuditWarps * sizeof(WarpScratch<LimitsSmall>); }
size_t audit_large_smem_bytes() { return kLargeWarps * sizeof(WarpScratch<LimitsLarge>); }
size_t audit_huge_scratch_bytes(uint32_t sms) { return size_t(sms) * kHugeWarps * sizeof(WarpScratch<LimitsHuge>); }
size_t audit_giant_scratch_bytes(uint32_t blocks) {
    return size_t(blocks) * kGiantWarps * sizeof(WarpScratch<LimitsGiant>);
}

namespace {
template <class K> void set_smem(K kernel, size_t bytes) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}
// Warp tier kernels: [variant][multi]
using AuditKernel = void (*)(AuditJob, unsigned long long*, uint32_t*, uint32_t*);
AuditKernel warp_tier(int variant, bool multi) {
    if (variant == kAuditTierMedium) return multi ? k_audit<true, LimitsMedium, 1> : k_audit<false, LimitsMedium, 1>;
    return multi ? k_audit<true, LimitsSmall, B200_AUDIT_MIN_BLOCKS> : k_audit<false, LimitsSmall, B200_AUDIT_MIN_BLOCKS>;
}
size_t warp_tier_smem(int variant) {
    return kAuditWarps * (variant == kAuditTierMedium ? sizeof(WarpScratch<LimitsMedium>) : sizeof(WarpScratch<LimitsSmall>));
}
} // namespace

void launch_audit(const AuditJob& job, unsigned long long* stats, uint32_t* queue, uint32_t* spill,
                  uint32_t* spill_huge, unsigned char* huge_scratch, uint32_t huge_blocks, cudaStream_t s,
                  int variant, const GiantTier* giant, cudaEvent_t* marks) {
    if (!job.total) return;
    static bool configured = false;
    const size_t large = audit_large_smem_bytes();
    if (!configured) {
        for (int v = 0; v < 2; ++v)
            for (int m = 0; m < 2; ++m) set_smem(warp_tier(v, m != 0), warp_tier_smem(v));
        set_smem(k_audit_large, large);
        set_smem(k_audit_global<LimitsHuge, kHugeWarps>, kHugeWarps * kGlobalTierWarpSmem);
        set_smem(k_audit_global<LimitsGiant, kGiantWarps>, kGiantWarps * kGlobalTierWarpSmem);
        configured = true;
    }
    const int tier = variant & 1;
    const AuditKernel kernel = warp_tier(tier, job.entries != nullptr);
    const size_t smem = warp_tier_smem(tier);
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kAuditWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = uint64_t(sms) * per_sm;
    uint64_t needed = (job.total + kAuditWarps - 1) / kAuditWarps;
    if (grid > needed) grid = needed;
    const bool huge = spill && spill_huge && huge_scratch && huge_blocks;
    const bool big = huge && giant && giant->spill && giant->scratch && giant->blocks;
    AuditJob tuned = job;
    tuned.heavy = (variant & kAuditSpillHeavy) && huge && huge_blocks >= uint32_t(sms) ? kHeavyUnit : 0xffffffffu;
    // units beyond the huge tier's regions go from the warp tier straight to
    // the giant tier, which takes them while the huge tier runs
    const bool far = big && giant->far;
    tuned.far = far ? giant->far : nullptr;
    cudaMemsetAsync(queue, 0, 20, s);
    if (spill) cudaMemsetAsync(spill, 0, 4, s);
    if (huge) cudaMemsetAsync(spill_huge, 0, 4, s);
    if (big) cudaMemsetAsync(giant->spill, 0, 4, s);
    if (far) cudaMemsetAsync(giant->far, 0, 4, s);
    uint32_t* next = big ? giant->spill : nullptr;
    if (marks) cudaEventRecord(marks[0], s);
    kernel<<<uint32_t(grid), kAuditWarps * 32, smem, s>>>(tuned, stats, queue, spill);
    if (marks) cudaEventRecord(marks[1], s);
    const bool beside = far && giant->side && giant->fork && giant->join;
    if (far) {
        cudaStream_t gs = s;
        if (beside) {
            cudaEventRecord(giant->fork, s);
            cudaStreamWaitEvent(giant->side, giant->fork, 0);
            gs = giant->side;
        }
        k_audit_global<LimitsGiant, kGiantWarps>
            <<<giant->blocks, kGiantWarps * 32, kGiantWarps * kGlobalTierWarpSmem, gs>>>(job, stats, giant->far,
                                                                                        queue + 4, giant->scratch,
                                                                                        nullptr);
        if (beside) cudaEventRecord(giant->join, giant->side);
    }
    if (huge && huge_blocks >= uint32_t(sms)) {
        // enough huge-tier warps: units the warp tier spills go there directly
        k_audit_global<LimitsHuge, kHugeWarps>
            <<<huge_blocks, kHugeWarps * 32, kHugeWarps * kGlobalTierWarpSmem, s>>>(job, stats, spill, queue + 1,
                                                                                   huge_scratch, next);
    } else {
        if (spill)
            k_audit_large<<<uint32_t(sms), kLargeWarps * 32, large, s>>>(job, stats, spill, queue + 1,
                                                                         huge ? spill_huge : nullptr);
        if (huge)
            k_audit_global<LimitsHuge, kHugeWarps>
                <<<huge_blocks, kHugeWarps * 32, kHugeWarps * kGlobalTierWarpSmem, s>>>(job, stats, spill_huge,
                                                                                       queue + 2, huge_scratch, next);
    }
    if (marks) cudaEventRecord(marks[2], s);
    if (beside) cudaStreamWaitEvent(s, giant->join, 0); // the giant scratch is free again
    if (big)
        k_audit_global<LimitsGiant, kGiantWarps>
            <<<giant->blocks, kGiantWarps * 32, kGiantWarps * kGlobalTierWarpSmem, s>>>(job, stats, giant->spill,
                                                                                       queue + 3, giant->scratch,
                                                                                       nullptr);
    if (marks) cudaEventRecord(marks[3], s);
}

void launch_verdicts(const ViewRecord* const* plan_records, const uint32_t* plan_views, const uint32_t* plan_ss,
                     const GateDev* gates, const CandidateRecord* records, uint32_t n, void* verdicts,
                     void* measurements, uint32_t* exact_count, cudaStream_t s) {
    if (!n) return;
    k_verdicts<<<(n + 127) / 128, 128, 0, s>>>(plan_records, plan_views, plan_ss, gates, records, n,
                                               static_cast<VerdictOut*>(verdicts),
                                               static_cast<Measurement*>(measurements), exact_count);
}

} // namespace b200
