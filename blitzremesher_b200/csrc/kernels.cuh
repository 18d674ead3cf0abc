// Device data layouts and kernel launchers of the candidate-audit engine.
#pragma once
#include "common.cuh"
#include "legality.cuh"
#include <cuda_runtime.h>

namespace b200 {

// Borrowed device view of one mesh state (FP32 master streams).
struct DevMesh {
    const float* pos;     // 3 per vertex slot
    const uint32_t* idx;  // 3 per face
    const uint16_t* mat;  // per face or null
    const uint8_t* sided; // per material or null
    const float* uv;      // 2 per vertex slot or null
    uint32_t nv, nf, nsided, pad;
};

// Topology on geometric classes (a class is named by its smallest slot).
struct DevTopology {
    const uint32_t* geometry;     // slot -> class root
    const uint32_t* canonical;    // slot -> attribute chart root
    const uint32_t* face_offsets; // class -> range in faces (nv+1)
    const uint32_t* faces;        // face per class corner, ascending per class
    const uint32_t* nbr_offsets;  // class -> range in neighbors (nv+1)
    const uint32_t* neighbors;    // sorted unique neighbour classes
    const uint8_t* nbr_count;     // face-edge multiplicity, capped at 3
    const uint8_t* boundary;      // class flags
    const uint8_t* invalid;
    const uint32_t* slot_offsets; // class -> range in slots (nv+1)
    const uint32_t* slots;        // vertex slots per class, ascending
};

// The legality view of a mesh state and its topology.
__host__ __device__ inline ClassRing class_ring(const DevMesh& m, const DevTopology& t) {
    return ClassRing{m.idx, m.mat, t.geometry, t.face_offsets, t.faces, t.nbr_offsets, t.neighbors, t.nbr_count,
                     t.boundary, t.invalid, m.nv, m.nf};
}

// Attribute charts for uv transport (place_vertices): the session's source
// mesh and, per canonical class of the source (position + uv weld with
// preserve_uv, the geometric classes without), its source faces in
// ascending order, each face once. uv == null: the mesh has no uv. flip:
// preserve_uv, which adds the uv orientation check of validate_placement.
struct UvSource {
    const float* pos;
    const float* uv;
    const uint32_t* idx;
    const uint32_t* offsets; // canonical class -> range in faces (nv + 1)
    const uint32_t* faces;
    bool flip;
};

// Slots of the audit kernels' profiling counters (launch_audit `stats`).
constexpr int kAuditStats = 35;

constexpr int kMaxAffected = 32; // faces in faces(from) U faces(to) handled on the fast path
constexpr int kMaxLocal = 31;    // distinct vertex slots of those faces; local index 31 = placement
constexpr uint8_t kPlacementLocal = 31;

// A candidate's neighbourhood: the distinct vertex slots of faces(from) U
// faces(to) with their current positions, each affected face as local corner
// indices before and after the collapse (moved corners point at the
// placement), whether it survives and whether its material is two-sided.
struct CandidateRecord {
    float placement[3];
    uint32_t from, to;
    uint8_t nverts, nfaces; // local vertices, affected faces
    uint8_t valid;          // legal + placement valid
    uint8_t fast;           // handled by the incremental path
    uint8_t removed;        // faces removed
    uint8_t failed;         // 5 illegal, 6 invalid placement
    uint8_t pad[2];
    float verts[kMaxLocal * 3];
    uint8_t old_face[kMaxAffected * 3];
    uint8_t new_face[kMaxAffected * 3];
    uint8_t flags[kMaxAffected]; // bit0 kept, bit1 two-sided
};
constexpr uint8_t kFaceKept = 1, kFaceTwo = 2;

// One audit plan: a reference, a camera set, a screen size and a sampling.
struct PlanView {
    const uint32_t* ref_bits;   // reference mask, CPU semantics (u64 layout as u32 words)
    const uint32_t* state_bits; // current state: count > 0
    const uint8_t* state_count; // current state: covering faces per sample
    const uint32_t* ref_field;  // exact squared distance to the reference mask, or null
    const int32_t* tile_t1;     // per 32x32 tile: max ref_field over state-only samples (-1 none)
    const int32_t* tile_t2;     // per 32x32 tile: max state field over reference-only samples
    uint32_t changed, total;    // state vs reference
    uint32_t cov_ref, cov_state;
    uint32_t clip_state;        // clipped faces of the state
    uint32_t clipped_ref;       // reference raster clipped
};
struct PlanDev {
    const Camera* cameras;
    const PlanView* views;
    float center[3];
    uint32_t nviews, ss, size;
    uint32_t force_two;
    uint32_t state_is_ref; // state masks equal the reference masks
    // Verdict-only bounds on the squared distance (see audit_unit): samples
    // nearer than d2_floor need no exact value, a view whose maximum exceeds
    // d2_ceiling fails every gate of the plan. Exact: 0 and UINT32_MAX.
    uint32_t d2_floor, d2_ceiling;
};

// ---- launchers (kernels.cu) ----
void launch_weld(const DevMesh& m, uint32_t* table, uint32_t capacity, bool with_uv, uint32_t* out,
                 cudaStream_t s);
void launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, cudaStream_t s);
size_t scan_scratch_words(uint32_t n);
void launch_topology(const DevMesh& m, uint32_t* geometry, uint32_t* face_offsets, uint32_t* faces,
                     uint32_t* cursor, uint32_t* entry_offsets, uint32_t* entries, uint32_t* nbr_offsets,
                     uint32_t* neighbors, uint8_t* nbr_count, uint8_t* boundary, uint8_t* invalid,
                     uint32_t* slot_offsets, uint32_t* slots, uint32_t* scan_scratch, uint32_t* host_counts,
                     cudaStream_t s);
void launch_enumerate(const DevMesh& m, const DevTopology& t, uint32_t* edge_base, uint8_t* valid,
                      Edit* slots, uint32_t* offsets, Edit* out, uint32_t* scan_scratch, uint32_t total_nbrs,
                      bool preserve_uv, cudaStream_t s);
void launch_flat_faces(const DevMesh& m, uint32_t* flat_count, cudaStream_t s);
void launch_position_table(const DevMesh& m, const DevTopology& t, uint32_t* table, uint32_t capacity,
                           cudaStream_t s);
void launch_prepare(const DevMesh& m, const DevTopology& t, const DevMesh& original, const DevTopology& ot,
                    const void* collapses, uint32_t n, const uint32_t* table, uint32_t capacity,
                    const uint32_t* flat_total, bool preserve_uv, CandidateRecord* out, cudaStream_t s,
                    const UvSource* uv = nullptr);
void launch_raster(const DevMesh& m, const Camera* cam_host, const float* center, uint32_t ss, uint32_t size,
                   bool force_two, bool cpu_semantics, uint32_t* bits, uint8_t* counts, uint32_t* state,
                   cudaStream_t s);
// Popcounts {a^b, a|b, a, b} over `words` u32 words; samples != 0 counts
// only the first `samples` bits (bits past the last sample are ignored).
void launch_popcounts(const uint32_t* a, const uint32_t* b, uint32_t words, unsigned long long* out,
                      cudaStream_t s, uint64_t samples = 0);
void launch_distance(const uint32_t* from, const uint32_t* to, uint32_t width, uint32_t height, uint32_t* g,
                     uint32_t* d2, int32_t* stack_v, long long* stack_num, long long* stack_den, uint32_t* out_max,
                     cudaStream_t s);
void launch_counts_to_bits(const uint8_t* counts, uint32_t size, uint32_t* bits, cudaStream_t s);
void launch_tile_maxima(const uint32_t* ref_bits, const uint32_t* state_bits, const uint32_t* ref_field,
                        const uint32_t* state_field, uint32_t size, int32_t* t1, int32_t* t2, cudaStream_t s);
void launch_field(const uint32_t* bits, uint32_t width, uint32_t height, uint32_t* g, uint32_t* d2, int32_t* stack_v,
                  long long* stack_num, long long* stack_den, cudaStream_t s);
// State data of `nviews` consecutive views of a size x size plan in one pass:
// per-sample face counts (stride cstride), raster state {-, -, clipped faces,
// count overflow} per view, coverage words (stride wstride; skipped when
// state_bits is null), popcounts {changed, total, ref, state} against
// ref_bits and, when state_field is given, the exact state field and the
// 32x32 tile maxima. g/sv/sn/sd hold nviews x size^2 entries.
void launch_refresh_views(const DevMesh& m, const Camera* cams_dev, uint32_t nviews, const float* center, uint32_t ss,
                          uint32_t size, bool force_two, uint8_t* counts, size_t cstride, uint32_t* state,
                          uint32_t* state_bits, const uint32_t* ref_bits, uint32_t wstride,
                          unsigned long long* pop, const uint32_t* ref_field, uint32_t* state_field, uint32_t* g,
                          int32_t* sv, long long* sn, long long* sd, int32_t* t1, int32_t* t2, bool saturate,
                          cudaStream_t s, uint32_t* wide = nullptr,
                          bool recount = true);
// A combined trial as changes of the state: which state faces the batch
// changes (a corner remapped by `remap`, or in a class that `owner` moves to
// a placement), whether each survives (`keep`) and where (`offsets` into the
// trial mesh `trial`).
struct TrialDelta {
    const uint32_t* geometry;
    const uint32_t* remap;
    const uint32_t* owner;
    const uint32_t* keep;
    const uint32_t* offsets;
    DevMesh trial;
};
// The trial's face counts of all views from the state's (already copied into
// `counts`, clip counters into `state`): each changed state face's samples
// -1, its surviving trial face's +1 (overflow past 255 sets state[4v+3]).
void launch_count_delta_views(const DevMesh& m, const TrialDelta& d, const Camera* cams_dev, uint32_t nviews,
                              const float* center, uint32_t ss, uint32_t size, bool force_two, uint8_t* counts,
                              size_t cstride, uint32_t* state, cudaStream_t s);
// Exact squared distance fields of nviews masks at once (launch_field's row
// pass and column envelope; scratch g, sv, sn, sd of size^2 * nviews).
void launch_fields_views(const uint32_t* bits, uint32_t wstride, uint32_t nviews, uint32_t size, uint32_t* g,
                         uint32_t* field, int32_t* sv, long long* sn, long long* sd, cudaStream_t s);
// Tile maxima and popcounts of already computed state views against another
// reference (the last stages of launch_refresh_views).
void launch_compare_views(uint32_t nviews, uint32_t size, const uint32_t* state_bits, const uint32_t* ref_bits,
                          uint32_t wstride, const uint32_t* ref_field, const uint32_t* state_field, int32_t* t1,
                          int32_t* t2, unsigned long long* pop, cudaStream_t s);
// Per view, the max of t1 and of t2 over its tiles: out[2v], out[2v+1].
void launch_view_maxima(const int32_t* t1, const int32_t* t2, uint32_t tiles, uint32_t nviews, int32_t* out,
                        cudaStream_t s);
// Disjoint-footprint batch selection (select_batch, action_gpu.cu:865-899).
// ctl = {ranked position, faces that may still be removed}; out = {selected,
// first selected position, next position}. used_global: (nv+31)/32 words,
// used when the claimed-id bitmap does not fit in shared memory.
size_t select_batch_smem(uint32_t nv);
cudaError_t launch_select_batch(const DevTopology& t, const Edit* edits, const uint32_t* order, uint32_t ranked,
                                const uint32_t* ctl, uint32_t maximum, uint32_t nv, uint32_t* used_global,
                                uint32_t* selected, uint32_t* out, cudaStream_t s);
// Combined trial of `count` selected edits with midpoint placements, then
// validate_placement over it; info[0] = 1 when the placement is invalid.
// remap/owner: nv words; table: table_cap (power of two >= 2 nv) words.
void launch_batch_trial(const DevMesh& m, const DevTopology& t, const Edit* edits, const uint32_t* selected,
                        uint32_t count, uint32_t* remap, uint32_t* owner, float* placements, uint32_t* keep,
                        uint32_t* offsets, uint32_t* out_idx, uint16_t* out_mat, float* out_pos, uint32_t* table,
                        uint32_t table_cap, uint32_t* info, uint32_t* scan_scratch, cudaStream_t s,
                        const UvSource* uv = nullptr, float* out_uv = nullptr);
// Ranking scores of the legal edits (rank_actions, action_gpu.cu:809-844),
// keys for a stable descending sort. ranking: 1 Constant, 3 ShortestEdge,
// 4 CurrentPlane (neural.hpp:9).
void launch_rank(const DevMesh& m, const DevTopology& t, const Edit* edits, const uint32_t* count, uint32_t capacity,
                 double diameter, int ranking, float* scores, uint32_t* order, cudaStream_t s);
void launch_gather_window(const Edit* edits, const uint32_t* order, uint32_t first, uint32_t n, void* collapses,
                          cudaStream_t s);
cudaError_t sort_scores_desc(const float* keys_in, float* keys_out, const uint32_t* vals_in, uint32_t* vals_out,
                             uint32_t n, void* temp, size_t& temp_bytes, cudaStream_t s);
// queue: 3 words (work cursors); spill: 1 + n * nviews words for the units
// that overflow the warp tier's limits and go to the large tier (null: no
// large tier, such units fall back to the full-raster path); spill_huge: the
// same for units that overflow the large tier, audited by the huge tier with
// huge_scratch (audit_huge_scratch_bytes(huge_blocks)) in global memory.
// One plan's units (candidates x views), or (entries != null) the
// concatenated units of several sessions' plans audited in one launch.
struct AuditEntry {
    PlanDev plan;
    const CandidateRecord* recs;
    ViewRecord* out;
    uint64_t first_unit;
};
struct AuditJob {
    PlanDev plan;
    const CandidateRecord* recs;
    ViewRecord* out;
    const AuditEntry* entries; // device table, sorted by first_unit, or null
    uint32_t nentries;
    uint64_t total;            // units
    uint32_t heavy;            // set by launch_audit
    uint32_t* far;             // set by launch_audit: units beyond the huge tier's regions (1 + units), or null
};
// variant: the warp tier's limits (kAuditTierSmall: regions up to 128 x 64
// samples, 3 blocks per SM; kAuditTierMedium: 256 x 128, 1 block per SM).
constexpr int kAuditTierSmall = 0, kAuditTierMedium = 1;
// variant | kAuditSpillHeavy: warp-tier units with many changed samples go to
// the huge tier when it runs at least one block per SM.
constexpr int kAuditSpillHeavy = 2;
// The giant tier (regions up to 4160 x 4160 samples) for what overflows the
// huge tier: its spill list (1 + units words), scratch
// (audit_giant_scratch_bytes(blocks)) and blocks.
struct GiantTier {
    uint32_t* spill;
    unsigned char* scratch;
    uint32_t blocks;
    // Units whose region is beyond the huge tier's, listed by the warp tier
    // (1 + units words, or null): the giant tier takes them while the huge
    // tier runs, on `side` (forked from and joined to the launch stream by
    // `fork` / `join`; null: after the warp tier on the same stream).
    uint32_t* far = nullptr;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
// queue: 5 words (work cursors). marks (profiling, may be null): 4 events
// recorded before the warp tier, after it, after the large / huge tier and
// after the giant tier.
void launch_audit(const AuditJob& job, unsigned long long* stats, uint32_t* queue, uint32_t* spill,
                  uint32_t* spill_huge, unsigned char* huge_scratch, uint32_t huge_blocks, cudaStream_t s,
                  int variant = kAuditTierSmall, const GiantTier* giant = nullptr, cudaEvent_t* marks = nullptr);
size_t audit_huge_scratch_bytes(uint32_t blocks);
size_t audit_giant_scratch_bytes(uint32_t blocks);
struct GateDev {
    GateSettings settings;
    uint32_t plan;
};
void launch_verdicts(const ViewRecord* const* plan_records, const uint32_t* plan_views,
                     const uint32_t* plan_ss, const GateDev* gates, const CandidateRecord* records,
                     uint32_t n, void* verdicts, void* measurements, uint32_t* exact_count, cudaStream_t s);
size_t audit_smem_bytes();

// Full trial mesh of one collapse (exact path): indices compacted in face order,
// positions with every slot of class `to` at the placement.
struct TrialInfo {
    Edit edit;
    float placement[3];
    uint32_t ok;
};
// out_uv (with uv): the trial's uv per vertex slot, transported for moved slots.
void launch_trial(const DevMesh& m, const DevTopology& t, const void* collapse, TrialInfo* info, uint32_t* keep,
                  uint32_t* offsets, uint32_t* out_idx, uint16_t* out_mat, float* out_pos, uint32_t* scan_scratch,
                  cudaStream_t s, const UvSource* uv = nullptr, float* out_uv = nullptr);

} // namespace b200
