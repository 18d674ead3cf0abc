/* blitz_audit.h — C ABI of the B200 candidate-audit engine.
 *
 * Drop-in boundary for BlitzRemesher's audit call. The ABI-5 descriptors
 * (blitz_status, blitz_stream, blitz_mesh) and the neural v2 options and
 * diagnostics (blitz_neural_options_v2, blitz_neural_info) keep the exact
 * layouts of BlitzRemesher's include/blitz/blitz.h, so a client that already
 * fills them passes the same structs here. The audit entry points are new: the
 * reference has no C function for its audit (it is internal C++,
 * src/neural/evaluate.cu AuditCuda::evaluate/certify and
 * src/neural/action_gpu.cu GpuActionState::execute); each declaration below
 * names the internal call it replaces.
 *
 * Conventions (as blitz.h): every call returns a blitz_status; C++ exceptions
 * never cross; an optional caller buffer receives a NUL-terminated message;
 * struct_size / abi_version are validated; source streams are borrowed and
 * never freed or mutated; a missing GPU yields BLITZ_UNAVAILABLE. A session is
 * used by one thread at a time; it preserves the caller's current CUDA device.
 */
#ifndef BLITZ_AUDIT_H
#define BLITZ_AUDIT_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#ifndef BLITZ_REMESHER_H
#define BLITZ_ABI_VERSION 5u
/* blitz.h:9-17 */
typedef enum blitz_status {
    BLITZ_OK = 0,
    BLITZ_INVALID_ARGUMENT = 1,
    BLITZ_OUT_OF_MEMORY = 2,
    BLITZ_INTERNAL_ERROR = 3,
    BLITZ_CANCELLED = 4,
    BLITZ_BUDGET_LIMITED = 5,
    BLITZ_UNAVAILABLE = 6
} blitz_status;
/* blitz.h:18-21 */
typedef struct blitz_stream {
    const void* data;
    size_t count, stride;
} blitz_stream;
/* blitz.h:28-37 */
typedef struct blitz_mesh {
    uint32_t struct_size, abi_version;
    blitz_stream positions, normals, uv, colors, tangents;
    const uint32_t* indices;
    size_t index_count;
    const uint16_t* materials;
    size_t material_count;
    const uint8_t* double_sided;
    size_t double_sided_count;
} blitz_mesh;
/* blitz.h:127-141 */
typedef struct blitz_neural_options_v2 {
    uint32_t struct_size, version;
    int32_t device;
    uint32_t memory_mib, action_trials, ranking_seed;
    uint16_t exact_position_bps;
    uint8_t action_batch, origin;
    uint8_t ranking;
    uint8_t confirmation;
    uint8_t raster_backend; /* 0 = CUDA (the only backend here) */
    uint8_t vertex_storage; /* FP32 master streams only */
    uint8_t preserve_uv;
    uint8_t overdraw_tiebreak, cache_rasters, mask_only_coverage, direct_targets;
    uint8_t view_batch, candidate_batch;
    uint8_t reserved[3];
} blitz_neural_options_v2;
/* blitz.h:150-155 */
typedef struct blitz_neural_info {
    uint32_t struct_size;
    uint64_t encode_ns, inference_ns, decode_ns, gpu_audit_ns, reference_audit_ns;
    uint64_t decoded, legal_collapses, rejected_collapses, reference_rejections;
    uint32_t fallback_levels;
} blitz_neural_info;
uint32_t blitz_abi_version(void);
/* c_api.cpp:228-245 — defaults of blitz::NeuralOptions. */
blitz_status blitz_neural_options_v2_init(blitz_neural_options_v2*, size_t);

/* ---- The rest of blitz.h (blitz.h:22-27, 38-88, 95-171), same layouts ----
 * Generation here is the neural path only: blitz_generate_neural routes every
 * audit of the LOD chain to this engine (blitz_audit_chain: the schedule of
 * chain.cpp:101-118, the four gates of generate.cpp:365-388, the executor's
 * collapses with midpoint placement, the confirmation of generate.cpp:456-562
 * at the audit views). blitz_generate (the classical CPU reducer) and the
 * normals/attributes profiles return BLITZ_UNAVAILABLE. */
typedef struct blitz_color_rgba8 {
    uint8_t r, g, b, a;
} blitz_color_rgba8;
typedef struct blitz_curve_point {
    float x, y;
} blitz_curve_point;
typedef struct blitz_settings {
    uint32_t struct_size, abi_version;
    uint8_t levels, profile;
    uint16_t triangle_overhead_bps;
    uint32_t max_added_vertex_bytes_bps;
    uint8_t objective, beam_width, search_supersample, audit_supersample;
    uint8_t max_supersample, prune, force_scalar, coupled_wedges;
    uint16_t candidate_budget, search_ortho, search_perspective, audit_ortho, audit_perspective;
    uint32_t search_seed, audit_seed;
    double pixels_per_meter, meters_per_unit, base_pixels, last_pixels, max_lod0_delta_px;
    double normal_weight, color_weight, material_weight;
    double max_changed_area;
    const blitz_curve_point* transition;
    size_t transition_count;
    const blitz_curve_point* normal_importance;
    size_t normal_importance_count;
    const blitz_curve_point* attribute_importance;
    size_t attribute_importance_count;
    int (*cancelled)(void*);
    void* user_data;
} blitz_settings;
typedef struct blitz_lod_info {
    uint32_t struct_size;
    blitz_mesh mesh;
    double screen_pixels, transition_limit, source_limit, transition_error, source_error;
    uint32_t transition_worst_view, source_worst_view;
    uint8_t shared_vertices, passed;
    uint32_t reference_triangles;
    double transition_changed_area, source_changed_area;
    uint32_t transition_changed_area_worst_view, source_changed_area_worst_view;
} blitz_lod_info;
typedef struct blitz_result blitz_result;
typedef struct blitz_storage_info {
    uint32_t struct_size;
    uint64_t source_vertex_bytes, added_vertex_bytes, index_bytes, total_bytes;
    uint64_t added_vertex_budget_bytes;
    uint32_t max_added_vertex_bytes_bps;
} blitz_storage_info;
blitz_status blitz_result_storage(const blitz_result*, blitz_storage_info*);
typedef struct blitz_runtime_lod_storage_info {
    uint32_t struct_size;
    uint8_t scheduled_index;
    uint64_t added_vertex_bytes, index_bytes, cumulative_added_vertex_bytes;
} blitz_runtime_lod_storage_info;
blitz_status blitz_result_runtime_lod_storage(const blitz_result*, size_t, blitz_runtime_lod_storage_info*);
/* c_api.cpp:82-122 — defaults of blitz::Settings (remesher.hpp:31-56). */
blitz_status blitz_settings_init(blitz_settings*, size_t);
/* The classical reducer is not part of this engine: BLITZ_UNAVAILABLE. */
blitz_status blitz_generate(const blitz_mesh*, const blitz_settings*, blitz_result**, char* error,
                            size_t error_capacity);
size_t blitz_result_lod_count(const blitz_result*);
size_t blitz_result_runtime_lod_count(const blitz_result*);
size_t blitz_result_runtime_lod_index(const blitz_result*, size_t);
blitz_status blitz_result_lod(const blitz_result*, size_t, blitz_lod_info*);
void blitz_result_destroy(blitz_result*);
typedef struct blitz_neural_model blitz_neural_model;
typedef struct blitz_neural_options {
    uint32_t struct_size, version;
    int32_t device;
    uint32_t memory_mib;
    uint8_t overdraw_tiebreak;
    uint8_t reserved[3];
} blitz_neural_options;
typedef enum blitz_neural_origin {
    BLITZ_NEURAL_SOURCE = 0,
    BLITZ_NEURAL_PREVIOUS = 1,
    BLITZ_NEURAL_BOTH = 2
} blitz_neural_origin;
typedef enum blitz_neural_action_stop {
    BLITZ_NEURAL_TARGET_REACHED = 0,
    BLITZ_NEURAL_TRIAL_BUDGET = 1,
    BLITZ_NEURAL_NO_LEGAL_ACTIONS = 2,
    BLITZ_NEURAL_NO_ACCEPTED_ACTION = 3,
    BLITZ_NEURAL_ACTION_CANCELLED = 4,
    BLITZ_NEURAL_ACTION_RESOURCE = 5,
    BLITZ_NEURAL_INFEASIBLE_SEED = 6
} blitz_neural_action_stop;
typedef struct blitz_neural_action_proposal {
    uint32_t struct_size, version;
    uint32_t start_triangles, target_triangles, final_triangles, trial_budget, trials, accepted_batches;
    double screen_pixels;
    uint8_t origin, output, stop_reason;
    uint8_t reserved[5];
} blitz_neural_action_proposal;
/* c_api.cpp:208-213 */
blitz_status blitz_neural_options_init(blitz_neural_options*, size_t);
/* BLZNET01/02/03 policy files (model_io.cpp:59-107: header, provenance,
 * FP32 weights, SHA-256 checksum of the payload). The policy's weights are
 * loaded and checked; rankings here are ShortestEdge, CurrentPlane and
 * Constant (options v2 `ranking` 3, 4, 1); Learned and Shuffled, which score
 * edits with the policy network, return BLITZ_UNAVAILABLE at generation. */
blitz_status blitz_neural_model_load(const char* path, const blitz_neural_options*, blitz_neural_model**,
                                     char* error, size_t error_capacity);
blitz_status blitz_neural_model_load_v2(const char* path, const blitz_neural_options_v2*,
                                        blitz_neural_model**, char* error, size_t error_capacity);
void blitz_neural_model_destroy(blitz_neural_model*);
/* Borrowed lowercase hex SHA-256 of the model file, valid until destruction. */
const char* blitz_neural_model_sha256(const blitz_neural_model*);
blitz_status blitz_generate_neural(const blitz_mesh*, const blitz_settings*, const blitz_neural_model*,
                                   blitz_result**, char* error, size_t error_capacity);
blitz_status blitz_result_neural_info(const blitz_result*, blitz_neural_info*);
size_t blitz_result_neural_action_proposal_count(const blitz_result*);
blitz_status blitz_result_neural_action_proposal(const blitz_result*, size_t, blitz_neural_action_proposal*);
#endif

/* ---- Mesh files ----------------------------------------------------------
 * Import (the rules of load_mesh, src/io.cpp:118-229): OBJ (corners
 * deduplicated by position/normal/uv index, polygons fanned, material ids
 * 1 + place in the material library, non-opaque materials refused), PLY
 * (ascii, binary either endianness, triangles only) and STL (binary or ascii,
 * corners welded on exact position bits); 1 GiB cap; the reference's mesh
 * validation (mesh.cpp:27-41). glTF import returns BLITZ_UNAVAILABLE. The
 * descriptor borrows the file object's streams until it is destroyed. */
typedef struct blitz_mesh_file blitz_mesh_file;
blitz_status blitz_mesh_file_load(const char* path, blitz_mesh_file** out, blitz_mesh* mesh, char* error,
                                  size_t error_capacity);
void blitz_mesh_file_destroy(blitz_mesh_file*);
/* Binary little-endian PLY of a mesh (save_ply, io.cpp:236-249). */
blitz_status blitz_mesh_save_ply(const blitz_mesh* mesh, const char* path, char* error, size_t error_capacity);
/* A generated chain as one glTF 2.0 scene (chain.gltf, chain.bin: one mesh
 * per runtime level, one primitive per material, one node per scheduled
 * level) and the lods.json manifest (save_chain, io.cpp:298-359). */
blitz_status blitz_result_save_chain(const blitz_result* result, const char* directory, char* error,
                                     size_t error_capacity);

/* POD mirror of blitz::EvalSettings for the coverage profile
 * (include/blitz/evaluate.hpp:24-33; ViewSet evaluate.hpp:8). */
typedef struct blitz_eval_settings {
    uint32_t struct_size;
    uint8_t profile;          /* 0 = coverage; normals/attributes: BLITZ_UNAVAILABLE */
    uint8_t supersample;      /* 1..32 */
    uint8_t max_supersample;  /* supersample..32 */
    uint8_t force_two_sided;
    uint8_t conservative_screen;
    uint8_t reserved[1];
    uint16_t views_orthographic, views_perspective;
    uint32_t views_seed;
    double screen_size, limit, max_changed_area;
} blitz_eval_settings;

/* POD mirror of blitz::Measurement (include/blitz/evaluate.hpp:34-39). */
typedef struct blitz_measurement {
    double error, coverage, coverage_upper, changed_area, normal_degrees;
    uint32_t worst_view, changed_area_worst_view, views_evaluated;
    uint8_t supersample, complete, passed, resource_limited, cancelled;
    uint8_t reserved[3];
} blitz_measurement;

/* One proposed directed edge contraction relative to the session's current
 * state: geometric class `from` contracts into class `to` (class = smallest
 * vertex slot at the same position), written at `position` or at the edge
 * midpoint. Mirrors neural::Action + Placement (action.hpp:11-14,
 * placement.hpp:6-20). */
typedef struct blitz_collapse {
    uint32_t from, to;
    uint32_t placement; /* 0 = midpoint of the two class roots, 1 = explicit */
    float position[3];
} blitz_collapse;

/* Four-gate result for one collapse (generate.cpp:365-388). */
typedef struct blitz_candidate_verdict {
    uint8_t accepted;    /* all four gates passed */
    uint8_t failed_gate; /* 0 accepted; 1..4 source-search, previous-search,
                            source-audit, previous-audit; 5 illegal; 6 invalid placement */
    uint8_t exact_path;  /* 1 when a view needed the full-raster path */
    uint8_t reserved;
    uint32_t removed;    /* faces the collapse removes */
} blitz_candidate_verdict;

typedef struct blitz_audit_session blitz_audit_session;

blitz_status blitz_eval_settings_init(blitz_eval_settings*, size_t);

/* Uploads the source (LOD0) and builds the local-collapse topology of the
 * session's current state (initially the source). Replaces the construction
 * of neural::AuditCuda (evaluate.cu:2179-2212) and GpuActionState
 * (action_gpu.cu:1459-1569). `options` may be NULL (defaults). */
blitz_status blitz_audit_session_create(const blitz_mesh* source, const blitz_neural_options_v2* options,
                                        blitz_audit_session** out, char* error, size_t error_capacity);
void blitz_audit_session_destroy(blitz_audit_session*);

/* Binds the previous emitted LOD as the adjacent reference
 * (AuditCuda::bind_reference, generate.cpp:313). NULL binds the source. */
blitz_status blitz_audit_bind_reference(blitz_audit_session*, const blitz_mesh* previous, char* error,
                                        size_t error_capacity);

/* Full audit of an arbitrary candidate against an arbitrary reference with the
 * session's bounds: the twin of blitz::evaluate (evaluate.cpp:353) and
 * AuditCuda::evaluate (evaluate.cu:2261-2341), coverage profile. */
blitz_status blitz_audit_evaluate(blitz_audit_session*, const blitz_mesh* reference,
                                  const blitz_mesh* candidate, const blitz_eval_settings* settings,
                                  blitz_measurement* out, char* error, size_t error_capacity);

/* One view of a camera set: blitz::Camera (evaluate.hpp:46). */
typedef struct blitz_view_camera {
    float right[3], up[3], forward[3];
    double distance, focal, scale;
    uint32_t perspective, pad;
} blitz_view_camera;
/* Host only, no session or GPU: the bounds every audit projects with
 * (blitz::bounds, mesh.cpp:12-20: bbox centre, largest distance to it) and
 * the camera set of (ortho, persp, seed) at `screen` (blitz::cameras,
 * evaluate.cpp:108-124, with this platform's libm as the reference uses its
 * own). `capacity` >= ortho + persp cameras. */
blitz_status blitz_mesh_bounds(const blitz_mesh* mesh, float center[3], double* radius, char* error,
                               size_t error_capacity);
blitz_status blitz_view_cameras(const float center[3], double radius, double screen, uint16_t ortho, uint16_t persp,
                                uint32_t seed, blitz_view_camera* out, size_t capacity, char* error,
                                size_t error_capacity);

/* Packed coverage mask of `mesh` in camera `view` of the camera set
 * (ortho, persp, seed) at `screen` x `supersample`, with the session's bounds:
 * the twin of blitz::detail::rasterize_coverage (evaluate.cpp:193-195).
 * `words` receives ceil(size*size/64) little-endian u64 words (bit i%64 of
 * word i/64 is sample i = y*size+x; tail bits zero); `*size` the raster side. */
blitz_status blitz_audit_raster(blitz_audit_session*, const blitz_mesh* mesh, double screen, uint8_t supersample,
                                uint16_t views_orthographic, uint16_t views_perspective, uint32_t views_seed,
                                uint32_t view, uint8_t force_two_sided, uint64_t* words, size_t word_capacity,
                                uint32_t* size, uint8_t* clipped, char* error, size_t error_capacity);

/* Symmetric coverage distance in pixels between two packed masks of
 * width x height samples (the layout of blitz_audit_raster): 0 when the masks
 * are equal, infinity when exactly one is empty, else sqrt(max squared
 * distance)/supersample. The twin of blitz::detail::coverage_distance
 * (coverage.hpp:13, evaluate.cpp:196-216). `masks_on_device` selects device
 * or host pointers for a and b. */
blitz_status blitz_audit_coverage_distance(blitz_audit_session*, const uint64_t* a, const uint64_t* b,
                                           uint32_t width, uint32_t height, uint8_t supersample,
                                           int masks_on_device, double* out, char* error, size_t error_capacity);

/* The same coverage distance computed without allocating anything. This entry
 * point has no counterpart in the reference. It exists for callers that may
 * not call cudaMalloc: plugins whose host process gives all device memory to
 * another allocator (a framework's caching allocator, an engine that hands
 * out fixed budgets), or loops that must avoid the synchronisation that
 * cudaMalloc/cudaFree can imply. Its scratch is one static device array of
 * about 7 MiB, held by every GPU that loads the library until the process
 * exits; masks are limited to 512 x 512 = 262144 samples (larger masks return
 * BLITZ_INVALID_ARGUMENT). Inputs are device masks (layout of
 * blitz_audit_raster, no padding needed; bits at or past width x height are
 * ignored) and the result is written to the device double `out_device`, all
 * enqueued on `stream` (a cudaStream_t, NULL = default stream) on the current
 * device; the call does not synchronise. Each call outside stream capture
 * looks up the array's device address on the current device (so a context
 * created anew after cudaDeviceReset is followed); a call during capture
 * reuses the address of the last call outside it, so make the first call on a
 * device before any stream capture. A CUDA error already pending on the
 * calling thread is left in place and reported as BLITZ_INTERNAL_ERROR with
 * nothing enqueued. All calls share the one array, so calls that overlap on
 * the GPU race: serialise them. */
blitz_status blitz_audit_coverage_distance_static(const uint64_t* a_device, const uint64_t* b_device,
                                                  uint32_t width, uint32_t height, uint8_t supersample,
                                                  double* out_device, void* stream, char* error,
                                                  size_t error_capacity);

/* Legal directed collapses of the current state, in the reference's
 * enumeration order (action_gpu.cu:626-643 enumerate + DeviceSelect::Flagged).
 * Writes min(count, capacity) collapses with midpoint placement; *count
 * receives the total. */
blitz_status blitz_audit_actions(blitz_audit_session*, blitz_collapse* out, size_t capacity, size_t* count,
                                 char* error, size_t error_capacity);

/* Batched four-gate audit of `n` collapses of the current state: each is
 * applied with its placement, rasterized over the gates' views and compared
 * with the source (gates 1, 3) and the bound previous LOD (gates 2, 4).
 * Replaces the gate lambda of generate.cpp:365-388 over
 * GpuActionState::trial + AuditCuda::certify. Host buffers; `measurements`
 * may be NULL, else it receives 4 per collapse (gates not reached stay
 * zero-initialised defaults). */
blitz_status blitz_audit_candidates(blitz_audit_session*, const blitz_collapse* candidates, size_t n,
                                    const blitz_eval_settings gates[4], blitz_candidate_verdict* out,
                                    blitz_measurement* measurements, char* error, size_t error_capacity);

/* Same as blitz_audit_candidates with device-resident candidate and verdict
 * arrays, enqueued on `stream` (a cudaStream_t; NULL = the session stream).
 * Synchronises before returning. */
blitz_status blitz_audit_candidates_device(blitz_audit_session*, const blitz_collapse* candidates_device,
                                           size_t n, const blitz_eval_settings gates[4],
                                           blitz_candidate_verdict* out_device,
                                           blitz_measurement* measurements_device, void* stream,
                                           char* error, size_t error_capacity);

/* Result of blitz_audit_execute (mirrors neural::ActionStats, action.hpp). */
typedef struct blitz_audit_execution {
    uint32_t struct_size;
    uint32_t commits;     /* accepted collapses */
    uint32_t trials;      /* audited trials, as counted by the reference executor */
    uint32_t final_faces;
    uint64_t audited;     /* candidates audited, speculative windows included */
    uint8_t stop_reason;  /* 0 target reached, 1 trial budget, 2 no legal actions, 3 no accepted action */
    uint8_t fallbacks;    /* surrogate walks that fell back to the full order (saturates at 255) */
    uint8_t reserved[6];
} blitz_audit_execution;

/* Greedy LOD step on the session's current state, batches of one, ShortestEdge
 * ranking, midpoint placement: the reference's GpuActionState::execute
 * (action_gpu.cu:1947-2086) / execute_actions (action.cpp:453-525) with the
 * four-gate gate of generate.cpp:365-388 against the source and the bound
 * previous LOD. Writes the accepted (from, to) pairs in order (up to
 * `commit_capacity`). The state keeps the result; blitz_audit_state reads it. */
blitz_status blitz_audit_execute(blitz_audit_session*, uint32_t target_faces, uint32_t trial_budget,
                                 const blitz_eval_settings gates[4], uint32_t* commits_from_to,
                                 size_t commit_capacity, blitz_audit_execution* out, char* error,
                                 size_t error_capacity);
/* Executor options (the reference's neural option `action_batch`,
 * blitz.h:130-133, and GpuActionState::execute's `batch`, action_gpu.cu:1947-1954). */
typedef struct blitz_execute_options {
    uint32_t struct_size;
    uint32_t batch;         /* 1..64 independent collapses audited as one combined trial */
    uint32_t keep_permille; /* 0: no surrogate; else the share of ranked edits the attached surrogate
                               keeps (250 = top 25%), with the full order as fallback */
    uint32_t ranking;       /* NeuralRanking (neural.hpp:9): 0 learned = the attached surrogate's acceptance
                               logits, 1 constant, 3 shortest edge (default), 4 current plane */
    uint32_t reserved[4];   /* zero */
} blitz_execute_options;
void blitz_execute_options_init(blitz_execute_options*);

/* blitz_audit_execute with options. batch = 1 is blitz_audit_execute; batch > 1
 * selects disjoint-footprint batches in rank order (select_batch,
 * action_gpu.cu:865-899), audits each batch's combined trial through the four
 * gates, halves a rejected batch and after a rejected singleton resumes one
 * past the batch's first edit (verdict, action_gpu.cu:904-915; execute_actions,
 * action.cpp:486-515). `trials` counts audited batch trials, `commits` the
 * collapses they committed. */
blitz_status blitz_audit_execute_ex(blitz_audit_session*, uint32_t target_faces, uint32_t trial_budget,
                                    const blitz_eval_settings gates[4], const blitz_execute_options* options,
                                    uint32_t* commits_from_to, size_t commit_capacity,
                                    blitz_audit_execution* out, char* error, size_t error_capacity);
/* ---- Learned audit surrogate ---------------------------------------------
 * A 48 -> 128 -> 128 -> 2 MLP (ReLU) with BF16 weights and FP32 accumulation,
 * run by the library's own tcgen05 kernels, that predicts per candidate
 * collapse the logit of acceptance by the exact four-gate audit and the ratio
 * error / limit of the worst gate. It has no reference counterpart: the
 * reference's learned policies (inference.cu, fused.cu) rank endpoint edits
 * with FP32 networks; this model only prunes the ranked edits of the batched
 * executor and never accepts a collapse itself. */
#define BLITZ_SURROGATE_FEATURES 48
/* FP32 parameters in this order: W1 128x64 (inputs padded 48 -> 64), b1 128,
 * W2 128x128, b2 128, W3 16x128 (outputs padded 2 -> 16), b3 16; row-major
 * [out][in]. Padding entries are zero. */
#define BLITZ_SURROGATE_PARAMS 26896
typedef struct blitz_surrogate blitz_surrogate;
/* New model on `device` with He-uniform weights drawn from `seed`, zero
 * biases, identity feature normalisation. */
blitz_status blitz_surrogate_create(int device, uint32_t seed, blitz_surrogate** out, char* error,
                                    size_t error_capacity);
void blitz_surrogate_destroy(blitz_surrogate*);
/* Parameters (BLITZ_SURROGATE_PARAMS floats) and the feature normalisation
 * x' = (x - mean) * inv_std (48 floats each; null keeps the current one).
 * Loading resets the Adam state. */
blitz_status blitz_surrogate_load(blitz_surrogate*, const float* params, size_t count, const float* mean,
                                  const float* inv_std, char* error, size_t error_capacity);
blitz_status blitz_surrogate_save(const blitz_surrogate*, float* params, size_t capacity, float* mean,
                                  float* inv_std, char* error, size_t error_capacity);
/* Forward pass over n rows of device features (n x 48 FP32) into device
 * outputs (n x 2: acceptance logit, predicted error / limit), enqueued on
 * `stream` (NULL = the model's stream); synchronises before returning. */
blitz_status blitz_surrogate_score(blitz_surrogate*, const float* features_device, size_t n, float* out_device,
                                   void* stream, char* error, size_t error_capacity);
/* Gradients of mean over the n rows of BCE(logit, accepted) + Huber(pred -
 * error ratio) (labels_device: n x 2 = {accepted 0/1, error / limit}) in the
 * parameter order above, without updating the model; *loss = the mean loss. */
blitz_status blitz_surrogate_gradients(blitz_surrogate*, const float* features_device, const float* labels_device,
                                       size_t n, float* gradients_host, size_t capacity, float* loss, char* error,
                                       size_t error_capacity);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the mean loss of the n rows. */
blitz_status blitz_surrogate_train_step(blitz_surrogate*, const float* features_device, const float* labels_device,
                                        size_t n, float learning_rate, float* loss, void* stream, char* error,
                                        size_t error_capacity);
/* Features (n x 48, device) of the session state's legal edits in the order
 * of blitz_audit_actions, with those edits as midpoint collapses on the host
 * (capacity rows each); `screen` and `screen2` are the search and audit
 * screen sizes in pixels. */
blitz_status blitz_audit_surrogate_features(blitz_audit_session*, double screen, double screen2,
                                            float* features_device, blitz_collapse* collapses, size_t capacity,
                                            size_t* count, char* error, size_t error_capacity);
/* Attaches a model (same device; NULL detaches) for blitz_execute_options.keep_permille. */
blitz_status blitz_audit_attach_surrogate(blitz_audit_session*, blitz_surrogate*, char* error, size_t error_capacity);

/* ---- Batched audit over several sessions ----------------------------------
 * Candidates of many meshes audited together: one k_prepare per session, one
 * persistent audit launch per distinct plan slot over all sessions' (candidate,
 * view) units, one k_verdicts per session. Verdicts equal those of
 * blitz_audit_candidates on each session. The reference audits one mesh at a
 * time (AuditCuda::certify_candidates, evaluate.cu:2394-2412, at most 8
 * candidates); this entry point has no reference counterpart. The sessions
 * must be on one device and must not be used by other threads meanwhile. */
typedef struct blitz_audit_batch blitz_audit_batch;
#define BLITZ_BATCH_GRAPH 1u    /* capture the launch sequence once and replay it while the candidate and
                                   verdict buffers, counts, gates, stream and session states are unchanged */
#define BLITZ_BATCH_AUTOTUNE 2u /* time the audit variants on this call and keep the fastest */
#define BLITZ_BATCH_PROFILE 4u  /* record the audit launches' device time and work counters (no graph) */
#define BLITZ_BATCH_TIMING 8u   /* record the audit launches' device time only: the kernels run without
                                   their per-unit counters (no graph) */
typedef struct blitz_audit_batch_info {
    uint32_t struct_size;
    uint32_t sessions;
    uint32_t tier;            /* bit 0: warp tier (0: 128 x 64-sample regions, 3 blocks/SM; 1: 256 x 128,
                                 1 block/SM); bit 1: units with many changed samples go to the huge tier */
    uint32_t tuned, graph_captured;
    float tune_ms[4];         /* device time of one batch with each variant when tuned (0: not tried) */
    uint64_t graph_launches;  /* replays of the captured graph */
    uint64_t exact_candidates;
    /* last BLITZ_BATCH_PROFILE call: audit launches' device time, (candidate,
     * view) units audited by any tier, region samples rasterized, changed
     * samples measured */
    float audit_ms;
    uint64_t units, region_samples, changed_samples;
    /* the same call, per tier (warp, large, huge, giant): units audited and
     * the SM cycles their warps spent; SM cycles of all units' face setup,
     * region phases and distance phase; samples whose coverage flipped */
    uint64_t tier_units[4], tier_cycles[4], phase_cycles[3], flipped_samples;
    /* region phases split: SM cycles zeroing the region words; direct-test
     * path cycles and units; row-sweep path cycles and units; the sweep's
     * cycles building sorted interval ends and visiting pieces (each the max
     * over a warp's lanes); rows swept; word-row path cycles and units, its
     * cycles computing intervals, OR-ing word masks, testing words and (the
     * max over a warp's lanes) counting old faces of losing samples; rows */
    uint64_t region_split[15];
    /* the same call: samples of the rasterized faces' bounding boxes summed
     * over units (the (face, sample) pairs a per-sample raster would test) */
    uint64_t face_samples;
    /* the same call, per tier: SM cycles of its longest unit */
    uint64_t tier_max_cycles[4];
    /* last BLITZ_BATCH_PROFILE or BLITZ_BATCH_TIMING call: device time of the
     * warp tier's launches, of the large / huge tier's (units whose regions
     * are beyond the huge tier's run in the giant tier beside it) and of the
     * giant tier's launches after it */
    float tier_ms[3];
} blitz_audit_batch_info;
blitz_status blitz_audit_batch_create(blitz_audit_session* const* sessions, size_t count, blitz_audit_batch** out,
                                      char* error, size_t error_capacity);
void blitz_audit_batch_destroy(blitz_audit_batch*);
/* candidates_device: the sessions' candidates concatenated in session order
 * (counts[i] each, relative to each session's current state); verdicts_device
 * the same layout. `stream`: a cudaStream_t or NULL (the batch's stream).
 * Synchronises before returning. */
blitz_status blitz_audit_batch_candidates(blitz_audit_batch*, const blitz_collapse* candidates_device,
                                          const size_t* counts, const blitz_eval_settings gates[4],
                                          blitz_candidate_verdict* verdicts_device, uint32_t flags, void* stream,
                                          char* error, size_t error_capacity);
/* The same batched audit from host memory: the sessions' candidates
 * concatenated in session order are copied in, the verdicts copied out
 * (through device buffers the batch owns, so a captured graph keeps
 * replaying), on the batch's stream. The host-buffer counterpart of
 * blitz_audit_candidates (the reference's audit takes host meshes:
 * AuditCuda::evaluate, src/neural/internal.hpp:131-175) for many sessions.
 * Synchronises before returning. */
blitz_status blitz_audit_batch_candidates_host(blitz_audit_batch*, const blitz_collapse* candidates,
                                               const size_t* counts, const blitz_eval_settings gates[4],
                                               blitz_candidate_verdict* verdicts, uint32_t flags, char* error,
                                               size_t error_capacity);
blitz_status blitz_audit_batch_read_info(const blitz_audit_batch*, blitz_audit_batch_info* out);

/* ---- LOD chain -------------------------------------------------------------
 * Levels 1..levels-1 from the source: per level the schedule of chain.cpp
 * (schedule 101-118, Curve::at 25-36: pixels S_i = base (last/base)^(i/(levels-1)),
 * transition d_i from the curve, LOD0 bound B_i = min(B_{i-1} S_i/S_{i-1} + d_i,
 * max_lod0_delta_px)), the four gates of eval_config (179-199: search views and
 * max_changed_area 1, audit views and max_changed_area), the previous level
 * bound as the adjacent reference, the executor (blitz_audit_execute_ex) down
 * to `min_faces`, then the confirmation of the emitted level at the audit
 * views against the source (B_i) and the previous level (d_i)
 * (generate.cpp:456-562, hooks.confirm). The session's state ends as the last
 * level. */
typedef struct blitz_chain_settings {
    uint32_t struct_size;
    uint32_t levels;               /* 2..32, LOD0 included */
    double base_pixels;            /* S_0 */
    double last_pixels;            /* S_{levels-1} */
    double max_lod0_delta_px;      /* 0: no cap */
    float transition_curve[16];    /* (x, y) pairs, x ascending */
    uint32_t transition_points;    /* 1..8 */
    uint16_t search_orthographic, search_perspective;
    uint32_t search_seed;
    uint16_t audit_orthographic, audit_perspective;
    uint32_t audit_seed;
    uint8_t search_supersample, audit_supersample, max_supersample, force_two_sided;
    double max_changed_area;       /* audit gates; search gates use 1 */
    uint32_t batch;                /* 1..64 */
    uint32_t keep_permille;        /* surrogate pruning (attached model), 0 off */
    uint32_t trial_budget;         /* per level */
    uint32_t min_faces;            /* per-level target faces (1: as far as the gates allow) */
    uint32_t ranking;              /* as blitz_execute_options.ranking */
    uint32_t reserved[3];
} blitz_chain_settings;
void blitz_chain_settings_init(blitz_chain_settings*);
typedef struct blitz_chain_level {
    uint32_t struct_size;
    uint32_t level;
    double pixels, transition, source_bound;
    uint32_t faces, commits, trials;
    uint8_t stop_reason;           /* as blitz_audit_execution */
    uint8_t confirmed;             /* both confirmation audits passed */
    uint8_t reserved[2];
    blitz_measurement source_audit, transition_audit;
    double seconds;                /* executor + confirmation */
} blitz_chain_level;
/* Called once per level with the level's compacted indices and every vertex
 * slot's position (host memory valid during the call). During the call the
 * session's state is that level: blitz_audit_state_uv returns its uv. */
typedef void (*blitz_chain_emit)(void* user, uint32_t level, const uint32_t* indices, uint32_t face_count,
                                 const float* positions, uint32_t vertex_count);
/* The chain's schedule alone (blitz::schedule, chain.cpp:101-118; no GPU):
 * per level (0 = the source) the audited screen size, the transition bound
 * and the LOD0 bound that blitz_audit_chain uses. `capacity` >= levels. */
blitz_status blitz_chain_schedule(const blitz_chain_settings* settings, double* pixels, double* transition,
                                  double* source_bound, size_t capacity, char* error, size_t error_capacity);
blitz_status blitz_audit_chain(blitz_audit_session*, const blitz_chain_settings* settings,
                               blitz_chain_level* levels, size_t capacity, blitz_chain_emit emit, void* user,
                               char* error, size_t error_capacity);

/* Current state: compacted indices (3 per face) and every vertex slot's position. */
blitz_status blitz_audit_state(blitz_audit_session*, uint32_t* indices, size_t index_capacity, float* positions,
                               size_t position_capacity, uint32_t* face_count, char* error, size_t error_capacity);
/* Current state's uv, 2 per vertex slot (the uv stream of GpuActionState's
 * mesh, transported by place_vertices, action_gpu.cu:962-1067). Invalid
 * argument when the session's mesh has no uv. */
blitz_status blitz_audit_state_uv(blitz_audit_session*, float* uv, size_t uv_capacity, char* error,
                                  size_t error_capacity);
/* Current state's per-face materials (compacted like the indices; the
 * state keeps each surviving face's material). Invalid argument when the
 * session's mesh has no materials. */
blitz_status blitz_audit_state_materials(blitz_audit_session*, uint16_t* materials, size_t capacity,
                                         uint32_t* face_count, char* error, size_t error_capacity);
/* Restores the state to the source (GpuActionState::reset, action_gpu.cu:1884-1906). */
blitz_status blitz_audit_reset(blitz_audit_session*, char* error, size_t error_capacity);

/* Device-side profile of the session's own kernels (no reference
 * counterpart; the reference exposes NVTX ranges, timeline.hpp:6-19). With
 * enable = 1 every candidate call times its kernels with CUDA events on the
 * launching stream and counts the samples the audit kernel touched (per-unit
 * clock reads and counter atomics inside the kernel); with enable = 2 it only
 * times them (the kernels run as in production, the counters stay zero);
 * 0 disables. */
typedef struct blitz_audit_profile {
    uint32_t struct_size, enabled;
    uint64_t launches;         /* kernels launched by candidate calls */
    uint64_t audit_launches;   /* incremental audit kernel launches */
    double audit_ms, prepare_ms, verdict_ms; /* summed device time */
    uint64_t units;            /* (candidate, view) pairs audited */
    uint64_t region_samples;   /* samples rasterized by the audit kernel */
    uint64_t changed_samples;  /* samples whose distance was searched */
    uint64_t record_bytes;     /* candidate records read by the audit kernel */
} blitz_audit_profile;
blitz_status blitz_audit_profile_enable(blitz_audit_session*, int enable);
blitz_status blitz_audit_profile_read(const blitz_audit_session*, blitz_audit_profile*);

/* Session diagnostics in the reference's counter block (blitz.h:150-155):
 * gpu_audit_ns, legal_collapses, rejected_collapses, decoded (audited). */
blitz_status blitz_audit_session_info(const blitz_audit_session*, blitz_neural_info*);

#ifdef __cplusplus
}
#endif
#endif
