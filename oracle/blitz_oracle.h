/* CPU oracle for the candidate-audit path — TEST INFRASTRUCTURE ONLY.
 *
 * This header declares a plain-C interface over a CPU restatement of
 * BlitzRemesher's audit path (cameras, packed coverage raster, squared EDT
 * distance, per-view finish, evaluate loop, schedule, collapse topology,
 * legality with placement, midpoint placement/validation, trial build and the
 * four-gate verdict). It exists only so tests, the smoke check and the CPU
 * baseline leg of the benchmark can check the CUDA product against it. The
 * product library never links or calls it.
 *
 * Reference citations (file:line) are relative to the BlitzRemesher project.
 */
#ifndef BLITZ_ORACLE_H
#define BLITZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct bo_mesh {
    const float* positions;      /* xyz per vertex */
    uint32_t vertex_count;
    const uint32_t* indices;     /* 3 per face */
    uint32_t face_count;
    const uint16_t* materials;   /* per face or NULL */
    const uint8_t* double_sided; /* per material or NULL */
    uint32_t double_sided_count;
    const float* uv;             /* uv per vertex or NULL */
} bo_mesh;

typedef struct bo_bounds {
    float center[3];
    double radius;
} bo_bounds;

/* Mirrors blitz::Camera (include/blitz/evaluate.hpp:46). */
typedef struct bo_camera {
    float right[3], up[3], forward[3];
    double distance, focal, scale;
    uint8_t perspective;
    uint8_t pad[7];
} bo_camera;

/* POD mirror of blitz::EvalSettings for the coverage profile (evaluate.hpp:24-33). */
typedef struct bo_eval_settings {
    double screen_size, limit, max_changed_area;
    uint16_t views_orthographic, views_perspective;
    uint32_t views_seed;
    uint8_t supersample, max_supersample, force_two_sided, conservative_screen;
    uint8_t profile; /* 0 = coverage; others unsupported here */
    uint8_t pad[3];
} bo_eval_settings;

/* POD mirror of blitz::Measurement (evaluate.hpp:34-39). */
typedef struct bo_measurement {
    double error, coverage, coverage_upper, changed_area, normal_degrees;
    uint32_t worst_view, changed_area_worst_view, views_evaluated;
    uint8_t supersample, complete, passed, resource_limited, cancelled;
    uint8_t pad[3];
} bo_measurement;

/* Raw per-view record: what finish_view consumes for one (view, ss). */
typedef struct bo_view_record {
    double max_d2;          /* max squared EDT value over XOR samples (as the CPU float field) */
    uint64_t changed, total; /* popcount(a^c), popcount(a|c) */
    uint8_t ca, cb, same, clipped_ref, clipped_cand;
    uint8_t pad[3];
} bo_view_record;

/* One directed collapse edit (action_gpu.cu:129-132). */
typedef struct bo_edit {
    uint32_t from, to, source[2], target[2];
    uint8_t wedges, removed, valid, pad;
} bo_edit;

typedef struct bo_verdict {
    uint8_t accepted;     /* all four gates passed */
    uint8_t failed_gate;  /* 0 accepted, 1..4 failing gate, 6 invalid placement */
    uint8_t placement_valid;
    uint8_t pad[5];
    bo_measurement gates[4];
} bo_verdict;

/* status: 0 ok, 1 invalid argument, 2 length/resource error */
/* Closest point of triangle (a, b, c) to p as barycentric weights
 * (action_gpu.cu:919-952), the uv transport's projection. */
int bo_barycentric(const float p[3], const float a[3], const float b[3], const float c[3], float w[3]);
int bo_bounds_of(const bo_mesh* m, bo_bounds* out);
int bo_cameras(const bo_bounds* b, double screen, uint16_t ortho, uint16_t persp, uint32_t seed,
               bo_camera* out);
uint32_t bo_raster_size(double screen, uint8_t ss);
int bo_rasterize_coverage(const bo_mesh* m, const bo_bounds* b, const bo_camera* c, double screen,
                          uint8_t ss, int force_two, uint64_t* words, uint8_t* clipped);
int bo_coverage_distance(const uint64_t* a, const uint64_t* b, uint32_t width, uint32_t height,
                         uint8_t ss, double* out);
int bo_distance_field(const uint64_t* words, uint32_t width, uint32_t height, float* out);
int bo_view_record_of(const bo_mesh* reference, const bo_mesh* candidate, const bo_bounds* b,
                      const bo_camera* c, double screen, uint8_t ss, int force_two,
                      bo_view_record* out);
void bo_finish_view(const bo_view_record* r, const bo_eval_settings* s, uint8_t ss,
                    bo_measurement* out);
int bo_evaluate(const bo_mesh* reference, const bo_mesh* candidate, const bo_bounds* b,
                const bo_eval_settings* s, bo_measurement* out);
int bo_identical(const bo_mesh* a, const bo_mesh* b);
uint8_t bo_bounded_refinement(double screen, uint8_t supersample, uint8_t max_supersample);
int bo_schedule(double first_pixels, double last_pixels, uint32_t levels, const float* curve_xy,
                uint32_t curve_points, double max_lod0_delta_px, double* pixels,
                double* transition, double* source);

/* Collapse topology on geometric classes and legal directed actions with
 * placement (action_gpu.cu:487-643). Returns the number of legal edits written
 * (up to capacity), or -1 on error. */
int64_t bo_actions(const bo_mesh* m, int placement, int preserve_uv, bo_edit* out,
                   uint64_t capacity);
/* Topology flags per vertex slot (geometric class roots carry the flags). */
int bo_topology_flags(const bo_mesh* m, uint32_t* geometry, uint8_t* boundary, uint8_t* invalid);
/* Trial of one edit with midpoint placement. Writes the trial indices (compacted,
 * face order preserved) and positions (vertex_count*3). Returns trial face count
 * or -1; *valid receives the placement validity (place_vertices + validate_placement). */
int64_t bo_trial_midpoint(const bo_mesh* m, const bo_edit* e, int preserve_uv, uint32_t* indices,
                          float* positions, float* uv, uint8_t* valid);
/* Four-gate audit of one midpoint collapse. gates[i] settings; refs[i] selects
 * the reference mesh (0 source, 1 previous). */
int bo_audit_candidate(const bo_mesh* parent, const bo_edit* e, const bo_mesh* source,
                       const bo_mesh* previous, const bo_bounds* b, const bo_eval_settings gates[4],
                       int preserve_uv, bo_verdict* out);

/* Greedy executor, batches of one, ShortestEdge ranking, midpoint placement
 * (action.cpp:453-525). previous may be NULL (= source). Returns 0 on success;
 * *stop: 0 target reached, 1 trial budget, 2 no legal actions, 3 no accepted. */
int bo_execute(const bo_mesh* source, const bo_mesh* previous, uint32_t target, uint32_t budget,
               const bo_eval_settings gates[4], int preserve_uv, uint32_t* commits_from_to, uint32_t capacity,
               uint32_t* commits, uint32_t* trials, uint32_t* out_indices, uint32_t* out_faces,
               float* out_positions, uint8_t* stop);
/* The same executor with batches of 1..64 independent collapses, each batch
 * audited as one combined trial and halved on rejection (action.cpp:486-515). */
int bo_execute_batched(const bo_mesh* source, const bo_mesh* previous, uint32_t target, uint32_t budget,
                       const bo_eval_settings gates[4], int preserve_uv, uint32_t batch,
                       uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits, uint32_t* trials,
                       uint32_t* out_indices, uint32_t* out_faces, float* out_positions, uint8_t* stop);
/* The batched walk from `start` (a later state of `source`, same vertex
 * slots; NULL = the source) against the source and `previous`; out_uv
 * receives the final state's uv when the meshes have uv. */
/* ranking: 1 Constant, 3 ShortestEdge, 4 CurrentPlane (neural.hpp:9). */
int bo_execute_from(const bo_mesh* source, const bo_mesh* previous, const bo_mesh* start, uint32_t target,
                    uint32_t budget, const bo_eval_settings gates[4], int preserve_uv, uint32_t batch, int ranking,
                    uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits, uint32_t* trials,
                    uint32_t* out_indices, uint32_t* out_faces, float* out_positions, uint8_t* stop,
                    float* out_uv /* 2 per vertex, or NULL */);

/* The same walk over the reference CPU executor's endpoint collapses
 * (legality without placement, ActionState::trial: wedge remap, positions
 * unchanged), ShortestEdge ranking, previous = source: the restatement of
 * neural::execute_actions (action.cpp:453-525) that oracle/_ref runs itself. */
int bo_execute_endpoint(const bo_mesh* source, uint32_t target, uint32_t budget, const bo_eval_settings gates[4],
                        uint32_t batch, uint32_t* commits_from_to, uint32_t capacity, uint32_t* commits,
                        uint32_t* trials, uint32_t* out_indices, uint32_t* out_faces, uint8_t* stop);

#ifdef __cplusplus
}
#endif
#endif
