/*
 * jgs2_scene.h — C-ABI of the host-side scene builder and JGS2 precompute
 * that produce a jgs2_input for the step.
 *
 * The reference builds scenes in TypeScript: procedural tetrahedral meshes
 * (src/simulation/cpu/mesh.ts:101-201), FEM rest data and lumped masses
 * (src/simulation/cpu/fem.ts:70-335), the exact full-coordinate JGS2 bases
 * (src/simulation/cpu/precompute.ts:141-206), the nonlinear cubature pose
 * corpus and training (src/simulation/cpu/nonlinear-cubature.ts:452-620;
 * src/simulation/cpu/nonlinear-cubature-training.ts:689-843) and the GPU
 * packer toJGS2GpuInput (src/scenes/index.ts:975-1114).  This library restates
 * that pipeline in C++ (double precision, OpenMP over source vertices).
 *
 * Two precompute methods:
 *  - JGS2_PRECOMPUTE_EXACT: the reference's method on the whole mesh (dense
 *    rest Hessian + Cholesky, global low-frequency pose corpus, candidate
 *    tetrahedra = all tetrahedra).  Cost grows as O(n^3); meant for meshes of a
 *    few thousand vertices.
 *  - JGS2_PRECOMPUTE_PATCH: the same algorithm applied to a local patch around
 *    each source vertex (free vertices within `patch_radius` graph rings,
 *    everything beyond held fixed, candidate tetrahedra = tetrahedra incident
 *    to the free vertices).  Patches with identical rest geometry, topology,
 *    material, masses and pin flags share one training result, so regular
 *    grids precompute in seconds at millions of vertices.
 */
#ifndef JGS2_SCENE_H_
#define JGS2_SCENE_H_

#include "jgs2.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct jgs2_scene jgs2_scene;

#define JGS2_PRECOMPUTE_EXACT 0u
#define JGS2_PRECOMPUTE_PATCH 1u

/* Where the greedy cubature selection (the nonnegative least-squares search,
 * src/simulation/cpu/cubature.ts:387-690) runs.  Both give the same records
 * bit for bit; the GPU runs every training problem of a batch at once on the
 * current CUDA device. */
#define JGS2_SELECTION_CPU 0u
#define JGS2_SELECTION_GPU 1u   /* error unless the current CUDA device is sm_100 */
#define JGS2_SELECTION_AUTO 2u  /* the GPU when the current CUDA device is sm_100 */

/* Face bits for generated cuboids: a vertex is pinned when it lies on any
 * selected face (the reference passes a predicate, src/simulation/cpu/mesh.ts:142). */
#define JGS2_FACE_X_MIN (1u << 0)
#define JGS2_FACE_X_MAX (1u << 1)
#define JGS2_FACE_Y_MIN (1u << 2)
#define JGS2_FACE_Y_MAX (1u << 3)
#define JGS2_FACE_Z_MIN (1u << 4)
#define JGS2_FACE_Z_MAX (1u << 5)

typedef struct jgs2_precompute_options {
  double timestep;          /* the step's timestep; bases include M / h^2 */
  uint32_t cubature_k;      /* settings.cubatureSamples (6 in every reference scene) */
  uint32_t method;          /* JGS2_PRECOMPUTE_* */
  uint32_t patch_radius;    /* free rings around the source vertex (patch method) */
  uint32_t threads;         /* 0 = all hardware threads */
  uint32_t mode_count;      /* training modes, 8 (nonlinear-cubature.ts:13;
                             * precompute.ts:20 for co-rotated scenes) */
  uint32_t inverse_iterations; /* 24 (nonlinear-cubature.ts:15; precompute.ts:21) */
  double training_amplitude;   /* 0.12 (nonlinear-cubature.ts:16) */
  uint32_t refinement_passes;  /* 12 (nonlinear-cubature-training.ts:737);
                                * co-rotated scenes use 4 (cubature.ts:52) */
  /* Nonzero: skip training and write the exact complement instead — one
   * weight-1 record per candidate tetrahedron (the "exact-all remainder" of
   * assembleStableNeoHookeanJGS2LocalSystem, nonlinear-cubature-training.ts:
   * 620-660).  cubature_k must then be at least the candidate count. */
  uint32_t exact_complement;
  uint32_t selection_device;   /* JGS2_SELECTION_*, default JGS2_SELECTION_AUTO */
} jgs2_precompute_options;

typedef struct jgs2_precompute_stats {
  uint32_t source_vertices;    /* active vertices that received records */
  uint32_t training_classes;   /* distinct trainings run (patch caching) */
  uint32_t records_written;    /* positive-weight records */
  uint32_t max_records_per_vertex;
  double max_residual;         /* max normalized training residual (f64) */
  double mean_residual;
  uint32_t vertices_over_tolerance; /* residual > 1% */
  uint32_t reduced_amplitude_classes; /* corpora whose amplitude was halved */
  double seconds;
  uint32_t selection_on_gpu;   /* 1 when the selections ran on the GPU */
  uint32_t selection_batches;  /* GPU selection launches */
  double training_seconds;     /* wall time of the training phase (systems, selections, records) */
  double selection_seconds;    /* wall time inside the GPU selection calls (copies and kernel) */
} jgs2_precompute_stats;

jgs2_scene* jgs2_scene_new(void);
void jgs2_scene_destroy(jgs2_scene* scene);
const char* jgs2_scene_last_error(const jgs2_scene* scene);

/* Defaults of jgs2_precompute_options. */
void jgs2_default_precompute_options(jgs2_precompute_options* out);

/* LinearMaterial (src/simulation/cpu/types.ts) with its model tag.  Returns the
 * material id (>= 0) or -1. */
int32_t jgs2_scene_add_material(jgs2_scene* scene, double density,
                                double young_modulus, double poisson_ratio,
                                uint32_t model);

/* generateRegularCuboidMesh (src/simulation/cpu/mesh.ts:101-201) appended as
 * one body.  Returns the first vertex id of the new body or -1. */
int64_t jgs2_scene_add_cuboid(jgs2_scene* scene, const uint32_t cells[3],
                              const double origin[3], const double size[3],
                              uint32_t material, uint32_t body,
                              uint32_t pinned_faces);

/* Generic tetrahedral body (appendTetrahedralMeshes, mesh.ts:254-301).
 * tet_materials may be NULL (all `material`). pinned may be NULL. */
int64_t jgs2_scene_add_mesh(jgs2_scene* scene, uint32_t vertex_count,
                            const double* positions, uint32_t tet_count,
                            const uint32_t* tets, const uint32_t* tet_materials,
                            uint32_t material, const uint8_t* pinned,
                            uint32_t body);

/* Triangle cloth appended as one body: SceneDefinition.cloth
 * (src/scenes/index.ts:632-720) with its areal masses density * thickness *
 * area / 3 per triangle vertex (validateAndAddClothMasses,
 * src/simulation/cpu/precompute.ts:44-95).  triangles index the new vertices
 * (0 .. vertex_count - 1); pinned may be NULL.  A scene holds one cloth
 * material.  The packer derives the rest bases, rest areas, hinges and rest
 * dihedrals (buildJGS2GpuClothInput, src/scenes/index.ts:881-973) and points
 * jgs2_input.cloth at them.  Returns the first vertex id or -1. */
int64_t jgs2_scene_add_cloth(jgs2_scene* scene, uint32_t vertex_count, const double* positions,
                             uint32_t triangle_count, const uint32_t* triangles, const uint8_t* pinned,
                             uint32_t body, double density, double young_modulus, double poisson_ratio,
                             double thickness, double bending_stiffness);
uint32_t jgs2_scene_cloth_triangle_count(const jgs2_scene* scene);

/* Replace the rest positions of every vertex (3 * V doubles) and re-orient the
 * tetrahedra, as transformTetrahedralMesh does (src/simulation/cpu/mesh.ts:
 * 237-280) for rotated, warped or translated bodies. */
jgs2_status jgs2_scene_set_rest_positions(jgs2_scene* scene, const double* positions);

/* IPC contact over the scene's surface (the tet boundary plus the cloth
 * triangles).  JGS2_SCENE_CONTACT_STATIC: the packer enumerates the static
 * candidates (buildStaticIpcContactCandidates,
 * src/simulation/cpu/ipc-contact.ts:591-665) into jgs2_input.contact_indices;
 * the enumeration is quadratic in the surface size, like the reference's
 * static superset.  JGS2_SCENE_CONTACT_SURFACE: the packer hands the surface
 * to the device broad phase (jgs2_input.contact_surface) with
 * `candidate_capacity` (0: the default).  JGS2_SCENE_CONTACT_NONE: no
 * contact. */
#define JGS2_SCENE_CONTACT_NONE 0u
#define JGS2_SCENE_CONTACT_STATIC 1u
#define JGS2_SCENE_CONTACT_SURFACE 2u
jgs2_status jgs2_scene_set_contact(jgs2_scene* scene, uint32_t mode);
jgs2_status jgs2_scene_set_contact_capacity(jgs2_scene* scene, uint64_t candidate_capacity);

/* buildStaticIpcContactCandidates (src/simulation/cpu/ipc-contact.ts:591-665)
 * for an arbitrary triangle surface: returns the candidate count (-1 on
 * invalid input) and, when out holds at least that many candidates (4 u32
 * each), writes them, vertex-triangle first. */
int64_t jgs2_build_static_contact_candidates(uint32_t vertex_count, const uint32_t* triangles,
                                             uint32_t triangle_count, uint32_t* out, uint64_t capacity,
                                             uint32_t* vertex_triangle_count, uint32_t* edge_edge_count);

/* Replace the pin flags of every vertex (V bytes, nonzero = pinned); the
 * reference's cuboid generator takes an arbitrary predicate (mesh.ts:142). */
jgs2_status jgs2_scene_set_pinned(jgs2_scene* scene, const uint8_t* pinned);

uint32_t jgs2_scene_vertex_count(const jgs2_scene* scene);
uint32_t jgs2_scene_tet_count(const jgs2_scene* scene);
/* Rest positions (3 * V doubles). */
jgs2_status jgs2_scene_rest_positions(const jgs2_scene* scene, double* out);

/* Run the precompute.  options may be NULL for defaults. */
jgs2_status jgs2_scene_precompute(jgs2_scene* scene,
                                  const jgs2_precompute_options* options,
                                  jgs2_precompute_stats* stats);

/* selectGreedyNonnegativeColumns (src/simulation/cpu/cubature.ts:508-690),
 * through the cubature trainer's own selection core.  columns: column_count
 * columns of `rows` values each, stored one column after another; target:
 * `rows` values.  The columns whose squared norm exceeds 1e-18 are the
 * candidates.  Each greedy step appends the candidate whose nonnegative
 * least-squares fit leaves the smallest residual, ties going to the lower
 * index.  Growth stops at max_columns (at most 12), when no candidate
 * helps, or when the normalised residual drops below residual_tolerance.
 * Then refinement_passes swap passes follow.  selected and weights receive
 * *selected_count entries in selection order; normalized_residual is the
 * final residual over the target norm (0 for a zero target, 1 when no
 * candidate exists).  Invalid sizes, non-finite values or a tolerance
 * outside [0, 1] give JGS2_INVALID_ARGUMENT. */
jgs2_status jgs2_select_nonnegative_columns(const double* columns, uint32_t column_count, uint32_t rows,
                                            const double* target, uint32_t max_columns,
                                            uint32_t refinement_passes, double residual_tolerance,
                                            uint32_t* selected, double* weights, uint32_t* selected_count,
                                            double* normalized_residual);

/* Initial pose (4 * V floats, xyz used) and optional velocities (4 * V).
 * With pin_at_initial != 0 the pin targets (vertex_rest.xyz of pinned
 * vertices) are set to the initial positions instead of the rest positions. */
jgs2_status jgs2_scene_set_initial_state(jgs2_scene* scene,
                                         const float* positions,
                                         const float* velocities,
                                         uint32_t pin_at_initial);

/* Objectives packed into the input (objectives.*, layout.ts:32-39). */
jgs2_status jgs2_scene_set_objectives(jgs2_scene* scene,
                                      const float* external_forces,
                                      const float* target_positions,
                                      const float* target_stiffnesses);

/* packJGS2GpuInput (src/scenes/index.ts:975-1109): fill `out` with pointers
 * into arrays owned by the scene (valid until the next mutating call or
 * jgs2_scene_destroy).  Requires a finished precompute. */
jgs2_status jgs2_scene_pack(jgs2_scene* scene, jgs2_input* out);

#ifdef __cplusplus
}
#endif

#endif /* JGS2_SCENE_H_ */
