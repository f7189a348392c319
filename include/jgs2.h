/*
 * jgs2.h — C-ABI of the B200 (sm_100a) JGS2 elastodynamics step.
 *
 * This header is the drop-in boundary for the per-frame simulation loop of
 * CallumFerguson/webgpu-physics.  Every entry point replaces one public member
 * of `class JGS2GpuSolver` (src/simulation/gpu/jgs2-solver.ts:905-3051); the
 * citation beside each declaration names the member it stands in for.  The
 * input record mirrors `interface JGS2GpuInput` (src/simulation/gpu/layout.ts:41-90)
 * and the settings record mirrors `interface JGS2StepSettings`
 * (src/simulation/gpu/jgs2-solver.ts:64-100).
 *
 * Conventions
 *  - Plain pointers and sizes only.  Arrays use the reference's packing: vec4
 *    per vertex (xyz + w), four u32 per tetrahedron, three padded vec4 columns
 *    of inverse Dm per tetrahedron, row-major 3x3 cubature blocks.
 *  - Every call returns a jgs2_status.  A non-OK status leaves a message that
 *    jgs2_last_error() returns (per solver) or jgs2_global_last_error() returns
 *    (for failures before a solver exists).  The reference throws RangeError /
 *    TypeError / Error with the same conditions.
 *  - One solver owns one CUDA stream and all of its device memory.  Calls on
 *    one solver must come from one host thread at a time.
 *  - Host output buffers are caller owned; the library copies inputs at
 *    create time (the reference copies typed arrays into GPU buffers).
 */
#ifndef JGS2_H_
#define JGS2_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JGS2_ABI_VERSION 1u

typedef enum jgs2_status {
  JGS2_OK = 0,
  JGS2_INVALID_ARGUMENT = 1,  /* RangeError / TypeError in the reference */
  JGS2_INFEASIBLE_INPUT = 2,  /* initial pose fails the determinant / contact preflight */
  JGS2_OUT_OF_MEMORY = 3,
  JGS2_DEVICE_ERROR = 4,      /* CUDA runtime error; message carries the CUDA string */
  JGS2_TIMEOUT = 5,           /* a bounded device wait gave up */
  JGS2_DESTROYED = 6,         /* use after jgs2_destroy (reference: "has been destroyed") */
  JGS2_UNSUPPORTED = 7,       /* feature not built into this library */
  JGS2_NOT_READY = 8          /* diagnostics requested before any stable iteration */
} jgs2_status;

/* Material tags stored in tetMeta.w (src/simulation/gpu/layout.ts:29-30). */
#define JGS2_MATERIAL_COROTATED_LINEAR 0u
#define JGS2_MATERIAL_STABLE_NEO_HOOKEAN 1u

/* Schedules (src/simulation/gpu/jgs2-solver.ts:62). */
#define JGS2_SCHEDULE_JACOBI 0u
#define JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL 1u

/* Limits (src/simulation/gpu/jgs2-solver.ts:145,154,255;
 * src/simulation/gpu/jgs2-globalization.ts:2). */
#define JGS2_MAX_BATCH_FRAMES 240u
#define JGS2_MAX_GLOBALIZED_ITERATIONS_PER_SUBMISSION 2048u
#define JGS2_MAX_SCHEDULE_COLORS 256u
#define JGS2_HISTORY_CAPACITY 64u

/* Record widths in floats (src/simulation/gpu/jgs2-globalization.ts:5-15). */
#define JGS2_LOCAL_DIAGNOSTIC_FLOATS 16u
#define JGS2_HISTORY_RECORD_FLOATS 32u
#define JGS2_CONTROL_RECORD_FLOATS 16u

/*
 * Triangle cloth: JGS2GpuClothInput (src/simulation/gpu/cloth-layout.ts:88-104).
 * St. Venant-Kirchhoff membrane triangles in plane stress and quadratic
 * dihedral hinges over vertices of the same scene.  Hinges are oriented: the
 * hinge (i0, i1, i2, i3) joins triangles (i0, i1, i2) and (i1, i0, i3).  Cloth
 * requires the stable Neo-Hookean path (jgs2-solver.ts:998-1002).
 */
typedef struct jgs2_cloth_input {
  uint32_t vertex_count;                    /* must equal the scene's vertex_count */
  uint32_t triangle_count;
  uint32_t hinge_count;
  uint32_t reserved0;
  const uint32_t* triangle_indices;         /* 3 * triangles */
  const float* triangle_inverse_rest_bases; /* 4 * triangles, row-major 2x2 */
  const float* triangle_rest_areas;         /* triangles, positive */
  const uint32_t* hinge_indices;            /* 4 * hinges */
  const float* hinge_rest_angles;           /* hinges */
  const float* hinge_rest_edge_lengths;     /* hinges, positive */
  float young_modulus;                      /* > 0 */
  float poisson_ratio;                      /* [0, 0.5) */
  float thickness;                          /* > 0 */
  float bending_stiffness;                  /* >= 0 */
} jgs2_cloth_input;

/*
 * Input record: JGS2GpuInput (src/simulation/gpu/layout.ts:41-90).
 * Optional arrays may be NULL.  tet_rest_stiffness may be NULL when every
 * tetrahedron is stable Neo-Hookean (the stable path never reads it).
 */
typedef struct jgs2_input {
  uint32_t vertex_count;
  uint32_t tet_count;
  uint32_t cubature_k;
  uint32_t reserved0;
  const float* positions;          /* 4 * V; w is normalised to one */
  const float* velocities;         /* 4 * V or NULL */
  const float* vertex_rest;        /* 4 * V: rest / pin target xyz, mass w */
  const float* vertex_colors;      /* 4 * V or NULL (render colour, unused by the step) */
  const uint32_t* vertex_info;     /* 4 * V: adjacency start, count, pinned, body */
  const float* external_forces;    /* 3 * V or NULL (objectives.externalForces) */
  const float* target_positions;   /* 3 * V or NULL (objectives.targetPositions) */
  const float* target_stiffnesses; /* V or NULL (objectives.targetStiffnesses) */
  const uint32_t* tet_indices;     /* 4 * T */
  const float* tet_inverse_dm;     /* 12 * T, three padded columns */
  const float* tet_meta;           /* 4 * T: volume, lambda, mu, model tag */
  const float* tet_rest_stiffness; /* 144 * T row-major, or NULL when all stable */
  const uint32_t* adjacency;       /* CSR payload of incident tetrahedra */
  uint64_t adjacency_length;
  const uint32_t* cubature_tet_ids;  /* V * K; 0xffffffff = empty slot */
  const float* cubature_weights;     /* V * K */
  const float* cubature_basis;       /* V * K * 36: four row-major Ubar blocks */
  const jgs2_cloth_input* cloth;     /* NULL: no cloth (input.cloth, layout.ts:62) */
  /* Static IPC contact candidates (input.contactCandidates, layout.ts:63;
   * StaticIpcContactCandidates, src/simulation/cpu/ipc-contact.ts:28-38):
   * four vertex indices per candidate, the vertex-triangle candidates
   * (point, t0, t1, t2) first, then the edge-edge candidates (a0, a1, b0, b1).
   * NULL with zero counts: no contact.  Contact requires the stable
   * Neo-Hookean path (jgs2-solver.ts:1014-1018). */
  const uint32_t* contact_indices;
  uint32_t contact_vertex_triangle_count;
  uint32_t contact_edge_edge_count;
  /* Contact surface for the device broad phase (NULL: none); excludes
   * contact_indices.  No counterpart in the reference, whose candidates are
   * the static superset above. */
  const struct jgs2_contact_surface* contact_surface;
} jgs2_input;

/*
 * Device broad phase over the static candidate superset.  The superset of a
 * surface grows with (surface vertices x triangles + edges^2), so instead of
 * listing it the solver enumerates, every iteration on the device, the
 * superset's candidates whose boxes, widened by each vertex's largest
 * possible motion in the iteration (maxStep for free vertices, the snap to
 * rest for pinned ones), come within the activation distance plus the f32
 * rounding reach; candidates that carry lagged friction stay listed for the
 * frame.  Every candidate left out contributes nothing to the reference's
 * step (no active row, a full safe step, a valid check, zero energy), so
 * the step is the one the static superset gives, in the superset's
 * canonical order.  Requires the Jacobi schedule and maxStep > 0.
 */
typedef struct jgs2_contact_surface {
  uint32_t triangle_count;
  uint32_t reserved0;
  const uint32_t* triangles;     /* 3 * triangle_count vertex indices; any order, duplicates merged */
  uint64_t candidate_capacity;   /* candidates one iteration may list; 0 = 65536 + 16 x (vertices + edges) */
} jgs2_contact_surface;

/*
 * Step settings: JGS2StepSettings (src/simulation/gpu/jgs2-solver.ts:64-100),
 * defaults DEFAULT_JGS2_STEP_SETTINGS (:164-187).
 */
typedef struct jgs2_settings {
  uint32_t schedule;               /* JGS2_SCHEDULE_* */
  uint32_t iterations;
  float timestep;
  float gravity[3];
  float floor_height;
  float floor_stiffness;
  float velocity_damping;
  float regularization;
  float rotation_epsilon;
  float max_step;
  float residual_tolerance;
  float normalized_update_tolerance;
  float contact_tangential_damping;
  float contact_margin;
  float ipc_activation_distance;
  float ipc_minimum_distance;
  float ipc_barrier_stiffness;
  float ipc_friction_coefficient;
  float ipc_friction_velocity_epsilon;
  float ipc_step_safety;
  uint32_t horizontal_body_correction;
  uint32_t parity_mode;
} jgs2_settings;

/* Bits of the override mask: set bit i to take field i from an override
 * record (the reference's Partial<JGS2StepSettings>). */
enum {
  JGS2_SET_SCHEDULE = 1u << 0,
  JGS2_SET_ITERATIONS = 1u << 1,
  JGS2_SET_TIMESTEP = 1u << 2,
  JGS2_SET_GRAVITY = 1u << 3,
  JGS2_SET_FLOOR_HEIGHT = 1u << 4,
  JGS2_SET_FLOOR_STIFFNESS = 1u << 5,
  JGS2_SET_VELOCITY_DAMPING = 1u << 6,
  JGS2_SET_REGULARIZATION = 1u << 7,
  JGS2_SET_ROTATION_EPSILON = 1u << 8,
  JGS2_SET_MAX_STEP = 1u << 9,
  JGS2_SET_RESIDUAL_TOLERANCE = 1u << 10,
  JGS2_SET_NORMALIZED_UPDATE_TOLERANCE = 1u << 11,
  JGS2_SET_CONTACT_TANGENTIAL_DAMPING = 1u << 12,
  JGS2_SET_CONTACT_MARGIN = 1u << 13,
  JGS2_SET_IPC_ACTIVATION_DISTANCE = 1u << 14,
  JGS2_SET_IPC_MINIMUM_DISTANCE = 1u << 15,
  JGS2_SET_IPC_BARRIER_STIFFNESS = 1u << 16,
  JGS2_SET_IPC_FRICTION_COEFFICIENT = 1u << 17,
  JGS2_SET_IPC_FRICTION_VELOCITY_EPSILON = 1u << 18,
  JGS2_SET_IPC_STEP_SAFETY = 1u << 19,
  JGS2_SET_HORIZONTAL_BODY_CORRECTION = 1u << 20,
  JGS2_SET_PARITY_MODE = 1u << 21,
  JGS2_SET_ALL = (1u << 22) - 1u
};

typedef struct jgs2_solver jgs2_solver;

/* Solver shape and activity, the reference's readonly members and getters
 * (src/simulation/gpu/jgs2-solver.ts:905-969, 1504-1575). */
typedef struct jgs2_info {
  uint32_t vertex_count;
  uint32_t tet_count;
  uint32_t cubature_k;
  uint32_t body_count;
  uint32_t schedule_color_count;
  uint32_t globalization_enabled;  /* 1 for the stable Neo-Hookean path */
  uint32_t objective_flags;        /* bit0 forces, bit1 targets */
  uint32_t external_force_vertex_count;
  uint32_t quadratic_target_vertex_count;
  uint32_t objective_revision;
  uint32_t last_submitted_iterations;
  uint32_t history_count;          /* executed records of the last frame */
  float scene_scale;               /* initial dynamic AABB diagonal */
  float preprocessing_timestep;
  uint32_t current_position_buffer;/* 0 = A, reported for zero-copy consumers */
  uint32_t cloth_triangle_count;   /* clothTriangleCount (:911) */
  uint32_t contact_candidate_count;/* contactCandidateCount; with a contact surface, the
                                      candidates of the last iteration */
  uint32_t contact_candidate_capacity; /* broad-phase capacity (0 for static candidates) */
} jgs2_info;

/* ---- library ---------------------------------------------------------- */

/* ABI version and build string. */
uint32_t jgs2_version(void);
const char* jgs2_build_string(void);
/* Message of the last failure that happened without a solver (create). */
const char* jgs2_global_last_error(void);

/* DEFAULT_JGS2_STEP_SETTINGS (src/simulation/gpu/jgs2-solver.ts:164-187). */
void jgs2_default_settings(jgs2_settings* out);

/* resolveJGS2StepSettings + validateStepSettings
 * (src/simulation/gpu/jgs2-solver.ts:429-550): merge, apply parity, validate. */
jgs2_status jgs2_resolve_settings(const jgs2_settings* defaults,
                                  const jgs2_settings* overrides,
                                  uint32_t override_mask, jgs2_settings* out);

/* validateJGS2GpuInput (src/simulation/gpu/layout.ts:223-416). */
jgs2_status jgs2_validate_input(const jgs2_input* input);

/* minimumStaticIpcContactDistance (src/simulation/cpu/ipc-contact.ts:385) in
 * double at input->positions: over the static candidates, or over the
 * superset of input->contact_surface restricted to pairs whose boxes come
 * within `cutoff` (+infinity when none does).  The exact intersection check
 * of a contact run: feed it the positions read back after each frame. */
jgs2_status jgs2_minimum_contact_distance(const jgs2_input* input, double cutoff, double* distance);

/* The device closest-feature routine of the IPC passes on caller pairs
 * (a diagnostic): the GPU counterpart of evaluateIpcVertexTriangleDistance
 * and evaluateIpcEdgeEdgeDistance (src/simulation/cpu/ipc-contact.ts:194,
 * 277), i.e. jgs2_ipc_point_triangle_contact / jgs2_ipc_edge_edge_contact
 * (src/simulation/gpu/ipc-contact-wgsl.ts:151, 228) as every contact pass of
 * this library evaluates them: f32, with near-degenerate pairs (sliver
 * triangles, near-parallel edges, near-touching features) recomputed in FP64
 * and rounded once.  points: 12 floats per pair (type 0: point, triangle;
 * type 1: edge a, edge b); types: 0 or 1 per pair; out: 9 floats per pair
 * (distance, normal xyz, weights xyzw with sum w_i x_i = a - b, valid);
 * fp64_used (may be NULL): 1 where the FP64 run was taken.  Host arrays; the
 * call allocates and frees its own device buffers on `device`. */
jgs2_status jgs2_evaluate_contact_features(const float* points, const uint32_t* types, uint32_t count,
                                           float* out, uint32_t* fp64_used, int device);

/* Candidates of the static superset of input->contact_surface (what
 * buildStaticIpcContactCandidates would list), counted without listing. */
jgs2_status jgs2_contact_superset_size(const jgs2_input* input, uint64_t* count);

/* buildJGS2InputVertexColoring + buildGreedyVertexColoring
 * (src/simulation/gpu/jgs2-solver.ts:308-367;
 *  src/simulation/cpu/vertex-coloring.ts:20-110).  colors has V entries. */
jgs2_status jgs2_build_vertex_coloring(const jgs2_input* input,
                                       uint32_t* colors,
                                       uint32_t* color_count);

/* ---- lifetime --------------------------------------------------------- */

/* static JGS2GpuSolver.create(device, input, settings)
 * (src/simulation/gpu/jgs2-solver.ts:971-1502).  device is a CUDA ordinal. */
jgs2_status jgs2_create(const jgs2_input* input, const jgs2_settings* settings,
                        uint32_t settings_mask, int device, jgs2_solver** out);

/* destroy() (src/simulation/gpu/jgs2-solver.ts:3029-3044); idempotent, NULL ok. */
void jgs2_destroy(jgs2_solver* solver);

/* Message of this solver's last failure. */
const char* jgs2_last_error(const jgs2_solver* solver);

/* Shape / activity getters. */
jgs2_status jgs2_get_info(jgs2_solver* solver, jgs2_info* out);

/* Settings getters: defaultStepSettings / lastSubmittedSettings (:1550-1556). */
jgs2_status jgs2_get_default_settings(jgs2_solver* solver, jgs2_settings* out);
jgs2_status jgs2_get_last_submitted_settings(jgs2_solver* solver,
                                             jgs2_settings* out);

/* ---- stepping (all asynchronous on the solver stream) ----------------- */

/* step(overrides) (src/simulation/gpu/jgs2-solver.ts:1767-1782): odd
 * iteration normalisation and the convergence stop latch. */
jgs2_status jgs2_step(jgs2_solver* solver, const jgs2_settings* overrides,
                      uint32_t override_mask);

/* stepFrames(n, overrides) (:1791-1810). */
jgs2_status jgs2_step_frames(jgs2_solver* solver, uint32_t frame_count,
                             const jgs2_settings* overrides,
                             uint32_t override_mask);

/* stepExactIterations(iterations, overrides) (:1817-1835). */
jgs2_status jgs2_step_exact_iterations(jgs2_solver* solver, uint32_t iterations,
                                       const jgs2_settings* overrides,
                                       uint32_t override_mask);

/* stepFramesExactIterations(n, iterations, overrides) (:1842-1862). */
jgs2_status jgs2_step_frames_exact_iterations(jgs2_solver* solver,
                                              uint32_t frame_count,
                                              uint32_t iterations,
                                              const jgs2_settings* overrides,
                                              uint32_t override_mask);

/* awaitIdle() (:2496-2499). */
jgs2_status jgs2_sync(jgs2_solver* solver);

/* Per-kernel GPU timing of stepped frames: the counterpart of the reference's
 * GPU-timestamp step variants (stepWithGpuTimestamp / stepFramesWith-
 * GpuTimestampWrites, :1869-1972).  Frames run exactly like
 * jgs2_step_frames_exact_iterations but without graph replay, with a CUDA
 * event pair around every kernel on the solver stream; the call waits for the
 * frames and fills one entry per kernel kind. */
#define JGS2_PROFILE_KINDS 9
typedef struct jgs2_kernel_profile {
  uint32_t kinds;
  uint32_t launches[JGS2_PROFILE_KINDS];
  double milliseconds[JGS2_PROFILE_KINDS];
  char names[JGS2_PROFILE_KINDS][24];
} jgs2_kernel_profile;

jgs2_status jgs2_step_with_gpu_timestamps(jgs2_solver* solver, uint32_t frame_count, uint32_t iterations,
                                          const jgs2_settings* overrides, uint32_t override_mask,
                                          jgs2_kernel_profile* out);

/* ---- objectives -------------------------------------------------------- */

/* setExternalForce (:1576-1611). */
jgs2_status jgs2_set_external_force(jgs2_solver* solver, uint32_t vertex,
                                    const float force[3]);
/* replaceExternalForces (:1614-1642); forces has 3 * V floats. */
jgs2_status jgs2_replace_external_forces(jgs2_solver* solver,
                                         const float* forces);
/* clearExternalForces (:1644-1646). */
jgs2_status jgs2_clear_external_forces(jgs2_solver* solver);
/* setQuadraticTarget (:1649-1688). */
jgs2_status jgs2_set_quadratic_target(jgs2_solver* solver, uint32_t vertex,
                                      const float target[3], float stiffness);
/* replaceQuadraticTargets (:1691-1733). */
jgs2_status jgs2_replace_quadratic_targets(jgs2_solver* solver,
                                           const float* target_positions,
                                           const float* target_stiffnesses);
/* releaseQuadraticTarget (:1736-1750). */
jgs2_status jgs2_release_quadratic_target(jgs2_solver* solver, uint32_t vertex);
/* releaseAllQuadraticTargets (:1753-1760). */
jgs2_status jgs2_release_all_quadratic_targets(jgs2_solver* solver);

/* ---- reads (synchronous: they wait for the solver stream) -------------- */

/* readPositions (:2501-2508); out has 4 * V floats. */
jgs2_status jgs2_read_positions(jgs2_solver* solver, float* out, size_t floats);
/* readPositions as the reference uses it (an asynchronous read resolved
 * later, :2501-2508 returns a Promise): enqueues the copy of the positions
 * after the work already submitted on the solver's stream and returns at
 * once.  `out` (4 * V floats; page-locked memory for a truly asynchronous
 * copy) must stay valid and unread until jgs2_wait_reads returns; later
 * steps may be submitted meanwhile, so the host's next frame overlaps the
 * copy and the device's work. */
jgs2_status jgs2_read_positions_async(jgs2_solver* solver, float* out, size_t floats);
/* Waits for every asynchronous read submitted so far (and reports a device
 * failure of the work before them, like any synchronising call). */
jgs2_status jgs2_wait_reads(jgs2_solver* solver);
/* readVelocities (:2510-2518). */
jgs2_status jgs2_read_velocities(jgs2_solver* solver, float* out, size_t floats);
/* readPredictedPositions (:2520-2528). */
jgs2_status jgs2_read_predicted_positions(jgs2_solver* solver, float* out,
                                          size_t floats);
/* readFinalIterationUpdates (:2535-2543). */
jgs2_status jgs2_read_final_iteration_updates(jgs2_solver* solver, float* out,
                                              size_t floats);
/* readVertexRotations (:2863-2870); 12 * V floats (three padded columns). */
jgs2_status jgs2_read_vertex_rotations(jgs2_solver* solver, float* out,
                                       size_t floats);
/* readGlobalizationDiagnostics (:2548-2604).  local: 16 * V floats (may be
 * NULL), control: 16 floats (may be NULL), history: 32 * 64 floats (may be
 * NULL).  *history_count receives the executed record count. */
jgs2_status jgs2_read_globalization(jgs2_solver* solver, float* local,
                                    size_t local_floats, float* control,
                                    float* history, size_t history_floats,
                                    uint32_t* history_count);

/* The IPC candidates of the last iteration (4 u32 each: VT point, t0, t1,
 * t2 or EE a0, a1, b0, b1 with bit 31 of the fourth set, canonical order).
 * *count receives the number
 * listed; out (may be NULL) holds `capacity` candidates.  Static candidates
 * are listed as given.  With a contact surface, a broad-phase list that did
 * not fit its capacity fails the step and this read with JGS2_DEVICE_ERROR. */
/* readOracleDiagnostics (src/simulation/gpu/jgs2-solver.ts:2882-2907;
 * JGS2GpuOracleDiagnostics, src/simulation/gpu/jgs2-diagnostics.ts:31-111):
 * the exact, all-element frozen-frame implicit-Euler oracle at the current
 * canonical pose against the last submitted inertial target and settings.
 * Opt-in: the frame loop never runs it; its device records are allocated at
 * the first call.  Fails with JGS2_UNSUPPORTED while IPC contact is enabled
 * (the reference excludes contact energy); cloth terms are not included, as
 * in the reference.  vertex_records (may be NULL) receive 36 floats per
 * vertex in the reference's layout (gradient + active; the Hessian block's
 * rows with inertia energy, floor energy and update magnitude beside them;
 * squared gradient norm, finite, inertia weight, update valid; inertia,
 * elasticity and floor squared norms, floor distance; floor active; external
 * force gradient + energy; target gradient + energy); tet_records (may be
 * NULL) 4 floats per tet (energy, determinant, finite, 0).  Sums in double. */
typedef struct jgs2_oracle_diagnostics {
  double energy;  /* the five components summed */
  double inertia, elasticity, external_force, quadratic_target, floor_contact;
  /* component gradient norms, in the production convergence order */
  double inertia_gradient_norm, material_gradient_norm, external_force_gradient_norm, target_gradient_norm,
      contact_gradient_norm;
  double gradient_norm, gradient_squared_norm, residual_denominator, relative_residual;
  double maximum_update, minimum_deformation_determinant, minimum_contact_distance;
  uint32_t active_vertex_count, active_contact_count;
  uint32_t relative_residual_valid, gradient_valid, maximum_update_valid, minimum_deformation_determinant_valid;
  uint32_t minimum_contact_distance_valid, finite;
} jgs2_oracle_diagnostics;
jgs2_status jgs2_read_oracle_diagnostics(jgs2_solver* solver, jgs2_oracle_diagnostics* out, float* vertex_records,
                                         size_t vertex_floats, float* tet_records, size_t tet_floats);

jgs2_status jgs2_read_contact_candidates(jgs2_solver* solver, uint32_t* out,
                                         uint64_t capacity, uint64_t* count);

/* evaluateAssembledCandidateForTest(source, candidate, overrides)
 * (:2611-2726): run the production assembled gate (vertex energies,
 * candidate determinants, reduce, whole-pose revert) and the convergence
 * reduction once on a given source / candidate pose pair (4 * V floats each,
 * host).  The canonical pose becomes the accepted one.  positions_out (4 * V),
 * control_out (16) and history_out (32: the single record) may be NULL. */
jgs2_status jgs2_evaluate_assembled_candidate(jgs2_solver* solver, const float* source_positions,
                                              const float* candidate_positions,
                                              const jgs2_settings* overrides, uint32_t override_mask,
                                              float* positions_out, float* control_out, float* history_out);

/* Allocation-free assembled gate.  This entry point has no counterpart in
 * the reference.  It evaluates the same determinant gate and assembled
 * energies as jgs2_evaluate_assembled_candidate, with the sweep records
 * taken as cleared, over caller DEVICE arrays: source, candidate and
 * predicted positions (4 * V floats each, 16-byte aligned), and writes the
 * 16-float control record (minimum determinants and validity bits, accept /
 * revert flags, energies, sweep aggregates; history slot 0) to the device
 * array control_out.  It reads the solver's mesh data and also its mutable
 * external-force, quadratic-target and rest-mass arrays, and changes no
 * solver state.  Solvers with IPC contact candidates get JGS2_UNSUPPORTED.
 *
 * It allocates no device memory: its reduction scratch is a fixed static
 * device array of 262,400 bytes (8192 block partials of 32 bytes after a
 * 256-byte header).  So the largest of vertex_count, tet_count and the cloth
 * triangle and hinge counts may be at most 1,048,576 (8192 blocks of 128);
 * larger solvers get JGS2_INVALID_ARGUMENT.
 * The first call on each device looks up the scratch address there (this may
 * load the kernel module onto the device), so make one call before any stream
 * capture begins.  The scratch's ticket word must start at zero: module load
 * zeroes it and every launch leaves it zero.  Calls whose launches overlap in
 * time on one device (different streams, threads or solvers) share the
 * scratch and race; order them.  stream is a cudaStream_t, or NULL for the
 * solver's stream; the call is asynchronous on it.  A non-NULL stream must be
 * ordered after the solver's stream (for example by an event wait), or the
 * solver's objectives must not change while the call is in flight: the read
 * of the force and target arrays is otherwise unordered against a step or an
 * objective upload on the solver's stream.  The looked-up scratch address is
 * kept for the life of the process: a device reset (cudaDeviceReset) or an
 * unload and reload of this library in the same process is not supported. */
jgs2_status jgs2_gate_candidate_no_alloc(jgs2_solver* solver, const float* device_source,
                                         const float* device_candidate, const float* device_predicted,
                                         const jgs2_settings* overrides, uint32_t override_mask,
                                         float* device_control_out, void* stream);

/* Checkpoint / resume.  The reference keeps no such call (its state lives in
 * GPU buffers for the page's lifetime); these serialise what the reference's
 * step carries from one frame to the next (positions, velocities, the
 * objectives, the frame's diagnostics records) so a run can be stopped and
 * resumed, or replayed, bit for bit.  The image is self-describing (magic,
 * version, element counts) and host-endian.
 * jgs2_export_state: *size receives the image's byte count; with out == NULL
 * nothing else happens.  Waits for the solver's stream.
 * jgs2_import_state: restores an image exported by a solver created from an
 * input with the same counts; the next step then continues exactly as the
 * exporting solver's would.  Single-scene solvers only. */
jgs2_status jgs2_export_state(jgs2_solver* solver, void* out, size_t capacity, size_t* size);
jgs2_status jgs2_import_state(jgs2_solver* solver, const void* image, size_t size);

/* Zero-copy consumers (the reference's currentPositionBuffer, :1504-1507):
 * device address of the canonical vec4 position array and the solver's
 * cudaStream_t.  Valid until jgs2_destroy. */
jgs2_status jgs2_device_positions(jgs2_solver* solver, void** device_ptr,
                                  void** cuda_stream);

/* Device kernels launched by this solver since creation (every launch the
 * library issues is counted, including graph replays). */
uint64_t jgs2_kernel_launch_count(const jgs2_solver* solver);

/* Launch shapes and their autotuner (no counterpart in the reference, whose
 * workgroup sizes are fixed in its shaders).  A shape sets how many vertices
 * one block of the local-solve kernel takes: the default (32 vertices of 4
 * lanes, or 4 warps of the contact-heavy warp-per-vertex form, fewer when
 * the cubature cache fills shared memory) shifted right by the shape, 0-2.
 * Each vertex's arithmetic is the same in every shape, so results are
 * bit-identical whichever shape runs.
 *
 * jgs2_autotune starts online tuning: the next rounds x JGS2_LAUNCH_SHAPES
 * frames stepped (by any step call) take the shapes in turn, each timed with
 * a CUDA event pair (the stream waits after each timed frame), and the shape
 * with the smallest median frame time is then kept.  rounds must be 1-64.
 * jgs2_set_launch_shape fixes a shape (a cached choice) and ends tuning. */
#define JGS2_LAUNCH_SHAPES 3
typedef struct jgs2_launch_shape {
  uint32_t shape;                     /* the shape in use, 0-2 */
  uint32_t solve_vertices_per_block;  /* of the 4-lane form, for this K */
  uint32_t tuning;                    /* frames still to time, 0 when done */
  uint32_t samples;                   /* fewest frames timed for one shape */
  double frame_ms[JGS2_LAUNCH_SHAPES];/* median timed frame per shape, 0 = none */
} jgs2_launch_shape;
jgs2_status jgs2_autotune(jgs2_solver* solver, uint32_t rounds);
jgs2_status jgs2_get_launch_shape(jgs2_solver* solver, jgs2_launch_shape* out);
jgs2_status jgs2_set_launch_shape(jgs2_solver* solver, uint32_t shape);

/* ---- batched form ---------------------------------------------------------
 * Many independent scenes stepped together by one launch sequence.  The
 * reference has no batched solver: each scene would be its own
 * JGS2GpuSolver.  A batch keeps every scene's semantics: its own settings,
 * its own assembled gate (a rejected candidate reverts only that scene), its
 * own convergence history and stop latch.  Scenes are concatenated in device
 * memory; kernels look up the scene of each vertex and the gate and
 * convergence reductions are segmented per scene. */
typedef struct jgs2_batch jgs2_batch;

/* inputs: scene_count scene inputs (validated and copied as jgs2_create
 * does); settings / masks: NULL or one per scene. */
jgs2_status jgs2_batch_create(const jgs2_input* const* inputs, uint32_t scene_count,
                              const jgs2_settings* settings, const uint32_t* masks, int device,
                              jgs2_batch** out);
void jgs2_batch_destroy(jgs2_batch* batch);
const char* jgs2_batch_last_error(const jgs2_batch* batch);
uint32_t jgs2_batch_scene_count(const jgs2_batch* batch);
/* Total vertices over all scenes. */
uint32_t jgs2_batch_vertex_count(const jgs2_batch* batch);

/* Advance every scene `frames` frames.  exact_iterations > 0 runs exactly
 * that many iterations per frame (stepFramesExactIterations); 0 runs the
 * production step (odd-normalised iteration count with the stop latch), and
 * then every scene's normalised count must agree.  overrides / masks: NULL or
 * one per scene.  All scenes must use the same schedule; a batch steps with the
 * graph-coloured schedule only if one of its scenes had that schedule at
 * creation (the colouring is built then). */
jgs2_status jgs2_batch_step_frames(jgs2_batch* batch, uint32_t frames, uint32_t exact_iterations,
                                   const jgs2_settings* overrides, const uint32_t* masks);
jgs2_status jgs2_batch_sync(jgs2_batch* batch);
jgs2_status jgs2_batch_get_info(jgs2_batch* batch, uint32_t scene, jgs2_info* out);
/* Per-scene reads, laid out as the solver reads. */
jgs2_status jgs2_batch_read_positions(jgs2_batch* batch, uint32_t scene, float* out, size_t floats);
jgs2_status jgs2_batch_read_velocities(jgs2_batch* batch, uint32_t scene, float* out, size_t floats);
jgs2_status jgs2_batch_read_globalization(jgs2_batch* batch, uint32_t scene, float* local,
                                          size_t local_floats, float* control, float* history,
                                          size_t history_floats, uint32_t* history_count);
/* Positions of all scenes, concatenated in scene order (4 floats per vertex). */
jgs2_status jgs2_batch_read_all_positions(jgs2_batch* batch, float* out, size_t floats);
uint64_t jgs2_batch_kernel_launch_count(const jgs2_batch* batch);
/* Launch shapes of a batch, as jgs2_autotune / jgs2_get_launch_shape /
 * jgs2_set_launch_shape for a solver. */
jgs2_status jgs2_batch_autotune(jgs2_batch* batch, uint32_t rounds);
jgs2_status jgs2_batch_get_launch_shape(jgs2_batch* batch, jgs2_launch_shape* out);
jgs2_status jgs2_batch_set_launch_shape(jgs2_batch* batch, uint32_t shape);
/* The batch's CUDA stream (a cudaStream_t), for event timing and ordering. */
void* jgs2_batch_stream(const jgs2_batch* batch);
/* An inactive scene sits every following frame out: its state stays as it
 * is until it is made active again (used to retire finished requests). */
jgs2_status jgs2_batch_set_scene_active(jgs2_batch* batch, uint32_t scene, uint32_t active);
/* Device bytes a scene occupies once packed (the serving admission estimate). */
uint64_t jgs2_estimate_device_bytes(const jgs2_input* input);

#ifdef __cplusplus
}
#endif

#endif /* JGS2_H_ */
