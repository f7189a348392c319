// Host runtime of the JGS2 step: the C-ABI of include/jgs2.h.
//
// Restates the host half of `class JGS2GpuSolver`
// (src/simulation/gpu/jgs2-solver.ts:905-3051): settings resolution and
// validation (:429-550), input validation (layout.ts:223-416), greedy
// colouring (:308-367 with src/simulation/cpu/vertex-coloring.ts:20-110),
// create-time feasibility checks (:1041-1083, 820-893), the per-frame
// dispatch order (:2207-2494) and the objective / readback API
// (:1576-1760, 2501-2604).  Device work is issued on one CUDA stream per
// solver; each frame shape is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <atomic>
#include <thread>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "jgs2.h"
#include "jgs2_kernels.cuh"

namespace {

using jgs2::Buffers;
using jgs2::DevParams;
using jgs2::FrameState;

constexpr float kDeterminantFloor = 1e-4f;
// jgs2-globalization.ts:40; compared in f32 because settings cross the ABI as f32.
constexpr float kMaxRuntimeTolerance = 1e-3f;
constexpr double kDegenerateSceneScale = 1e-12;    // jgs2-solver.ts:162
constexpr uint32_t kEmptyTet = 0xffffffffu;

thread_local std::string gGlobalError;

struct Error {
  jgs2_status status;
  std::string message;
};

std::string format(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return buf;
}

// ---- settings ---------------------------------------------------------------

void defaults(jgs2_settings* s) {
  std::memset(s, 0, sizeof(*s));
  s->schedule = JGS2_SCHEDULE_JACOBI;
  s->iterations = 9;
  s->timestep = static_cast<float>(1.0 / 60.0);
  s->gravity[0] = 0.f;
  s->gravity[1] = -9.81f;
  s->gravity[2] = 0.f;
  s->floor_height = 0.f;
  s->floor_stiffness = 20000.f;
  s->velocity_damping = 0.999f;
  s->regularization = 1e-6f;
  s->rotation_epsilon = 1e-7f;
  s->max_step = 0.1f;
  s->residual_tolerance = 1e-3f;
  s->normalized_update_tolerance = 1e-3f;
  s->contact_tangential_damping = 8.f;
  s->contact_margin = 0.01f;
  s->ipc_activation_distance = 0.05f;
  s->ipc_minimum_distance = 0.001f;
  s->ipc_barrier_stiffness = 0.f;
  s->ipc_friction_coefficient = 0.f;
  s->ipc_friction_velocity_epsilon = 0.01f;
  s->ipc_step_safety = 0.9f;
  s->horizontal_body_correction = 1;
  s->parity_mode = 0;
}

void merge(jgs2_settings* out, const jgs2_settings* o, uint32_t m) {
  if (!o) return;
  if (m & JGS2_SET_SCHEDULE) out->schedule = o->schedule;
  if (m & JGS2_SET_ITERATIONS) out->iterations = o->iterations;
  if (m & JGS2_SET_TIMESTEP) out->timestep = o->timestep;
  if (m & JGS2_SET_GRAVITY) std::memcpy(out->gravity, o->gravity, sizeof(out->gravity));
  if (m & JGS2_SET_FLOOR_HEIGHT) out->floor_height = o->floor_height;
  if (m & JGS2_SET_FLOOR_STIFFNESS) out->floor_stiffness = o->floor_stiffness;
  if (m & JGS2_SET_VELOCITY_DAMPING) out->velocity_damping = o->velocity_damping;
  if (m & JGS2_SET_REGULARIZATION) out->regularization = o->regularization;
  if (m & JGS2_SET_ROTATION_EPSILON) out->rotation_epsilon = o->rotation_epsilon;
  if (m & JGS2_SET_MAX_STEP) out->max_step = o->max_step;
  if (m & JGS2_SET_RESIDUAL_TOLERANCE) out->residual_tolerance = o->residual_tolerance;
  if (m & JGS2_SET_NORMALIZED_UPDATE_TOLERANCE) out->normalized_update_tolerance = o->normalized_update_tolerance;
  if (m & JGS2_SET_CONTACT_TANGENTIAL_DAMPING) out->contact_tangential_damping = o->contact_tangential_damping;
  if (m & JGS2_SET_CONTACT_MARGIN) out->contact_margin = o->contact_margin;
  if (m & JGS2_SET_IPC_ACTIVATION_DISTANCE) out->ipc_activation_distance = o->ipc_activation_distance;
  if (m & JGS2_SET_IPC_MINIMUM_DISTANCE) out->ipc_minimum_distance = o->ipc_minimum_distance;
  if (m & JGS2_SET_IPC_BARRIER_STIFFNESS) out->ipc_barrier_stiffness = o->ipc_barrier_stiffness;
  if (m & JGS2_SET_IPC_FRICTION_COEFFICIENT) out->ipc_friction_coefficient = o->ipc_friction_coefficient;
  if (m & JGS2_SET_IPC_FRICTION_VELOCITY_EPSILON)
    out->ipc_friction_velocity_epsilon = o->ipc_friction_velocity_epsilon;
  if (m & JGS2_SET_IPC_STEP_SAFETY) out->ipc_step_safety = o->ipc_step_safety;
  if (m & JGS2_SET_HORIZONTAL_BODY_CORRECTION) out->horizontal_body_correction = o->horizontal_body_correction;
  if (m & JGS2_SET_PARITY_MODE) out->parity_mode = o->parity_mode;
}

bool finite(float v) { return std::isfinite(v); }

// validateStepSettings (src/simulation/gpu/jgs2-solver.ts:429-529).
bool validateSettings(const jgs2_settings& s, std::string* err) {
  if (s.schedule != JGS2_SCHEDULE_JACOBI && s.schedule != JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL) {
    *err = format("Unknown JGS2 schedule: %u.", s.schedule);
    return false;
  }
  const std::pair<const char*, float> values[] = {
      {"timestep", s.timestep}, {"floorHeight", s.floor_height}, {"floorStiffness", s.floor_stiffness},
      {"velocityDamping", s.velocity_damping}, {"regularization", s.regularization},
      {"rotationEpsilon", s.rotation_epsilon}, {"maxStep", s.max_step},
      {"residualTolerance", s.residual_tolerance}, {"normalizedUpdateTolerance", s.normalized_update_tolerance},
      {"contactTangentialDamping", s.contact_tangential_damping}, {"contactMargin", s.contact_margin},
      {"ipcActivationDistance", s.ipc_activation_distance}, {"ipcMinimumDistance", s.ipc_minimum_distance},
      {"ipcBarrierStiffness", s.ipc_barrier_stiffness}, {"ipcFrictionCoefficient", s.ipc_friction_coefficient},
      {"ipcFrictionVelocityEpsilon", s.ipc_friction_velocity_epsilon}, {"ipcStepSafety", s.ipc_step_safety},
      {"gravity.x", s.gravity[0]}, {"gravity.y", s.gravity[1]}, {"gravity.z", s.gravity[2]}};
  for (const auto& kv : values)
    if (!finite(kv.second)) { *err = format("%s must be finite; got %g.", kv.first, kv.second); return false; }
  if (!(s.timestep > 0)) { *err = "timestep must be positive."; return false; }
  if (s.floor_stiffness < 0) { *err = "floorStiffness must be nonnegative."; return false; }
  if (s.velocity_damping < 0 || s.velocity_damping > 1) { *err = "velocityDamping must be between zero and one."; return false; }
  if (!(s.regularization > 0)) { *err = "regularization must be positive."; return false; }
  if (!(s.rotation_epsilon > 0)) { *err = "rotationEpsilon must be positive."; return false; }
  if (s.max_step < 0) { *err = "maxStep must be nonnegative."; return false; }
  if (!(s.residual_tolerance > 0) || s.residual_tolerance > kMaxRuntimeTolerance) {
    *err = format("residualTolerance must be positive and no greater than %g.", kMaxRuntimeTolerance);
    return false;
  }
  if (!(s.normalized_update_tolerance > 0) || s.normalized_update_tolerance > kMaxRuntimeTolerance) {
    *err = format("normalizedUpdateTolerance must be positive and no greater than %g.", kMaxRuntimeTolerance);
    return false;
  }
  if (s.contact_tangential_damping < 0) { *err = "contactTangentialDamping must be finite and nonnegative."; return false; }
  if (s.contact_margin < 0) { *err = "contactMargin must be finite and nonnegative."; return false; }
  if (!(s.ipc_activation_distance > 0)) { *err = "ipcActivationDistance must be positive."; return false; }
  if (s.ipc_minimum_distance < 0 || s.ipc_minimum_distance >= s.ipc_activation_distance) {
    *err = "ipcMinimumDistance must be nonnegative and below ipcActivationDistance.";
    return false;
  }
  if (s.ipc_barrier_stiffness < 0) { *err = "ipcBarrierStiffness must be nonnegative."; return false; }
  if (s.ipc_friction_coefficient < 0) { *err = "ipcFrictionCoefficient must be nonnegative."; return false; }
  if (!(s.ipc_friction_velocity_epsilon > 0)) { *err = "ipcFrictionVelocityEpsilon must be positive."; return false; }
  if (!(s.ipc_step_safety > 0) || !(s.ipc_step_safety < 1)) {
    *err = "ipcStepSafety must be strictly between zero and one.";
    return false;
  }
  if (s.horizontal_body_correction > 1) { *err = "horizontalBodyCorrection must be a boolean."; return false; }
  if (s.parity_mode > 1) { *err = "parityMode must be a boolean."; return false; }
  return true;
}

// resolveJGS2StepSettings (src/simulation/gpu/jgs2-solver.ts:531-550).
bool resolve(const jgs2_settings& base, const jgs2_settings* o, uint32_t mask, jgs2_settings* out,
             std::string* err) {
  *out = base;
  merge(out, o, mask);
  if (out->parity_mode) {
    out->velocity_damping = 1.f;
    out->contact_tangential_damping = 0.f;
    out->horizontal_body_correction = 0;
  }
  return validateSettings(*out, err);
}

// ---- input validation (src/simulation/gpu/layout.ts:223-416) ---------------

bool validateInput(const jgs2_input* in, std::string* err) {
  if (!in) { *err = "input is NULL."; return false; }
  const uint32_t V = in->vertex_count, T = in->tet_count, K = in->cubature_k;
  if (V < 1) { *err = format("vertexCount must be an integer >= 1; got %u.", V); return false; }
  if (T < 1) { *err = format("tetCount must be an integer >= 1; got %u.", T); return false; }
  if (!in->positions || !in->vertex_rest || !in->vertex_info || !in->tet_indices || !in->tet_inverse_dm ||
      !in->tet_meta || !in->adjacency || (K > 0 && (!in->cubature_tet_ids || !in->cubature_weights ||
                                                    !in->cubature_basis))) {
    *err = "A required input array is NULL.";
    return false;
  }
  if (V >= (1u << 30) || T >= (1u << 30)) { *err = "vertexCount and tetCount must be below 2^30."; return false; }
  if ((in->target_positions == nullptr) != (in->target_stiffnesses == nullptr)) {
    *err = "objectives.targetPositions and objectives.targetStiffnesses must be provided together.";
    return false;
  }
  auto finiteArray = [&](const float* a, size_t n, const char* name) {
    if (!a) return true;
    for (size_t i = 0; i < n; ++i)
      if (!std::isfinite(a[i])) { *err = format("%s[%zu] must be finite.", name, i); return false; }
    return true;
  };
  if (!finiteArray(in->positions, 4ull * V, "positions") || !finiteArray(in->velocities, 4ull * V, "velocities") ||
      !finiteArray(in->vertex_rest, 4ull * V, "vertexRest") ||
      !finiteArray(in->vertex_colors, 4ull * V, "vertexColors") ||
      !finiteArray(in->external_forces, 3ull * V, "objectives.externalForces") ||
      !finiteArray(in->target_positions, 3ull * V, "objectives.targetPositions") ||
      !finiteArray(in->target_stiffnesses, V, "objectives.targetStiffnesses") ||
      !finiteArray(in->tet_inverse_dm, 12ull * T, "tetInverseDm") || !finiteArray(in->tet_meta, 4ull * T, "tetMeta") ||
      !finiteArray(in->tet_rest_stiffness, 144ull * T, "tetRestStiffness") ||
      !finiteArray(in->cubature_weights, static_cast<size_t>(V) * K, "cubatureWeights") ||
      !finiteArray(in->cubature_basis, static_cast<size_t>(V) * K * 36, "cubatureBasis"))
    return false;
  if (in->target_stiffnesses)
    for (uint32_t v = 0; v < V; ++v)
      if (in->target_stiffnesses[v] < 0) {
        *err = format("objectives.targetStiffnesses[%u] must be nonnegative.", v);
        return false;
      }
  for (uint32_t v = 0; v < V; ++v) {
    if (in->vertex_info[4ull * v + 2] == 0) continue;
    const bool force = in->external_forces && (in->external_forces[3ull * v] != 0 ||
                                               in->external_forces[3ull * v + 1] != 0 ||
                                               in->external_forces[3ull * v + 2] != 0);
    const bool target = in->target_stiffnesses && in->target_stiffnesses[v] != 0;
    if (force || target) {
      *err = format("Pinned vertex %u cannot have a nonzero external force or quadratic-target stiffness.", v);
      return false;
    }
  }
  uint32_t maxBody = 0;
  for (uint32_t v = 0; v < V; ++v) maxBody = std::max(maxBody, in->vertex_info[4ull * v + 3]);
  if (static_cast<uint64_t>(maxBody) + 1 > V) {
    *err = format("vertexInfo body ids must be compact nonnegative values whose maximum is smaller than "
                  "vertexCount (%u); got %u.", V, maxBody);
    return false;
  }
  for (size_t i = 0; i < 4ull * T; ++i)
    if (in->tet_indices[i] >= V) {
      *err = format("tetIndices[%zu] references vertex %u, but vertexCount is %u.", i, in->tet_indices[i], V);
      return false;
    }
  bool anyCorotated = false;
  for (uint32_t t = 0; t < T; ++t) {
    const float vol = in->tet_meta[4ull * t], lambda = in->tet_meta[4ull * t + 1], mu = in->tet_meta[4ull * t + 2];
    const float model = in->tet_meta[4ull * t + 3];
    if (!(vol > 0) || !(mu > 0)) {
      *err = format("tetMeta for tetrahedron %u requires positive volume and mu.", t);
      return false;
    }
    if (model != 0.0f && model != 1.0f) {
      *err = format("tetMeta for tetrahedron %u has unknown material model %g.", t, model);
      return false;
    }
    if (model == 1.0f && !(lambda > 0)) {
      *err = format("Stable Neo-Hookean tetMeta for tetrahedron %u requires positive lambda.", t);
      return false;
    }
    if (model == 0.0f) {
      anyCorotated = true;
      if (!(3 * lambda + 2 * mu > 0)) {
        *err = format("Co-rotated tetMeta for tetrahedron %u requires positive bulk modulus.", t);
        return false;
      }
    }
  }
  if (anyCorotated && !in->tet_rest_stiffness) {
    *err = "tetRestStiffness is required when any tetrahedron is co-rotated.";
    return false;
  }
  for (uint64_t i = 0; i < in->adjacency_length; ++i)
    if (in->adjacency[i] >= T) {
      *err = format("adjacency[%llu] references tetrahedron %u, but tetCount is %u.",
                    static_cast<unsigned long long>(i), in->adjacency[i], T);
      return false;
    }
  // Canonical CSR of unique incident tets (layout.ts:359-398).
  std::vector<uint32_t> counts(V, 0), last(V, kEmptyTet);
  for (uint32_t t = 0; t < T; ++t)
    for (int l = 0; l < 4; ++l) {
      const uint32_t v = in->tet_indices[4ull * t + l];
      if (last[v] != t) { counts[v]++; last[v] = t; }
    }
  uint64_t offset = 0;
  std::vector<uint64_t> starts(V);
  for (uint32_t v = 0; v < V; ++v) {
    const uint32_t start = in->vertex_info[4ull * v], count = in->vertex_info[4ull * v + 1];
    if (static_cast<uint64_t>(start) + count > in->adjacency_length) {
      *err = format("vertexInfo for vertex %u addresses adjacency range [%u, %llu), beyond %llu.", v, start,
                    static_cast<unsigned long long>(start) + count,
                    static_cast<unsigned long long>(in->adjacency_length));
      return false;
    }
    if (start != offset) {
      *err = format("vertexInfo for vertex %u must start at canonical adjacency offset %llu; got %u.", v,
                    static_cast<unsigned long long>(offset), start);
      return false;
    }
    if (count != counts[v]) {
      *err = format("vertexInfo for vertex %u must list exactly %u unique incident tetrahedra; got %u.", v,
                    counts[v], count);
      return false;
    }
    starts[v] = offset;
    offset += count;
    const float mass = in->vertex_rest[4ull * v + 3];
    if (in->vertex_info[4ull * v + 2] == 0 && !(mass > 0)) {
      *err = format("Unpinned vertex %u must have positive mass.", v);
      return false;
    }
  }
  if (offset != in->adjacency_length) {
    const unsigned long long unused = in->adjacency_length - offset;
    *err = format("adjacency contains %llu unused entr%s.", unused, unused == 1 ? "y" : "ies");
    return false;
  }
  {
    std::vector<uint64_t> cursor(starts);
    std::fill(last.begin(), last.end(), kEmptyTet);
    for (uint32_t t = 0; t < T; ++t)
      for (int l = 0; l < 4; ++l) {
        const uint32_t v = in->tet_indices[4ull * t + l];
        if (last[v] == t) continue;
        last[v] = t;
        const uint64_t at = cursor[v]++;
        if (in->adjacency[at] != t) {
          *err = format("adjacency[%llu] for vertex %u must equal incident tetrahedron %u; got %u.",
                        static_cast<unsigned long long>(at), v, t, in->adjacency[at]);
          return false;
        }
      }
  }
  const size_t R = static_cast<size_t>(V) * K;
  for (size_t r = 0; r < R; ++r) {
    const float w = in->cubature_weights[r];
    const uint32_t t = in->cubature_tet_ids[r];
    if (w < 0) { *err = format("cubatureWeights[%zu] must be nonnegative.", r); return false; }
    if (w > 0 && t >= T) {
      *err = format("Positive cubature record %zu references tetrahedron %u, but tetCount is %u.", r, t, T);
      return false;
    }
  }
  if (in->cloth) {
    // validateJGS2GpuClothInput (cloth-layout.ts:225-332) and the vertex
    // count agreement of validateJGS2GpuInput (layout.ts:247-253).
    const jgs2_cloth_input& c = *in->cloth;
    if (c.vertex_count != V) {
      *err = format("Cloth vertexCount %u must equal solver vertexCount %u.", c.vertex_count, V);
      return false;
    }
    const uint32_t C = c.triangle_count, H = c.hinge_count;
    if ((C > 0 && (!c.triangle_indices || !c.triangle_inverse_rest_bases || !c.triangle_rest_areas)) ||
        (H > 0 && (!c.hinge_indices || !c.hinge_rest_angles || !c.hinge_rest_edge_lengths))) {
      *err = "A required cloth array is NULL.";
      return false;
    }
    if (C >= (1u << 29) || H >= (1u << 29)) { *err = "Cloth element counts must be below 2^29."; return false; }
    auto distinct = [&](const uint32_t* q, int n, const char* label, uint32_t e) {
      for (int a = 0; a < n; ++a) {
        if (q[a] >= V) {
          *err = format("%s %u index %u is outside vertexCount %u.", label, e, q[a], V);
          return false;
        }
        for (int b = 0; b < a; ++b)
          if (q[a] == q[b]) {
            *err = format("%s %u must reference %d distinct vertices.", label, e, n);
            return false;
          }
      }
      return true;
    };
    for (uint32_t t = 0; t < C; ++t)
      if (!distinct(&c.triangle_indices[3ull * t], 3, "Triangle", t)) return false;
    for (uint32_t h = 0; h < H; ++h)
      if (!distinct(&c.hinge_indices[4ull * h], 4, "Hinge", h)) return false;
    if (!finiteArray(c.triangle_inverse_rest_bases, 4ull * C, "triangleInverseRestBases") ||
        !finiteArray(c.triangle_rest_areas, C, "triangleRestAreas") ||
        !finiteArray(c.hinge_rest_angles, H, "hingeRestAngles") ||
        !finiteArray(c.hinge_rest_edge_lengths, H, "hingeRestEdgeLengths"))
      return false;
    for (uint32_t t = 0; t < C; ++t) {
      if (!(c.triangle_rest_areas[t] > 0)) { *err = format("triangleRestAreas[%u] must be positive.", t); return false; }
      const float* b = &c.triangle_inverse_rest_bases[4ull * t];
      const float d = b[0] * b[3] - b[1] * b[2];
      if (d == 0 || !std::isfinite(d)) {
        *err = format("triangleInverseRestBases for triangle %u must be invertible.", t);
        return false;
      }
    }
    for (uint32_t h = 0; h < H; ++h)
      if (!(c.hinge_rest_edge_lengths[h] > 0)) {
        *err = format("hingeRestEdgeLengths[%u] must be positive.", h);
        return false;
      }
    if (!(c.young_modulus > 0) || !std::isfinite(c.young_modulus)) {
      *err = "Cloth Young's modulus must be finite and positive.";
      return false;
    }
    if (!(c.poisson_ratio >= 0 && c.poisson_ratio < 0.5f)) {
      *err = "Cloth Poisson ratio must be finite and in [0, 0.5).";
      return false;
    }
    if (!(c.thickness > 0) || !std::isfinite(c.thickness)) {
      *err = "Cloth thickness must be finite and positive.";
      return false;
    }
    if (!(c.bending_stiffness >= 0) || !std::isfinite(c.bending_stiffness)) {
      *err = "Cloth bending stiffness must be finite and nonnegative.";
      return false;
    }
  }
  // validateIpcContactCandidatesForGpu (ipc-contact-layout.ts:119-176).
  const uint64_t nc = uint64_t(in->contact_vertex_triangle_count) + in->contact_edge_edge_count;
  if (nc > 0 && !in->contact_indices) {
    *err = "IPC contact candidate indices are NULL.";
    return false;
  }
  if (nc >= (1ull << 29)) {
    *err = "Total IPC candidate count must be below 2^29.";
    return false;
  }
  if (const jgs2_contact_surface* cs = in->contact_surface) {
    if (nc > 0) {
      *err = "Give either static IPC candidates or a contact surface, not both.";
      return false;
    }
    if (cs->triangle_count > 0 && !cs->triangles) {
      *err = "Contact surface triangles are NULL.";
      return false;
    }
    if (cs->candidate_capacity >= (1ull << 28)) {
      *err = "The contact candidate capacity must be below 2^28.";
      return false;
    }
    for (uint64_t t = 0; t < cs->triangle_count; ++t) {
      const uint32_t* q = &cs->triangles[3 * t];
      if (q[0] >= V || q[1] >= V || q[2] >= V) {
        *err = format("Contact surface triangle %llu references a vertex outside vertexCount %u.",
                      static_cast<unsigned long long>(t), V);
        return false;
      }
      if (q[0] == q[1] || q[1] == q[2] || q[0] == q[2]) {
        *err = format("Contact surface triangle %llu must reference three distinct vertices.",
                      static_cast<unsigned long long>(t));
        return false;
      }
    }
  }
  for (uint64_t c = 0; c < nc; ++c) {
    const uint32_t* q = &in->contact_indices[4 * c];
    const char* type = c < in->contact_vertex_triangle_count ? "VT" : "EE";
    for (int a = 0; a < 4; ++a) {
      if (q[a] >= V) {
        *err = format("IPC candidate references vertex %u, but vertexCount is %u.", q[a], V);
        return false;
      }
      for (int b = 0; b < a; ++b)
        if (q[a] == q[b]) {
          *err = format("%s candidate %llu must reference four distinct vertices.", type,
                        static_cast<unsigned long long>(c));
          return false;
        }
    }
  }
  return true;
}

// evaluateIpcVertexTriangleDistance / evaluateIpcEdgeEdgeDistance
// (src/simulation/cpu/ipc-contact.ts:192-385) in double on the f32 input
// positions: candidate q (vertex-triangle when vt, else edge-edge).
double candidateDistance(const jgs2_input* in, const uint32_t* q, bool vt) {
  struct P { double x, y, z; };
  auto at = [&](uint32_t v) {
    return P{in->positions[4ull * v], in->positions[4ull * v + 1], in->positions[4ull * v + 2]};
  };
  auto sub = [](P a, P b) { return P{a.x - b.x, a.y - b.y, a.z - b.z}; };
  auto dot = [](P a, P b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
  auto cross = [](P a, P b) { return P{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
  auto clamp01 = [](double v) { return !(v > 0) ? 0.0 : (v >= 1 ? 1.0 : v); };
  auto dist = [](P a, P b) {
    const double d = std::hypot(a.x - b.x, a.y - b.y, a.z - b.z);
    return std::isfinite(d) ? d : std::numeric_limits<double>::max();
  };
  auto lerp = [](P s, P e, double t) { return P{s.x + t * (e.x - s.x), s.y + t * (e.y - s.y), s.z + t * (e.z - s.z)}; };
  auto segment = [&](P q, P s, P e, double* t) {
    const P edge = sub(e, s);
    const double l2 = dot(edge, edge);
    *t = 0;
    if (std::isfinite(l2) && l2 > 1e-20) *t = clamp01(dot(sub(q, s), edge) / l2);
    return dist(q, lerp(s, e, *t));
  };
  {
    const P p0 = at(q[0]), p1 = at(q[1]), p2 = at(q[2]), p3 = at(q[3]);
    double d;
    if (vt) {
      const P e01 = sub(p2, p1), e02 = sub(p3, p1), e12 = sub(p3, p2);
      const double s01 = dot(e01, e01), s02 = dot(e02, e02), s12 = dot(e12, e12);
      const double largest = std::max(s01, std::max(s02, s12));
      const P an = cross(e01, e02);
      const double a2 = dot(an, an);
      const double threshold = std::max(1e-40, 1e-6 * largest * largest);
      d = -1;
      if (std::isfinite(a2) && a2 > threshold) {
        const double d01 = dot(e01, e02);
        const P po = sub(p0, p1);
        const double d20 = dot(po, e01), d21 = dot(po, e02);
        const double den = s01 * s02 - d01 * d01;
        const double b1 = (s02 * d20 - d01 * d21) / den, b2 = (s01 * d21 - d01 * d20) / den;
        const double b0 = 1 - b1 - b2;
        if (std::isfinite(b0) && std::isfinite(b1) && std::isfinite(b2) && b0 >= 0 && b1 >= 0 && b2 >= 0) {
          const P cp{b0 * p1.x + b1 * p2.x + b2 * p3.x, b0 * p1.y + b1 * p2.y + b2 * p3.y,
                     b0 * p1.z + b1 * p2.z + b2 * p3.z};
          if (std::isfinite(cp.x) && std::isfinite(cp.y) && std::isfinite(cp.z)) d = dist(p0, cp);
        }
      }
      if (d < 0) {
        double t;
        d = segment(p0, p1, p2, &t);
        d = std::min(d, segment(p0, p2, p3, &t));
        d = std::min(d, segment(p0, p3, p1, &t));
      }
    } else {
      const P da = sub(p1, p0), db = sub(p3, p2), off = sub(p0, p2);
      const double la = dot(da, da), lb = dot(db, db);
      const double degenerate = std::max(1e-20, 1e-6 * std::max(la, lb));
      const bool aDeg = !(la > degenerate), bDeg = !(lb > degenerate);
      double pa = 0, pb = 0;
      if (aDeg && !bDeg) {
        pb = clamp01(dot(db, off) / lb);
      } else if (!aDeg) {
        const double projA = dot(da, off);
        if (bDeg) {
          pa = clamp01(-projA / la);
        } else {
          const double coupling = dot(da, db), projB = dot(db, off);
          const double den = la * lb - coupling * coupling;
          if (den > 1e-6 * la * lb) pa = clamp01((coupling * projB - projA * lb) / den);
          const double pbu = (coupling * pa + projB) / lb;
          if (pbu < 0) { pb = 0; pa = clamp01(-projA / la); }
          else if (pbu > 1) { pb = 1; pa = clamp01((coupling - projA) / la); }
          else pb = clamp01(pbu);
        }
      }
      d = dist(lerp(p0, p1, pa), lerp(p2, p3, pb));
    }
    return d;
  }
}

// minimumStaticIpcContactDistance (src/simulation/cpu/ipc-contact.ts:385).
double staticContactDistance(const jgs2_input* in) {
  double minimum = std::numeric_limits<double>::max();
  const uint64_t nvt = in->contact_vertex_triangle_count;
  const uint64_t nc = nvt + in->contact_edge_edge_count;
  for (uint64_t c = 0; c < nc; ++c) minimum = std::min(minimum, candidateDistance(in, &in->contact_indices[4 * c], c < nvt));
  return minimum;
}

// A contact surface for the device broad phase: canonical triangles (sorted
// vertices, sorted, unique), their edges (sorted, unique) and each vertex's
// surface one-ring (sorted), the order and exclusions of the static superset
// (buildStaticIpcContactCandidates, src/simulation/cpu/ipc-contact.ts:591-665).
struct ContactSurface {
  std::vector<std::array<uint32_t, 3>> tris;
  std::vector<std::array<uint32_t, 2>> edges;
  std::vector<uint32_t> ringStart;  // V + 1
  std::vector<uint32_t> ring;
  uint64_t capacity = 0;            // candidates one iteration may list
  uint64_t superset = 0;            // candidates of the static superset
};

void buildContactSurface(const jgs2_input* in, ContactSurface* out) {
  const jgs2_contact_surface* cs = in->contact_surface;
  out->tris.resize(cs->triangle_count);
  for (uint32_t t = 0; t < cs->triangle_count; ++t) {
    std::array<uint32_t, 3> a = {cs->triangles[3ull * t], cs->triangles[3ull * t + 1], cs->triangles[3ull * t + 2]};
    std::sort(a.begin(), a.end());
    out->tris[t] = a;
  }
  std::sort(out->tris.begin(), out->tris.end());
  out->tris.erase(std::unique(out->tris.begin(), out->tris.end()), out->tris.end());
  for (const auto& t : out->tris) {
    out->edges.push_back({t[0], t[1]});
    out->edges.push_back({t[1], t[2]});
    out->edges.push_back({t[0], t[2]});
  }
  std::sort(out->edges.begin(), out->edges.end());
  out->edges.erase(std::unique(out->edges.begin(), out->edges.end()), out->edges.end());
  const uint32_t V = in->vertex_count;
  out->ringStart.assign(V + 1, 0);
  for (const auto& e : out->edges) {
    out->ringStart[e[0] + 1]++;
    out->ringStart[e[1] + 1]++;
  }
  for (uint32_t v = 0; v < V; ++v) out->ringStart[v + 1] += out->ringStart[v];
  out->ring.resize(out->ringStart[V]);
  std::vector<uint32_t> cursor(out->ringStart.begin(), out->ringStart.end() - 1);
  for (const auto& e : out->edges) {
    out->ring[cursor[e[0]]++] = e[1];
    out->ring[cursor[e[1]]++] = e[0];
  }
  for (uint32_t v = 0; v < V; ++v) std::sort(out->ring.begin() + out->ringStart[v], out->ring.begin() + out->ringStart[v + 1]);
  out->capacity = cs->candidate_capacity
                      ? cs->candidate_capacity
                      : 65536 + 16ull * (uint64_t(V) + out->edges.size());
  // Size of the superset: per vertex the triangles outside its closed
  // one-ring, per edge pair those whose endpoints avoid each other's closed
  // one-rings.
  const size_t nT = out->tris.size(), nE = out->edges.size();
  std::vector<std::vector<uint32_t>> vTris(V), vEdges(V);
  for (uint32_t t = 0; t < nT; ++t)
    for (uint32_t v : out->tris[t]) vTris[v].push_back(t);
  for (uint32_t e = 0; e < nE; ++e)
    for (uint32_t v : out->edges[e]) vEdges[v].push_back(e);
  std::vector<uint32_t> stamp(std::max(nT, nE), 0xffffffffu);
  uint64_t vt = 0, closedEdges = 0;
  auto closedSet = [&](uint32_t v, auto&& visit) {
    visit(v);
    for (uint32_t i = out->ringStart[v]; i < out->ringStart[v + 1]; ++i) visit(out->ring[i]);
  };
  for (uint32_t v = 0; v < V; ++v) {
    uint64_t touching = 0;
    closedSet(v, [&](uint32_t u) {
      for (uint32_t t : vTris[u])
        if (stamp[t] != v) { stamp[t] = v; ++touching; }
    });
    vt += nT - touching;
  }
  std::fill(stamp.begin(), stamp.end(), 0xffffffffu);
  for (uint32_t e = 0; e < nE; ++e) {
    auto visit = [&](uint32_t u) {
      for (uint32_t f : vEdges[u])
        if (f != e && stamp[f] != e) { stamp[f] = e; ++closedEdges; }
    };
    closedSet(out->edges[e][0], visit);
    closedSet(out->edges[e][1], visit);
  }
  out->superset = vt + (uint64_t(nE) * (nE - (nE ? 1 : 0)) / 2 - closedEdges / 2);
}

// The smallest distance over the superset's candidates whose boxes come
// within `cutoff` (a hashed grid over the primitive boxes); +infinity when
// no candidate does.  Pairs farther apart cannot decide the create-time
// feasibility check.
double surfaceContactDistance(const jgs2_input* in, const ContactSurface& cs, double cutoff) {
  struct Box { double lo[3], hi[3]; };
  const float* x = in->positions;
  auto boxOf = [&](const uint32_t* v, int n) {
    Box b;
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = b.hi[k] = x[4ull * v[0] + k];
      for (int l = 1; l < n; ++l) {
        b.lo[k] = std::min(b.lo[k], double(x[4ull * v[l] + k]));
        b.hi[k] = std::max(b.hi[k], double(x[4ull * v[l] + k]));
      }
    }
    return b;
  };
  const size_t nT = cs.tris.size(), nE = cs.edges.size();
  std::vector<Box> tb(nT), eb(nE);
  double extent = 0;
  for (size_t t = 0; t < nT; ++t) {
    tb[t] = boxOf(cs.tris[t].data(), 3);
    for (int k = 0; k < 3; ++k) extent = std::max(extent, tb[t].hi[k] - tb[t].lo[k]);
  }
  for (size_t e = 0; e < nE; ++e) eb[e] = boxOf(cs.edges[e].data(), 2);
  for (int k = 0; k < 3; ++k)
    for (size_t t = 0; t < nT; ++t)
      if (!std::isfinite(tb[t].lo[k]) || !std::isfinite(tb[t].hi[k])) return -1.0;  // non-finite pose
  const double cell = std::max(cutoff, extent / 4 + cutoff);
  auto key = [](int64_t i, int64_t j, int64_t k) {
    return (uint64_t(i & 0x1fffff) << 42) | (uint64_t(j & 0x1fffff) << 21) | uint64_t(k & 0x1fffff);
  };
  auto cellOf = [&](double v) { return static_cast<int64_t>(std::floor(v / cell)); };
  auto closed = [&](uint32_t a, uint32_t b) {
    return a == b || std::binary_search(cs.ring.begin() + cs.ringStart[a], cs.ring.begin() + cs.ringStart[a + 1], b);
  };
  auto gridOf = [&](const std::vector<Box>& boxes) {
    std::unordered_map<uint64_t, std::vector<uint32_t>> g;
    for (size_t i = 0; i < boxes.size(); ++i) {
      const Box& b = boxes[i];
      for (int64_t a = cellOf(b.lo[0] - cutoff); a <= cellOf(b.hi[0] + cutoff); ++a)
        for (int64_t c = cellOf(b.lo[1] - cutoff); c <= cellOf(b.hi[1] + cutoff); ++c)
          for (int64_t d = cellOf(b.lo[2] - cutoff); d <= cellOf(b.hi[2] + cutoff); ++d)
            g[key(a, c, d)].push_back(static_cast<uint32_t>(i));
    }
    return g;
  };
  auto gap = [](const Box& a, const Box& b) {
    double s = 0;
    for (int k = 0; k < 3; ++k) {
      const double g = std::max(0.0, std::max(b.lo[k] - a.hi[k], a.lo[k] - b.hi[k]));
      s += g * g;
    }
    return std::sqrt(s);
  };
  double minimum = INFINITY;
  {
    const auto g = gridOf(tb);
    for (uint32_t v = 0; v < in->vertex_count; ++v) {
      const uint32_t vv[1] = {v};
      const Box p = boxOf(vv, 1);
      auto it = g.find(key(cellOf(p.lo[0]), cellOf(p.lo[1]), cellOf(p.lo[2])));
      if (it == g.end()) continue;
      for (uint32_t t : it->second) {
        const auto& tri = cs.tris[t];
        if (closed(v, tri[0]) || closed(v, tri[1]) || closed(v, tri[2]) || gap(p, tb[t]) > cutoff) continue;
        const uint32_t q[4] = {v, tri[0], tri[1], tri[2]};
        minimum = std::min(minimum, candidateDistance(in, q, true));
      }
    }
  }
  {
    const auto g = gridOf(eb);
    std::vector<uint32_t> stamp(nE, 0xffffffffu);
    for (uint32_t i = 0; i < nE; ++i) {
      const Box& b = eb[i];
      for (int64_t a = cellOf(b.lo[0]); a <= cellOf(b.hi[0]); ++a)
        for (int64_t c = cellOf(b.lo[1]); c <= cellOf(b.hi[1]); ++c)
          for (int64_t d = cellOf(b.lo[2]); d <= cellOf(b.hi[2]); ++d) {
            auto it = g.find(key(a, c, d));
            if (it == g.end()) continue;
            for (uint32_t j : it->second) {
              if (j <= i || stamp[j] == i) continue;
              stamp[j] = i;
              const auto& ea = cs.edges[i];
              const auto& eb2 = cs.edges[j];
              if (closed(ea[0], eb2[0]) || closed(ea[0], eb2[1]) || closed(ea[1], eb2[0]) || closed(ea[1], eb2[1]) ||
                  gap(b, eb[j]) > cutoff)
                continue;
              const uint32_t q[4] = {ea[0], ea[1], eb2[0], eb2[1]};
              minimum = std::min(minimum, candidateDistance(in, q, false));
            }
          }
    }
  }
  return minimum;
}

// buildJGS2InputVertexColoring + buildGreedyVertexColoring.
std::vector<uint32_t> colorInput(const jgs2_input* in, uint32_t* count) {
  const uint32_t V = in->vertex_count;
  // Conflict adjacency as CSR built from the groups in the reference order.
  std::vector<std::vector<uint32_t>> adj(V);
  auto group = [&](const uint32_t* g, int n) {
    uint32_t u[8];
    int m = 0;
    for (int i = 0; i < n; ++i) {
      bool seen = false;
      for (int j = 0; j < m; ++j) seen |= u[j] == g[i];
      if (!seen) u[m++] = g[i];
    }
    for (int a = 0; a < m; ++a)
      for (int b = a + 1; b < m; ++b) {
        adj[u[a]].push_back(u[b]);
        adj[u[b]].push_back(u[a]);
      }
  };
  for (uint32_t t = 0; t < in->tet_count; ++t) group(&in->tet_indices[4ull * t], 4);
  for (uint32_t v = 0; v < V; ++v)
    for (uint32_t s = 0; s < in->cubature_k; ++s) {
      const size_t r = static_cast<size_t>(v) * in->cubature_k + s;
      const uint32_t t = in->cubature_tet_ids[r];
      if (t == kEmptyTet || !(in->cubature_weights[r] > 0)) continue;
      const uint32_t g[5] = {v, in->tet_indices[4ull * t], in->tet_indices[4ull * t + 1],
                             in->tet_indices[4ull * t + 2], in->tet_indices[4ull * t + 3]};
      group(g, 5);
    }
  if (in->cloth) {
    for (uint32_t c = 0; c < in->cloth->triangle_count; ++c) group(&in->cloth->triangle_indices[3ull * c], 3);
    for (uint32_t h = 0; h < in->cloth->hinge_count; ++h) group(&in->cloth->hinge_indices[4ull * h], 4);
  }
  if (in->contact_indices) {
    const uint64_t nc = uint64_t(in->contact_vertex_triangle_count) + in->contact_edge_edge_count;
    for (uint64_t c = 0; c < nc; ++c) group(&in->contact_indices[4 * c], 4);
  }
  std::vector<uint32_t> colors(V, 0xffffffffu), stamp(V + 1, 0);
  uint32_t n = 0, st = 0;
  for (uint32_t v = 0; v < V; ++v) {
    st += 1;
    for (uint32_t u : adj[v])
      if (colors[u] != 0xffffffffu) stamp[colors[u]] = st;
    uint32_t c = 0;
    while (c < n && stamp[c] == st) c += 1;
    colors[v] = c;
    n = std::max(n, c + 1);
  }
  *count = n;
  return colors;
}

// minimumJGS2InputDeformationDeterminant (src/simulation/gpu/layout.ts:541-583).
double minimumInputDeterminant(const jgs2_input* in) {
  auto det = [](double a0, double a1, double a2, double b0, double b1, double b2, double c0, double c1, double c2) {
    return a0 * (b1 * c2 - b2 * c1) - b0 * (a1 * c2 - a2 * c1) + c0 * (a1 * b2 - a2 * b1);
  };
  double m = INFINITY;
  for (uint32_t t = 0; t < in->tet_count; ++t) {
    const uint32_t* q = &in->tet_indices[4ull * t];
    const float* p = in->positions;
    const double ds = det(p[4 * q[1]] - p[4 * q[0]], p[4 * q[1] + 1] - p[4 * q[0] + 1], p[4 * q[1] + 2] - p[4 * q[0] + 2],
                          p[4 * q[2]] - p[4 * q[0]], p[4 * q[2] + 1] - p[4 * q[0] + 1], p[4 * q[2] + 2] - p[4 * q[0] + 2],
                          p[4 * q[3]] - p[4 * q[0]], p[4 * q[3] + 1] - p[4 * q[0] + 1], p[4 * q[3] + 2] - p[4 * q[0] + 2]);
    const float* d = &in->tet_inverse_dm[12ull * t];
    const double di = det(d[0], d[1], d[2], d[4], d[5], d[6], d[8], d[9], d[10]);
    const double v = ds * di;
    if (!std::isfinite(v)) return v;
    m = std::min(m, v);
  }
  return m;
}

}  // namespace

// ---- engine -------------------------------------------------------------------
//
// One engine steps one or more independent scenes together: their vertex, tet
// and cubature arrays are concatenated in device memory, every kernel looks up
// the scene of the element it works on, and the gate / convergence reductions
// are segmented per scene.  `jgs2_solver` is an engine of one scene (the
// reference's JGS2GpuSolver); `jgs2_batch` is an engine of many.

namespace {

// Host state of one scene.
struct SceneHost {
  uint32_t V = 0, T = 0, K = 0, vOff = 0, tOff = 0, bodyOff = 0, bodies = 1;
  uint32_t C = 0, H = 0, cOff = 0, hOff = 0;  // cloth triangles / hinges and their offsets
  float clothLambda = 0.f, clothMu = 0.f, clothThickness = 0.f, clothBending = 0.f;
  uint32_t KC = 0, kOff = 0;  // IPC candidates and their offset
  // Contact surface (device broad phase): surface triangles and edges, their
  // offsets, the scene's rows and its share of the list capacity.
  bool dynamic = false;
  uint32_t bpTris = 0, bpEdges = 0, bpTriOff = 0, bpEdgeOff = 0, bpRowOff = 0, bpRows = 0;
  uint64_t bpCapacity = 0, bpSuperset = 0;
  // IPC parameters fixed at create (jgs2-solver.ts:1096-1105).
  float ipcMinDistance = 0.f, ipcFriction = 0.f, ipcEpsilon = 0.f, ipcSafety = 0.f;
  float sceneScale = 1.f;
  float preprocessingTimestep = 0.f;
  jgs2_settings defaults{};
  jgs2_settings submitted{};
  uint32_t submittedIterations = 0;
  bool recordsAvailable = false;
  uint32_t colorCount = 1;
  std::vector<uint32_t> colors;  // scene-local colouring
  uint32_t objectiveFlags = 0, forceCount = 0, targetCount = 0, objectiveRevision = 0;
  bool active = true;  // an inactive scene sits every frame out
};

}  // namespace

struct Engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool destroyed = false;
  std::string error;
  uint32_t V = 0, T = 0, K = 0, bodies = 1;  // totals over the scenes; K = widest record count
  uint32_t C = 0, H = 0;                     // cloth triangles and hinges over the scenes
  uint32_t KC = 0;                           // IPC candidates over the scenes
  // Device broad phase: the two candidate lists (current and previous
  // iteration, alternating by iteration) and the sort's buffers.
  bool dynamic = false;
  uint64_t bpCapacity = 0;
  uint4* dynIdx[2] = {nullptr, nullptr};
  uint32_t* dynScene[2] = {nullptr, nullptr};
  float4* dynState[2] = {nullptr, nullptr};
  uint32_t* dynFlag[2] = {nullptr, nullptr};
  uint32_t* dynCols[2] = {nullptr, nullptr};
  uint32_t* dynRowOff[2] = {nullptr, nullptr};
  bool glob = true;
  std::vector<SceneHost> scenes;
  // Colour lists over all scenes: colour c holds every scene's colour-c vertices.
  uint32_t colorCount = 1;
  bool coloringBuilt = true;  // batches colour their scenes only when a scene asks for GGS2
  std::vector<uint32_t> colorOffsets;  // colorCount + 1 into colorVertices
  std::vector<uint32_t> needOffsets;   // colorCount + 1 into needVertices
  // Objectives: pinned host mirrors of the device force and target arrays
  // (force xyz, 0) and (target xyz, stiffness); uploads copy from them.
  float4* hForces = nullptr;
  float4* hTargets = nullptr;
  cudaEvent_t objectiveUpload = nullptr;  // recorded after the last upload
  cudaEvent_t readDone = nullptr;         // recorded after the last asynchronous read
  bool objectiveUploadPending = false;
  std::vector<uint8_t> pinned;
  // device
  Buffers b{};
  DevParams* dParams = nullptr;  // one per scene
  std::vector<DevParams> hParams;
  uint32_t* dColorVertices = nullptr;
  // The coloured sweep as one persistent kernel (JGS2_COLOR_SWEEP=persistent):
  // device copies of the colour and need offsets, its barrier words, and the
  // barrier spin bound (JGS2_BARRIER_SPIN_LIMIT, polls of about 32 ns).  The
  // launch-per-colour encoding is the default: measured on one B200 it was
  // faster at every size tried (cubes of 343 to 1 030 301 vertices).
  uint32_t* dColorOffsets = nullptr;
  uint32_t* dNeedOffsets = nullptr;
  void* dSweepBarrier = nullptr;
  uint32_t spinLimit = 1u << 24;
  bool persistentSweep = false;
  // Fault injection of device allocations (JGS2_FAIL_ALLOCATION); -1 off.
  int64_t failAllocationAt = -1, allocationCount = 0;
  bool sweepLaunched = false;
  uint32_t* dNeedVertices = nullptr;
  std::vector<void*> allocations;
  uint64_t launches = 0;
  // graphs: (iterations, schedule, bodyCorrection, contact, launch shape) ->
  // exec, launches per replay
  std::map<std::tuple<uint32_t, uint32_t, bool, bool, uint32_t>, std::pair<cudaGraphExec_t, int>> graphs;
  // Online launch-shape tuning: frames left to time, the next shape to time,
  // per-shape frame times (ms) and the event pair around a timed frame.
  uint32_t tuneLeft = 0, tuneNext = 0, tuneRounds = 0;
  std::vector<float> tuneMs[JGS2_LAUNCH_SHAPES];
  cudaEvent_t tuneEvents[2] = {nullptr, nullptr};
  // Oracle diagnostics records, allocated at the first request.
  float4* oracleTetRot = nullptr;
  float4* oracleTetMetric = nullptr;
  float4* oracleVertex = nullptr;
  double* oracleSummary = nullptr;
  bool useGraphs = true;
};

struct jgs2_solver : Engine {};
struct jgs2_batch : Engine {};

namespace {

jgs2_status fail(Engine* s, jgs2_status st, const std::string& msg) {
  if (s) s->error = msg;
  else gGlobalError = msg;
  return st;
}

jgs2_status cudaFail(Engine* s, cudaError_t e, const char* what) {
  return fail(s, e == cudaErrorMemoryAllocation ? JGS2_OUT_OF_MEMORY : JGS2_DEVICE_ERROR,
              format("%s: %s", what, cudaGetErrorString(e)));
}

#define CUDA_TRY(s, call)                               \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cudaFail((s), _e, #call); \
  } while (0)

// Runs fn(i) for i in [0, n) on up to hardware-concurrency threads (host-side
// scene preparation and packing; every i writes its own outputs).
template <class F>
void parallelFor(uint32_t n, F&& fn) {
  const uint32_t workers = std::min<uint32_t>(n, std::max(1u, std::thread::hardware_concurrency()));
  if (workers <= 1) {
    for (uint32_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (uint32_t w = 0; w < workers; ++w)
    pool.emplace_back([&] {
      for (uint32_t i = next++; i < n; i = next++) fn(i);
    });
  for (auto& t : pool) t.join();
}

template <class T>
jgs2_status deviceAlloc(Engine* s, T** out, size_t count) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(16, count * sizeof(T));
  // Host-side fault injection (JGS2_FAIL_ALLOCATION=n, read at create): the
  // n-th device allocation of a create fails as an exhausted device would.
  if (s->failAllocationAt >= 0 && s->allocationCount++ == s->failAllocationAt)
    return fail(s, JGS2_OUT_OF_MEMORY,
                format("cudaMalloc: out of memory (injected by JGS2_FAIL_ALLOCATION at allocation %lld)",
                       static_cast<long long>(s->failAllocationAt)));
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return cudaFail(s, e, "cudaMalloc");
  s->allocations.push_back(p);
  *out = static_cast<T*>(p);
  return JGS2_OK;
}

template <class T>
jgs2_status upload(Engine* s, T** out, const T* host, size_t count) {
  jgs2_status st = deviceAlloc(s, out, count);
  if (st != JGS2_OK) return st;
  if (count) CUDA_TRY(s, cudaMemcpyAsync(*out, host, count * sizeof(T), cudaMemcpyHostToDevice, s->stream));
  return JGS2_OK;
}

void releaseDevice(Engine* s) {
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second.first);
  s->graphs.clear();
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void* p : s->allocations) cudaFree(p);
  s->allocations.clear();
  if (s->hForces) cudaFreeHost(s->hForces);
  if (s->hTargets) cudaFreeHost(s->hTargets);
  s->hForces = s->hTargets = nullptr;
  for (cudaEvent_t& e : s->tuneEvents)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  if (s->objectiveUpload) cudaEventDestroy(s->objectiveUpload);
  if (s->readDone) cudaEventDestroy(s->readDone);
  s->objectiveUpload = nullptr;
  if (s->stream) cudaStreamDestroy(s->stream);
  s->stream = nullptr;
}

bool forceActive(const float4& f) { return f.x != 0 || f.y != 0 || f.z != 0; }

void refreshObjectiveFlags(SceneHost& sc) {
  sc.objectiveFlags = (sc.forceCount ? 1u : 0u) | (sc.targetCount ? 2u : 0u);
}

DevParams makeParams(const Engine* s, uint32_t scene, const jgs2_settings& st, bool stop) {
  const SceneHost& sc = s->scenes[scene];
  DevParams p{};
  // packUniforms (jgs2-solver.ts:604-730): (dt, 1/dt, 1/dt^2) formed in
  // double from the timestep and stored as f32.
  const double dt = st.timestep;
  const double inv = 1.0 / dt;
  p.dt = static_cast<float>(dt);
  p.invDt = static_cast<float>(inv);
  p.invDt2 = static_cast<float>(inv * inv);
  p.maxStep = st.max_step;
  for (int i = 0; i < 3; ++i) p.gravity[i] = st.gravity[i];
  p.floorHeight = st.floor_height;
  p.floorStiffness = st.floor_stiffness;
  p.regularization = st.regularization;
  p.rotationEpsilon = st.rotation_epsilon;
  p.velocityDamping = st.velocity_damping;
  p.contactTangentialDamping = st.contact_tangential_damping;
  p.contactMargin = st.contact_margin;
  p.residualTolerance = st.residual_tolerance;
  p.normalizedUpdateTolerance = st.normalized_update_tolerance;
  p.sceneScale = sc.sceneScale;
  p.objectiveFlags = sc.objectiveFlags;
  p.stopEnabled = (s->glob && stop) ? 1u : 0u;
  p.globalization = s->glob ? 1u : 0u;
  p.historyCapacity = JGS2_HISTORY_CAPACITY;
  p.vertexCount = sc.V;
  p.tetCount = sc.T;
  p.cubatureK = sc.K;
  p.bodyCount = sc.bodies;
  p.bodyCorrection = st.horizontal_body_correction ? 1u : 0u;
  p.active = sc.active ? 1u : 0u;
  p.cloth = (sc.C > 0 || sc.H > 0) ? 1u : 0u;
  p.clothLambda = sc.clothLambda;
  p.clothMu = sc.clothMu;
  p.clothThickness = sc.clothThickness;
  p.clothBending = sc.clothBending;
  // contactEnabled (jgs2-solver.ts:2213-2214) and ipcEnabled
  // (jgs2-shader.ts:458-464).
  p.ipcActivation = st.ipc_activation_distance;
  p.ipcStiffness = st.ipc_barrier_stiffness;
  p.ipcMinDistance = sc.ipcMinDistance;
  p.ipcFriction = sc.ipcFriction;
  p.ipcEpsilon = sc.ipcEpsilon;
  p.ipcSafety = sc.ipcSafety;
  p.ipc = (s->glob && (sc.KC > 0 || sc.dynamic) && st.ipc_barrier_stiffness > 0 &&
           st.ipc_activation_distance > sc.ipcMinDistance)
              ? 1u : 0u;
  return p;
}

// Optional per-kernel CUDA event timing of an encoded frame.
struct KernelProfiler {
  static constexpr const char* kNames[JGS2_PROFILE_KINDS] = {"prologue", "vertex_frames", "tet_frames",
                                                              "solve",    "gate",          "convergence",
                                                              "copy",     "epilogue",      "contact"};
  enum Kind { kPrologue = 0, kVertexFrames, kTetFrames, kSolve, kGate, kConvergence, kCopy, kEpilogue, kContact };
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  std::vector<int> kinds;
  size_t used = 0;
  ~KernelProfiler() {
    for (auto& e : pool) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  }
  std::pair<cudaEvent_t, cudaEvent_t> next(int kind) {
    if (used == pool.size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      pool.emplace_back(a, b);
      kinds.push_back(kind);
    }
    kinds[used] = kind;
    return pool[used++];
  }
};

// encodeFrame (src/simulation/gpu/jgs2-solver.ts:2207-2494) on the stream,
// for every scene of the engine at once.  contact: some scene has IPC
// contact this frame.
int encodeFrame(Engine* s, uint32_t iterations, uint32_t schedule, bool bodyCorrection, bool contact,
                KernelProfiler* prof = nullptr) {
  const Buffers& b = s->b;
  cudaStream_t st = s->stream;
  auto timed = [&](int kind, auto&& launch) -> int {
    if (!prof) return launch();
    const auto ev = prof->next(kind);
    cudaEventRecord(ev.first, st);
    const int k = launch();
    cudaEventRecord(ev.second, st);
    return k;
  };
  using P = KernelProfiler;
  int n = 0;
  n += timed(P::kPrologue, [&] { return jgs2::launchPrologue(b, s->dParams, st); });
  const bool colored = schedule == JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL;
  if (!s->glob) {
    // Co-rotated path (legacy frames of jgs2-solver.ts:2207-2494): tet and
    // vertex frames from the current pose, then the regularised solve; no gate.
    for (uint32_t it = 0; it < iterations; ++it) {
      float4* src = (it % 2 == 0) ? b.pos[1] : b.pos[0];
      float4* tgt = (it % 2 == 0) ? b.pos[0] : b.pos[1];
      if (colored) {
        n += timed(P::kCopy, [&] { return jgs2::launchCopy(b, s->dParams, src, tgt, s->V, st); });
        for (uint32_t c = 0; c < s->colorCount; ++c) {
          n += timed(P::kTetFrames, [&] { return jgs2::launchTetPolar(b, s->dParams, tgt, s->T, st); });
          const uint32_t nb = s->needOffsets[c], ne = s->needOffsets[c + 1];
          n += timed(P::kVertexFrames, [&] {
            return jgs2::launchVertexPolar(b, s->dParams, tgt, s->dNeedVertices + nb, ne - nb, st);
          });
          const uint32_t cb = s->colorOffsets[c], ce = s->colorOffsets[c + 1];
          n += timed(P::kSolve, [&] {
            return jgs2::launchCorotatedSolve(b, s->dParams, tgt, tgt, s->dColorVertices + cb, ce - cb, s->K, st);
          });
        }
      } else {
        n += timed(P::kTetFrames, [&] { return jgs2::launchTetPolar(b, s->dParams, src, s->T, st); });
        n += timed(P::kVertexFrames, [&] { return jgs2::launchVertexPolar(b, s->dParams, src, nullptr, s->V, st); });
        n += timed(P::kSolve, [&] { return jgs2::launchCorotatedSolve(b, s->dParams, src, tgt, nullptr, s->V, s->K, st); });
      }
    }
    const float4* finalPos = (iterations % 2 == 0) ? b.pos[1] : b.pos[0];
    n += timed(P::kEpilogue,
               [&] { return jgs2::launchEpilogue(b, s->dParams, finalPos, s->V, bodyCorrection, s->bodies, st); });
    return n;
  }
  const bool dynamic = contact && b.contactDynamic;
  if (contact && !dynamic) n += timed(P::kContact, [&] { return jgs2::launchContactLag(s->b, s->dParams, st); });
  for (uint32_t it = 0; it < iterations; ++it) {
    float4* src = (it % 2 == 0) ? s->b.pos[1] : s->b.pos[0];
    float4* tgt = (it % 2 == 0) ? s->b.pos[0] : s->b.pos[1];
    const bool last = it + 1 == iterations;
    // With a contact surface the iterations alternate between two candidate
    // lists: this iteration's and the previous one's (carried state).
    Buffers b = s->b;
    if (dynamic) {
      const int cur = static_cast<int>(it & 1u), prev = cur ^ 1;
      b.contactIdx = s->dynIdx[cur];
      b.contactScene = s->dynScene[cur];
      b.contactState = s->dynState[cur];
      b.contactFlag = s->dynFlag[cur];
      b.bpCols = s->dynCols[cur];
      b.bpRowOff = s->dynRowOff[cur];
      b.bpPrevRowOff = s->dynRowOff[prev];
      b.bpPrevCols = s->dynCols[prev];
      b.bpPrevState = s->dynState[prev];
      n += timed(P::kContact, [&] { return jgs2::launchBroadPhase(b, s->dParams, src, s->V, it == 0, st); });
    } else if (contact) {
      n += timed(P::kContact, [&] { return jgs2::launchContactRows(b, s->dParams, src, s->V, st); });
    }
    if (colored) {
      n += timed(P::kCopy, [&] { return jgs2::launchCopy(b, s->dParams, src, tgt, s->V, st); });
      // One persistent kernel for all colours (no contact candidates; a
      // contact engine picks its solve variant per colour).
      int sweep = -1;
      if (s->persistentSweep && !b.contactIdx && s->dColorOffsets) {
        sweep = timed(P::kSolve, [&] {
          uint32_t largestColor = 0, largestNeed = 0;
          for (uint32_t c = 0; c < s->colorCount; ++c) {
            largestColor = std::max(largestColor, s->colorOffsets[c + 1] - s->colorOffsets[c]);
            largestNeed = std::max(largestNeed, s->needOffsets[c + 1] - s->needOffsets[c]);
          }
          return jgs2::launchColoredSweep(b, s->dParams, tgt, s->dColorVertices, s->dColorOffsets, s->dNeedVertices,
                                          s->dNeedOffsets, s->colorCount, s->V, s->K, largestColor, largestNeed, last,
                                          s->dSweepBarrier, s->spinLimit, st);
        });
        if (sweep > 0) {
          n += sweep;
          s->sweepLaunched = true;
        }
      }
      for (uint32_t c = 0; sweep <= 0 && c < s->colorCount; ++c) {
        const uint32_t nb = s->needOffsets[c], ne = s->needOffsets[c + 1];
        n += timed(P::kVertexFrames, [&] {
          // The final colour of the frame refreshes every frame so the stored
          // frames match a full vertexPolarRotation pass.
          if (last && c + 1 == s->colorCount) return jgs2::launchVertexPolar(b, s->dParams, tgt, nullptr, s->V, st);
          return jgs2::launchVertexPolar(b, s->dParams, tgt, s->dNeedVertices + nb, ne - nb, st);
        });
        const uint32_t cb = s->colorOffsets[c], ce = s->colorOffsets[c + 1];
        n += timed(P::kSolve, [&] {
          return jgs2::launchSolve(b, s->dParams, tgt, tgt, s->dColorVertices + cb, ce - cb, s->K, false, st);
        });
      }
    } else {
      // Stable Jacobi: the prologue (iteration 0) and the previous iteration's
      // convergence pass leave the source pose's incident system in b.incident.
      n += timed(P::kSolve, [&] { return jgs2::launchSolve(b, s->dParams, src, tgt, nullptr, s->V, s->K, true, st); });
    }
    if (contact) {
      // Safe-step scaling, exact validation of the scaled pose (a failure
      // restores the source), before the assembled gate (jgs2-solver.ts:2340-2393).
      n += timed(P::kContact, [&] {
        int k = jgs2::launchContactStep(b, s->dParams, src, tgt, st);
        k += jgs2::launchContactApply(b, s->dParams, src, tgt, s->V, false, st);
        k += jgs2::launchContactValidate(b, s->dParams, tgt, st);
        k += jgs2::launchContactApply(b, s->dParams, src, tgt, s->V, true, st);
        return k;
      });
    }
    n += timed(P::kGate, [&] { return jgs2::launchGate(b, s->dParams, src, tgt, st); });
    if (contact)
      n += timed(P::kContact, [&] { return jgs2::launchContactGradient(b, s->dParams, src, tgt, s->V, st); });
    n += timed(P::kConvergence,
               [&] { return jgs2::launchConvergence(b, s->dParams, src, tgt, !colored && !last, st); });
    if (contact) n += timed(P::kContact, [&] { return jgs2::launchContactPromote(b, s->dParams, st); });
  }
  const float4* finalPos = (iterations % 2 == 0) ? s->b.pos[1] : s->b.pos[0];
  n += timed(P::kEpilogue,
             [&] { return jgs2::launchEpilogue(s->b, s->dParams, finalPos, s->V, bodyCorrection, s->bodies, st); });
  return n;
}

double medianMs(std::vector<float> v) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const size_t n = v.size();
  return n % 2 ? v[n / 2] : 0.5 * (static_cast<double>(v[n / 2 - 1]) + v[n / 2]);
}

// Encodes `frames` frames of `iterations` iterations for every scene with its
// resolved settings (one per scene; the schedule must agree).
jgs2_status runFrames(Engine* s, const std::vector<jgs2_settings>& st, uint32_t frames, uint32_t iterations,
                      bool stop, KernelProfiler* prof = nullptr) {
  if (s->glob && iterations > JGS2_HISTORY_CAPACITY)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("Stable JGS2 records at most %u nonlinear iterations per frame; got %u.",
                       JGS2_HISTORY_CAPACITY, iterations));
  const uint32_t schedule = st[0].schedule;
  bool body = false;
  for (size_t i = 0; i < st.size(); ++i) {
    if (st[i].schedule != schedule)
      return fail(s, JGS2_INVALID_ARGUMENT, "All scenes of one batched step must use the same schedule.");
    body = body || st[i].horizontal_body_correction != 0;
  }
  if (s->dynamic && schedule != JGS2_SCHEDULE_JACOBI)
    return fail(s, JGS2_INVALID_ARGUMENT, "The IPC broad phase steps the Jacobi schedule only.");
  if (schedule == JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL && !s->coloringBuilt)
    return fail(s, JGS2_UNSUPPORTED,
                "This batch was created without graph colouring: give one of its scenes the graph-coloured "
                "schedule when the batch is created to step it with that schedule.");
  const uint32_t sub = schedule == JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL ? s->colorCount : 1u;
  if (s->glob && static_cast<uint64_t>(iterations) * sub > JGS2_MAX_GLOBALIZED_ITERATIONS_PER_SUBMISSION / frames)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("Stable JGS2 may encode at most %u total nonlinear iterations per submission; got %u "
                       "frames * %u iterations.",
                       JGS2_MAX_GLOBALIZED_ITERATIONS_PER_SUBMISSION, frames, iterations * sub));
  bool contact = false;
  for (uint32_t i = 0; i < s->scenes.size(); ++i) {
    s->hParams[i] = makeParams(s, i, st[i], stop);
    contact = contact || s->hParams[i].ipc != 0;
  }
  if (s->dynamic && contact) {
    for (uint32_t i = 0; i < s->scenes.size(); ++i)
      if (s->hParams[i].ipc && !(s->hParams[i].maxStep > 0.0f))
        return fail(s, JGS2_INVALID_ARGUMENT,
                    "The IPC broad phase bounds each iteration's motion by maxStep; maxStep must be positive.");
  }
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaMemcpyAsync(s->dParams, s->hParams.data(), sizeof(DevParams) * s->hParams.size(),
                              cudaMemcpyHostToDevice, s->stream));
  // The graph of a frame in the engine's current launch shape, captured at
  // the first use of its key.
  using GraphMap = decltype(s->graphs);
  GraphMap::iterator it = s->graphs.end();
  auto graphFor = [&]() -> jgs2_status {
    const auto key = std::make_tuple(iterations, schedule, body, contact, s->b.solveShift);
    it = s->graphs.find(key);
    if (it == s->graphs.end()) {
      cudaGraph_t graph = nullptr;
      CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      const int n = encodeFrame(s, iterations, schedule, body, contact);
      cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
      if (e != cudaSuccess) return cudaFail(s, e, "cudaStreamEndCapture");
      cudaGraphExec_t exec = nullptr;
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return cudaFail(s, e, "cudaGraphInstantiate");
      it = s->graphs.emplace(key, std::make_pair(exec, n)).first;
    }
    return JGS2_OK;
  };
  const bool graphs = s->useGraphs && !prof;
  // One frame: a graph replay or, without graphs, direct launches.
  auto frame = [&]() -> jgs2_status {
    if (!graphs) {
      s->launches += encodeFrame(s, iterations, schedule, body, contact, prof);
      return JGS2_OK;
    }
    CUDA_TRY(s, cudaGraphLaunch(it->second.first, s->stream));
    s->launches += static_cast<uint64_t>(it->second.second);
    return JGS2_OK;
  };
  if (graphs) {
    const jgs2_status st2 = graphFor();
    if (st2 != JGS2_OK) return st2;
  }
  for (uint32_t f = 0; f < frames; ++f) {
    if (s->tuneLeft == 0 || prof) {
      const jgs2_status st2 = frame();
      if (st2 != JGS2_OK) return st2;
      continue;
    }
    // Tuned frame: the shapes take turns; each frame is timed on the stream,
    // its graph captured before the first event.
    const uint32_t shape = s->tuneNext;
    s->b.solveShift = shape;
    if (graphs) {
      const jgs2_status st3 = graphFor();
      if (st3 != JGS2_OK) return st3;
    }
    CUDA_TRY(s, cudaEventRecord(s->tuneEvents[0], s->stream));
    const jgs2_status st2 = frame();
    if (st2 != JGS2_OK) return st2;
    CUDA_TRY(s, cudaEventRecord(s->tuneEvents[1], s->stream));
    CUDA_TRY(s, cudaEventSynchronize(s->tuneEvents[1]));
    float ms = 0.0f;
    CUDA_TRY(s, cudaEventElapsedTime(&ms, s->tuneEvents[0], s->tuneEvents[1]));
    s->tuneMs[shape].push_back(ms);
    s->tuneNext = (shape + 1) % JGS2_LAUNCH_SHAPES;
    if (--s->tuneLeft == 0) {
      uint32_t best = 0;
      double bestMs = 0;
      for (uint32_t c = 0; c < JGS2_LAUNCH_SHAPES; ++c) {
        const double m = medianMs(s->tuneMs[c]);
        if (c == 0 || m < bestMs) { best = c; bestMs = m; }
      }
      s->b.solveShift = best;
      if (graphs) {
        const jgs2_status st3 = graphFor();
        if (st3 != JGS2_OK) return st3;
      }
    }
  }
  CUDA_TRY(s, cudaGetLastError());
  for (uint32_t i = 0; i < s->scenes.size(); ++i) {
    s->scenes[i].submitted = st[i];
    s->scenes[i].submittedIterations = iterations;
    if (s->glob) s->scenes[i].recordsAvailable = true;
  }
  return JGS2_OK;
}

uint32_t normalizeOdd(uint32_t it) {
  const uint32_t i = std::max(1u, it);
  return i % 2 == 0 ? i + 1 : i;
}

jgs2_status usable(Engine* s) {
  if (!s) return fail(nullptr, JGS2_INVALID_ARGUMENT, "solver is NULL.");
  if (s->destroyed) return fail(s, JGS2_DESTROYED, "JGS2GpuSolver has been destroyed.");
  return JGS2_OK;
}

// resolveStepSettings (jgs2-solver.ts:1974-2005) for one scene.
jgs2_status resolveStep(Engine* s, uint32_t scene, const jgs2_settings* o, uint32_t mask, jgs2_settings* out) {
  const SceneHost& sc = s->scenes[scene];
  if (o && (mask & JGS2_SET_TIMESTEP) && static_cast<float>(o->timestep) != sc.preprocessingTimestep)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("JGS2 was precomputed for timestep %g, but the step requested %g. Regenerate the "
                       "precomputation before changing timestep.",
                       sc.preprocessingTimestep, o->timestep));
  if (sc.KC > 0 && o && (mask & JGS2_SET_IPC_MINIMUM_DISTANCE) && o->ipc_minimum_distance != sc.ipcMinDistance)
    return fail(s, JGS2_INVALID_ARGUMENT,
                "ipcMinimumDistance is fixed when an IPC solver is created; recreate the solver before changing it.");
  std::string err;
  if (!resolve(sc.defaults, o, mask, out, &err)) return fail(s, JGS2_INVALID_ARGUMENT, err);
  // Objectives and mesh contacts are not translation invariant per body, so
  // they keep their solved centre-of-mass motion (jgs2-solver.ts:1999-2009).
  if (s->glob && (sc.objectiveFlags != 0 || (sc.KC > 0 && out->ipc_barrier_stiffness > 0)) &&
      out->horizontal_body_correction)
    out->horizontal_body_correction = 0;
  return JGS2_OK;
}

jgs2_status stepCommon(jgs2_solver* s, uint32_t frames, int exactIterations, const jgs2_settings* o,
                       uint32_t mask, bool batch, KernelProfiler* prof = nullptr) {
  if (!s) return fail(nullptr, JGS2_INVALID_ARGUMENT, "solver is NULL.");
  if (s->destroyed) return fail(s, JGS2_DESTROYED, "JGS2GpuSolver has been destroyed.");
  if (batch && (frames < 1 || frames > JGS2_MAX_BATCH_FRAMES))
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("frameCount must be a positive safe integer no greater than %u; got %u.",
                       JGS2_MAX_BATCH_FRAMES, frames));
  if (exactIterations == 0) return fail(s, JGS2_INVALID_ARGUMENT, "iterations must be a positive safe integer; got 0.");
  std::vector<jgs2_settings> st(1);
  const jgs2_status rs = resolveStep(s, 0, o, mask, &st[0]);
  if (rs != JGS2_OK) return rs;
  const bool production = exactIterations < 0;
  const uint32_t iterations = production ? normalizeOdd(st[0].iterations) : static_cast<uint32_t>(exactIterations);
  return runFrames(s, st, frames, iterations, production, prof);
}

// After a synchronisation: a broad-phase list that did not fit its capacity
// (the iteration then listed nothing) fails the call.
jgs2_status checkBroadPhase(Engine* s) {
  if (jgs2::boundsChecked()) {
    uint32_t site = 0;
    CUDA_TRY(s, jgs2::takeBoundsViolation(&site));
    if (site != 0)
      return fail(s, JGS2_DEVICE_ERROR,
                  format("A device index check failed (site %u); the out-of-range access was skipped and the step's "
                         "result is invalid.",
                         site));
  }
  if (s->sweepLaunched) {
    // The persistent coloured sweep's error word (a barrier that gave up).
    uint32_t words[4];
    CUDA_TRY(s, cudaMemcpy(words, s->dSweepBarrier, sizeof(words), cudaMemcpyDeviceToHost));
    if (words[2] != 0u)
      return fail(s, JGS2_TIMEOUT,
                  format("A grid barrier of the graph-coloured sweep waited longer than its bound of %u polls; the "
                         "step's result is invalid.",
                         s->spinLimit));
  }
  if (!s->dynamic) return JGS2_OK;
  uint32_t status[4];
  CUDA_TRY(s, cudaMemcpy(status, s->b.bpStatus, sizeof(status), cudaMemcpyDeviceToHost));
  if (status[1] == 0u) return JGS2_OK;
  return fail(s, JGS2_DEVICE_ERROR,
              format("The IPC broad phase needed %u candidates in one iteration, above its capacity of %llu; "
                     "raise contact_surface.candidate_capacity.",
                     status[2], static_cast<unsigned long long>(s->bpCapacity)));
}

jgs2_status readRegion(Engine* s, const void* dev, size_t bytes, void* host) {
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return checkBroadPhase(s);
}

// The host mirrors may change only after the previous upload from them has
// been consumed by the copy engine.
jgs2_status waitObjectiveMirror(Engine* s) {
  if (!s->objectiveUploadPending) return JGS2_OK;
  CUDA_TRY(s, cudaEventSynchronize(s->objectiveUpload));
  s->objectiveUploadPending = false;
  return JGS2_OK;
}

jgs2_status writeObjectives(Engine* s, uint32_t scene, uint32_t firstVertex, uint32_t vertexCount, bool forces,
                            bool targets) {
  CUDA_TRY(s, cudaSetDevice(s->device));
  if (forces)
    CUDA_TRY(s, cudaMemcpyAsync(s->b.forces + firstVertex, s->hForces + firstVertex, sizeof(float4) * vertexCount,
                                cudaMemcpyHostToDevice, s->stream));
  if (targets)
    CUDA_TRY(s, cudaMemcpyAsync(s->b.targets + firstVertex, s->hTargets + firstVertex,
                                sizeof(float4) * vertexCount, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaEventRecord(s->objectiveUpload, s->stream));
  s->objectiveUploadPending = true;
  SceneHost& sc = s->scenes[scene];
  refreshObjectiveFlags(sc);
  sc.objectiveRevision += 1;
  return JGS2_OK;
}

// ---- engine construction -------------------------------------------------------

// Host-side checks and derived data of one scene input (create, :971-1083).
struct PreparedScene {
  const jgs2_input* in = nullptr;
  jgs2_settings resolved{};
  uint32_t colorCount = 0;
  std::vector<uint32_t> colors;
  bool colored = false;
  bool stable = true;  // stable Neo-Hookean (else co-rotated linear)
  bool dynamic = false;        // contact surface for the device broad phase
  ContactSurface surface;
  std::string error;  // message of a failed preparation (thread-safe copy)
};

jgs2_status prepareScene(const jgs2_input* in, const jgs2_settings* settings, uint32_t mask, bool colour,
                         PreparedScene* out) {
  std::string err;
  if (!validateInput(in, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  // inferJGS2MaterialMode (layout.ts:509-522).
  uint32_t stable = 0;
  for (uint32_t t = 0; t < in->tet_count; ++t) stable += in->tet_meta[4ull * t + 3] == 1.0f ? 1u : 0u;
  if (stable != 0 && stable != in->tet_count)
    return fail(nullptr, JGS2_INVALID_ARGUMENT,
                "A production JGS2 solve cannot mix stable Neo-Hookean and co-rotated regression tetrahedra in one "
                "precomputation.");
  out->in = in;
  out->stable = stable == in->tet_count;
  if (in->cloth && in->cloth->triangle_count > 0 && !out->stable)
    return fail(nullptr, JGS2_INVALID_ARGUMENT, "Triangle cloth requires the stable Neo-Hookean production path.");
  const uint64_t contacts = uint64_t(in->contact_vertex_triangle_count) + in->contact_edge_edge_count;
  if (contacts > 0 && !out->stable)
    return fail(nullptr, JGS2_INVALID_ARGUMENT,
                "IPC contact candidates require the stable Neo-Hookean production path.");
  if (in->contact_surface) {
    if (!out->stable)
      return fail(nullptr, JGS2_INVALID_ARGUMENT, "IPC contact requires the stable Neo-Hookean production path.");
    // The broad phase steps the Jacobi schedule only: no colouring.
    colour = false;
    out->dynamic = true;
    buildContactSurface(in, &out->surface);
  }
  out->colored = colour;
  if (colour) out->colors = colorInput(in, &out->colorCount);
  if (out->colorCount > JGS2_MAX_SCHEDULE_COLORS)
    return fail(nullptr, JGS2_INVALID_ARGUMENT,
                format("Colored Gauss-Seidel supports at most %u colors; the small-scene conflict graph needs %u.",
                       JGS2_MAX_SCHEDULE_COLORS, out->colorCount));
  jgs2_settings base;
  defaults(&base);
  if (!resolve(base, settings, mask, &out->resolved, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  if (contacts > 0) {
    // The source pose must clear the minimum distance by an f32 rounding
    // margin (jgs2-solver.ts:1040-1070).
    const double minimum = staticContactDistance(in);
    const double margin = 8.0 * std::ldexp(1.0, -24) *
                          std::max(1.0, std::max(double(out->resolved.ipc_activation_distance), std::fabs(minimum)));
    const double required = double(out->resolved.ipc_minimum_distance) + margin;
    if (!std::isfinite(minimum) || !(minimum > required))
      return fail(nullptr, JGS2_INVALID_ARGUMENT,
                  format("IPC candidates require an initially feasible source pose with distance greater than %g "
                         "(minimum plus an f32 safety margin); got %g.", required, minimum));
  }
  if (out->dynamic) {
    // The same check over the superset of the contact surface; candidates
    // farther than the cutoff cannot fail it.
    const double dMin = out->resolved.ipc_minimum_distance;
    const double cutoff =
        2.0 * (dMin + 8.0 * std::ldexp(1.0, -24) * std::max(1.0, double(out->resolved.ipc_activation_distance))) +
        1e-9;
    const double minimum = surfaceContactDistance(in, out->surface, cutoff);
    if (minimum != INFINITY) {
      const double margin = 8.0 * std::ldexp(1.0, -24) *
                            std::max(1.0, std::max(double(out->resolved.ipc_activation_distance), std::fabs(minimum)));
      const double required = dMin + margin;
      if (!std::isfinite(minimum) || !(minimum > required))
        return fail(nullptr, JGS2_INVALID_ARGUMENT,
                    format("IPC candidates require an initially feasible source pose with distance greater than %g "
                           "(minimum plus an f32 safety margin); got %g.", required, minimum));
    }
  }
  const double m = out->stable ? minimumInputDeterminant(in) : 1.0;
  if (!std::isfinite(m) || !(m > kDeterminantFloor))
    return fail(nullptr, JGS2_INFEASIBLE_INPUT,
                format("A stable Neo-Hookean production solve requires an initially feasible pose with minimum J "
                       "greater than %g; got %g.", kDeterminantFloor, m));
  return JGS2_OK;
}

// computeJGS2InitialDynamicSceneScale (jgs2-solver.ts:732-768).
float initialSceneScale(const jgs2_input* in) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  uint32_t dyn = 0;
  for (uint32_t v = 0; v < in->vertex_count; ++v) {
    if (in->vertex_info[4ull * v + 2] != 0) continue;
    dyn++;
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], static_cast<double>(in->positions[4ull * v + k]));
      hi[k] = std::max(hi[k], static_cast<double>(in->positions[4ull * v + k]));
    }
  }
  const double d = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                             (hi[2] - lo[2]) * (hi[2] - lo[2]));
  return static_cast<float>(dyn > 0 && std::isfinite(d) && d > 0 ? d : kDegenerateSceneScale);
}

// Concatenates the scenes into one device arena, builds the reduction block
// tables and runs the GPU preflight of every scene's initial pose.
jgs2_status buildEngine(Engine* sp, const std::vector<PreparedScene>& prep, int device) {
  const uint32_t S = static_cast<uint32_t>(prep.size());
  sp->device = device;
  // JGS2_NO_GRAPHS=1 launches each frame's kernels directly (debugging).
  sp->useGraphs = std::getenv("JGS2_NO_GRAPHS") == nullptr;
  if (const char* e = std::getenv("JGS2_BARRIER_SPIN_LIMIT")) sp->spinLimit = static_cast<uint32_t>(std::strtoul(e, nullptr, 10));
  if (const char* e = std::getenv("JGS2_COLOR_SWEEP")) sp->persistentSweep = std::string(e) == "persistent";
  if (const char* e = std::getenv("JGS2_FAIL_ALLOCATION")) sp->failAllocationAt = std::strtoll(e, nullptr, 10);
  sp->glob = prep[0].stable;
  for (const PreparedScene& p : prep)
    if (p.stable != sp->glob)
      return fail(nullptr, JGS2_INVALID_ARGUMENT,
                  "A batch cannot mix stable Neo-Hookean scenes with co-rotated linear scenes.");
  sp->scenes.resize(S);
  uint64_t V = 0, T = 0, bodies = 0, C = 0, H = 0, KC = 0;
  uint32_t K = 0, colorCount = 1;
  for (uint32_t i = 0; i < S; ++i) {
    const jgs2_input* in = prep[i].in;
    SceneHost& sc = sp->scenes[i];
    sc.V = in->vertex_count;
    sc.T = in->tet_count;
    sc.K = in->cubature_k;
    sc.vOff = static_cast<uint32_t>(V);
    sc.tOff = static_cast<uint32_t>(T);
    sc.bodyOff = static_cast<uint32_t>(bodies);
    sc.cOff = static_cast<uint32_t>(C);
    sc.hOff = static_cast<uint32_t>(H);
    if (const jgs2_cloth_input* cl = in->cloth) {
      sc.C = cl->triangle_count;
      sc.H = cl->hinge_count;
      // packJGS2GpuClothArena (cloth-layout.ts:358-372): plane-stress Lame
      // parameters formed in double, stored as f32.
      const double E = cl->young_modulus, nu = cl->poisson_ratio;
      sc.clothLambda = static_cast<float>(E * nu / (1 - nu * nu));
      sc.clothMu = static_cast<float>(E / (2 * (1 + nu)));
      sc.clothThickness = cl->thickness;
      sc.clothBending = cl->bending_stiffness;
      C += sc.C;
      H += sc.H;
    }
    sc.kOff = static_cast<uint32_t>(KC);
    sc.KC = in->contact_indices ? in->contact_vertex_triangle_count + in->contact_edge_edge_count : 0u;
    sc.ipcMinDistance = prep[i].resolved.ipc_minimum_distance;
    sc.ipcFriction = prep[i].resolved.ipc_friction_coefficient;
    sc.ipcEpsilon = prep[i].resolved.ipc_friction_velocity_epsilon;
    sc.ipcSafety = prep[i].resolved.ipc_step_safety;
    KC += sc.KC;
    if (prep[i].dynamic) {
      sc.dynamic = true;
      sc.bpTris = static_cast<uint32_t>(prep[i].surface.tris.size());
      sc.bpEdges = static_cast<uint32_t>(prep[i].surface.edges.size());
      sc.bpCapacity = prep[i].surface.capacity;
      sc.bpSuperset = prep[i].surface.superset;
    }
    uint32_t maxBody = 0;
    for (uint32_t v = 0; v < sc.V; ++v) maxBody = std::max(maxBody, in->vertex_info[4ull * v + 3]);
    sc.bodies = maxBody + 1;
    sc.defaults = prep[i].resolved;
    sc.submitted = prep[i].resolved;
    sc.preprocessingTimestep = prep[i].resolved.timestep;
    sc.colors = prep[i].colors;
    sc.colorCount = prep[i].colored ? prep[i].colorCount : 0u;
    sc.sceneScale = initialSceneScale(in);
    V += sc.V;
    T += sc.T;
    bodies += sc.bodies;
    K = std::max(K, sc.K);
    colorCount = std::max(colorCount, sc.colorCount);
  }
  if (V > 0xffffffffull / 16 || T > 0xffffffffull / 16 || C > 0xffffffffull / 16 || H > 0xffffffffull / 16 ||
      KC > 0xffffffffull / 16)
    return fail(nullptr, JGS2_INVALID_ARGUMENT, "The scenes together exceed the engine's index range.");
  sp->V = static_cast<uint32_t>(V);
  sp->T = static_cast<uint32_t>(T);
  sp->C = static_cast<uint32_t>(C);
  sp->H = static_cast<uint32_t>(H);
  sp->KC = static_cast<uint32_t>(KC);
  sp->K = K;
  sp->bodies = static_cast<uint32_t>(bodies);
  sp->coloringBuilt = true;
  for (const PreparedScene& p : prep) sp->coloringBuilt = sp->coloringBuilt && p.colored;
  if (!sp->coloringBuilt) colorCount = 0;
  sp->colorCount = colorCount;
  const uint32_t nV = sp->V, nT = sp->T;
  // Contact surfaces: rows, triangles and edges of each scene in order.
  uint64_t bpT = 0, bpE = 0, bpR = 0, bpCap = 0;
  for (SceneHost& sc : sp->scenes) {
    if (!sc.dynamic) continue;
    sp->dynamic = true;
    sc.bpTriOff = static_cast<uint32_t>(bpT);
    sc.bpEdgeOff = static_cast<uint32_t>(bpE);
    sc.bpRowOff = static_cast<uint32_t>(bpR);
    sc.bpRows = sc.V + sc.bpEdges;
    bpT += sc.bpTris;
    bpE += sc.bpEdges;
    bpR += sc.bpRows;
    bpCap += sc.bpCapacity;
  }
  if (sp->dynamic && sp->KC > 0)
    return fail(nullptr, JGS2_INVALID_ARGUMENT, "A batch cannot mix static IPC candidates with contact surfaces.");
  if (bpCap >= (1ull << 28) || bpR >= (1ull << 31) || bpT >= (1ull << 31) || bpE >= (1ull << 31))
    return fail(nullptr, JGS2_INVALID_ARGUMENT,
                "The contact surfaces of one batch must stay below 2^28 candidates and 2^31 rows or primitives.");
  sp->bpCapacity = bpCap;

  // Objectives (packJGS2VertexObjectives, layout.ts:635-668).
  std::vector<float4> initialForces(nV), initialTargets(nV);
  sp->pinned.assign(nV, 0);
  parallelFor(S, [&](uint32_t i) {
    const jgs2_input* in = prep[i].in;
    SceneHost& sc = sp->scenes[i];
    sc.forceCount = sc.targetCount = 0;
    for (uint32_t v = 0; v < sc.V; ++v) {
      const uint32_t g = sc.vOff + v;
      const float* f = in->external_forces ? &in->external_forces[3ull * v] : nullptr;
      initialForces[g] = f ? make_float4(f[0], f[1], f[2], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float* tp = in->target_positions ? &in->target_positions[3ull * v] : &in->positions[4ull * v];
      initialTargets[g] = make_float4(tp[0], tp[1], tp[2], in->target_stiffnesses ? in->target_stiffnesses[v] : 0.f);
      if (forceActive(initialForces[g])) sc.forceCount++;
      if (initialTargets[g].w > 0) sc.targetCount++;
      sp->pinned[g] = in->vertex_info[4ull * v + 2] != 0;
    }
    refreshObjectiveFlags(sc);
  });

  // Colour lists (union over scenes) and per-colour frame lists.
  std::vector<uint32_t> byColor;
  std::vector<uint32_t> need;
  sp->colorOffsets.assign(colorCount + 1, 0);
  sp->needOffsets.assign(colorCount + 1, 0);
  if (sp->coloringBuilt) {
    std::vector<uint32_t> mark(nV, 0xffffffffu);
    for (uint32_t c = 0; c < colorCount; ++c) {
      std::vector<uint32_t> needList;
      for (uint32_t i = 0; i < S; ++i) {
        const jgs2_input* in = prep[i].in;
        const SceneHost& sc = sp->scenes[i];
        auto add = [&](uint32_t u) {
          if (mark[u] != c) { mark[u] = c; needList.push_back(u); }
        };
        for (uint32_t v = 0; v < sc.V; ++v) {
          if (sc.colors[v] != c) continue;
          byColor.push_back(sc.vOff + v);
          add(sc.vOff + v);
          for (uint32_t k = 0; k < sc.K; ++k) {
            const size_t r = static_cast<size_t>(v) * sc.K + k;
            const uint32_t t = in->cubature_tet_ids[r];
            if (t == kEmptyTet || t >= sc.T || !(in->cubature_weights[r] > 0)) continue;
            for (int l = 0; l < 4; ++l) add(sc.vOff + in->tet_indices[4ull * t + l]);
          }
        }
      }
      std::sort(needList.begin(), needList.end());
      need.insert(need.end(), needList.begin(), needList.end());
      sp->colorOffsets[c + 1] = static_cast<uint32_t>(byColor.size());
      sp->needOffsets[c + 1] = static_cast<uint32_t>(need.size());
    }
  }

  // Device packing.
  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) return fail(nullptr, JGS2_DEVICE_ERROR, format("cudaSetDevice: %s", cudaGetErrorString(ce)));
  if (jgs2::solveGroupsPerBlock(K) == 0)
    return fail(nullptr, JGS2_UNSUPPORTED,
                format("cubatureK %u is too large for the shared-memory record cache of one vertex.", K));
  ce = cudaStreamCreateWithFlags(&sp->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return fail(nullptr, JGS2_DEVICE_ERROR, format("cudaStreamCreate: %s", cudaGetErrorString(ce)));
  auto bail = [&](jgs2_status st) {
    gGlobalError = sp->error;
    releaseDevice(sp);
    return st;
  };
  std::vector<float4> pos(nV), rest(nV), vel(nV, make_float4(0, 0, 0, 0));
  std::vector<uint4> info(nV);
  std::vector<uint32_t> vertexScene(nV), colors(nV);
  // Tet record: rows of inverse Dm (shape gradients g1..g3) with volume,
  // lambda, mu in w, then the four (global) indices.
  std::vector<float4> tets(4ull * nT);
  std::vector<uint32_t> adjacencyOffsets(S + 1, 0);
  for (uint32_t i = 0; i < S; ++i)
    adjacencyOffsets[i + 1] = adjacencyOffsets[i] + static_cast<uint32_t>(prep[i].in->adjacency_length);
  std::vector<uint32_t> adjacency(adjacencyOffsets[S]);
  const size_t R = static_cast<size_t>(nV) * K;
  // Record headers: tet id and weight, then the tet's vertex indices, so a
  // record's vertex data can be fetched without waiting for its tet.  Scenes
  // with fewer records per vertex than the widest are padded with empty ones.
  std::vector<uint4> head(2 * R, make_uint4(kEmptyTet, 0u, 0u, 0u));
  for (size_t r = 0; r < R; ++r) head[2 * r + 1] = make_uint4(0u, 0u, 0u, 0u);
  std::vector<float> basis(36 * R, 0.f);
  parallelFor(S, [&](uint32_t i) {
    const jgs2_input* in = prep[i].in;
    const SceneHost& sc = sp->scenes[i];
    const uint32_t adjOff = adjacencyOffsets[i];
    for (uint32_t v = 0; v < sc.V; ++v) {
      const uint32_t g = sc.vOff + v;
      pos[g] = make_float4(in->positions[4ull * v], in->positions[4ull * v + 1], in->positions[4ull * v + 2], 1.f);
      rest[g] = make_float4(in->vertex_rest[4ull * v], in->vertex_rest[4ull * v + 1], in->vertex_rest[4ull * v + 2],
                            in->vertex_rest[4ull * v + 3]);
      info[g] = make_uint4(adjOff + in->vertex_info[4ull * v], in->vertex_info[4ull * v + 1],
                           in->vertex_info[4ull * v + 2], sc.bodyOff + in->vertex_info[4ull * v + 3]);
      if (in->velocities)
        vel[g] = make_float4(in->velocities[4ull * v], in->velocities[4ull * v + 1], in->velocities[4ull * v + 2], 0.f);
      vertexScene[g] = i;
      colors[g] = sc.colors.empty() ? 0u : sc.colors[v];
    }
    for (uint32_t t = 0; t < sc.T; ++t) {
      const float* m = &in->tet_inverse_dm[12ull * t];
      const float* meta = &in->tet_meta[4ull * t];
      const size_t g = sc.tOff + t;
      tets[4 * g] = make_float4(m[0], m[4], m[8], meta[0]);
      tets[4 * g + 1] = make_float4(m[1], m[5], m[9], meta[1]);
      tets[4 * g + 2] = make_float4(m[2], m[6], m[10], meta[2]);
      const uint4 q = make_uint4(sc.vOff + in->tet_indices[4ull * t], sc.vOff + in->tet_indices[4ull * t + 1],
                                 sc.vOff + in->tet_indices[4ull * t + 2], sc.vOff + in->tet_indices[4ull * t + 3]);
      std::memcpy(&tets[4 * g + 3], &q, sizeof(q));
    }
    for (uint32_t v = 0; v < sc.V; ++v) {
      const uint32_t start = in->vertex_info[4ull * v], count = in->vertex_info[4ull * v + 1];
      for (uint32_t a = 0; a < count; ++a) {
        const uint32_t t = in->adjacency[start + a];
        uint32_t slot = 0;
        for (uint32_t l = 0; l < 4; ++l)
          if (in->tet_indices[4ull * t + l] == v) { slot = l; break; }
        adjacency[adjOff + start + a] = (sc.tOff + t) * 4u + slot;
      }
    }
    for (uint32_t v = 0; v < sc.V; ++v) {
      for (uint32_t k = 0; k < sc.K; ++k) {
        const size_t src = static_cast<size_t>(v) * sc.K + k;
        const size_t dst = static_cast<size_t>(sc.vOff + v) * K + k;
        const uint32_t t = in->cubature_tet_ids[src];
        uint32_t wbits;
        std::memcpy(&wbits, &in->cubature_weights[src], 4);
        const bool valid = t != kEmptyTet && t < sc.T;
        head[2 * dst] = make_uint4(valid ? sc.tOff + t : kEmptyTet, wbits, 0u, 0u);
        if (valid)
          head[2 * dst + 1] =
              make_uint4(sc.vOff + in->tet_indices[4ull * t], sc.vOff + in->tet_indices[4ull * t + 1],
                         sc.vOff + in->tet_indices[4ull * t + 2], sc.vOff + in->tet_indices[4ull * t + 3]);
        std::memcpy(&basis[36 * dst], &in->cubature_basis[36 * src], sizeof(float) * 36);
      }
    }
  });
  // Cloth (packJGS2GpuClothArena, cloth-layout.ts:335-452, in this engine's
  // layout): triangles and hinges with global indices, and per vertex its
  // incident triangles then hinges in ascending element order, each entry
  // element * 4 + the vertex's local slot.
  const uint32_t nC = sp->C, nH = sp->H;
  const bool anyCloth = nC + nH > 0;
  std::vector<float4> clothTris(2ull * nC), clothHinges(2ull * nH);
  std::vector<uint4> clothRange(anyCloth ? nV : 0, make_uint4(0u, 0u, 0u, 0u));
  std::vector<uint32_t> incidence(3ull * nC + 4ull * nH);
  if (anyCloth) parallelFor(S, [&](uint32_t i) {
    const jgs2_cloth_input* cl = prep[i].in->cloth;
    const SceneHost& sc = sp->scenes[i];
    if (!cl || sc.C + sc.H == 0) return;
    auto bits = [](uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; };
    std::vector<uint32_t> tRows(sc.V + 1, 0), hRows(sc.V + 1, 0);
    for (uint32_t c = 0; c < sc.C; ++c) {
      const uint32_t* q = &cl->triangle_indices[3ull * c];
      const float* inv = &cl->triangle_inverse_rest_bases[4ull * c];
      const size_t g = sc.cOff + c;
      clothTris[2 * g] = make_float4(bits(sc.vOff + q[0]), bits(sc.vOff + q[1]), bits(sc.vOff + q[2]),
                                     cl->triangle_rest_areas[c]);
      clothTris[2 * g + 1] = make_float4(inv[0], inv[1], inv[2], inv[3]);
      for (int l = 0; l < 3; ++l) tRows[q[l] + 1]++;
    }
    for (uint32_t h = 0; h < sc.H; ++h) {
      const uint32_t* q = &cl->hinge_indices[4ull * h];
      const size_t g = sc.hOff + h;
      clothHinges[2 * g] = make_float4(bits(sc.vOff + q[0]), bits(sc.vOff + q[1]), bits(sc.vOff + q[2]),
                                       bits(sc.vOff + q[3]));
      clothHinges[2 * g + 1] = make_float4(cl->hinge_rest_angles[h], cl->hinge_rest_edge_lengths[h], 0.f, 0.f);
      for (int l = 0; l < 4; ++l) hRows[q[l] + 1]++;
    }
    for (uint32_t v = 0; v < sc.V; ++v) {
      tRows[v + 1] += tRows[v];
      hRows[v + 1] += hRows[v];
    }
    const uint32_t triBase = 3u * sc.cOff, hingeBase = 3u * nC + 4u * sc.hOff;
    for (uint32_t v = 0; v < sc.V; ++v)
      clothRange[sc.vOff + v] = make_uint4(triBase + tRows[v], tRows[v + 1] - tRows[v], hingeBase + hRows[v],
                                           hRows[v + 1] - hRows[v]);
    std::vector<uint32_t> cursor(tRows.begin(), tRows.end() - 1);
    for (uint32_t c = 0; c < sc.C; ++c)
      for (uint32_t l = 0; l < 3; ++l)
        incidence[triBase + cursor[cl->triangle_indices[3ull * c + l]]++] = (sc.cOff + c) * 4u + l;
    cursor.assign(hRows.begin(), hRows.end() - 1);
    for (uint32_t h = 0; h < sc.H; ++h)
      for (uint32_t l = 0; l < 4; ++l)
        incidence[hingeBase + cursor[cl->hinge_indices[4ull * h + l]]++] = (sc.hOff + h) * 4u + l;
  });
  // IPC candidates (packIpcContactBuffer and packIpcIncidentCandidateAdjacency,
  // ipc-contact-layout.ts:190-342, in this engine's layout): global vertex
  // indices with the edge-edge type in bit 31 of the fourth, the scene of each
  // candidate, and per vertex its incident candidates in ascending order.
  const uint32_t nK = sp->KC;
  std::vector<uint4> contactIdx(nK);
  std::vector<uint32_t> contactScene(nK);
  std::vector<uint2> contactRange(nK ? nV : 0, make_uint2(0u, 0u));
  std::vector<uint32_t> contactIds(4ull * nK);
  if (nK) parallelFor(S, [&](uint32_t i) {
    const jgs2_input* in = prep[i].in;
    const SceneHost& sc = sp->scenes[i];
    if (sc.KC == 0) return;
    const uint32_t nvt = in->contact_vertex_triangle_count;
    std::vector<uint32_t> rows(sc.V + 1, 0);
    for (uint32_t c = 0; c < sc.KC; ++c) {
      const uint32_t* q = &in->contact_indices[4ull * c];
      contactIdx[sc.kOff + c] = make_uint4(sc.vOff + q[0], sc.vOff + q[1], sc.vOff + q[2],
                                           (sc.vOff + q[3]) | (c < nvt ? 0u : 0x80000000u));
      contactScene[sc.kOff + c] = i;
      for (int l = 0; l < 4; ++l) rows[q[l] + 1]++;
    }
    for (uint32_t v = 0; v < sc.V; ++v) rows[v + 1] += rows[v];
    const uint32_t base = 4u * sc.kOff;
    for (uint32_t v = 0; v < sc.V; ++v) contactRange[sc.vOff + v] = make_uint2(base + rows[v], rows[v + 1] - rows[v]);
    std::vector<uint32_t> cursor(rows.begin(), rows.end() - 1);
    for (uint32_t c = 0; c < sc.KC; ++c)
      for (int l = 0; l < 4; ++l) contactIds[base + cursor[in->contact_indices[4ull * c + l]]++] = sc.kOff + c;
  });
  // Contact surfaces: triangles (global vertices, scene) and edges in each
  // scene's canonical order, per vertex its one-ring, and the rows: per
  // vertex of the scene against its triangles, per edge against its later
  // edges, in the superset's order.
  std::vector<uint4> bpRowsH(bpR), bpTrisH(bpT);
  std::vector<uint2> bpEdgesH(bpE), bpRingH(sp->dynamic ? nV : 0, make_uint2(0u, 0u));
  std::vector<uint32_t> ringBase(S + 1, 0);
  for (uint32_t i = 0; i < S; ++i)
    ringBase[i + 1] = ringBase[i] + (prep[i].dynamic ? static_cast<uint32_t>(prep[i].surface.ring.size()) : 0u);
  std::vector<uint32_t> bpRingIdsH(ringBase[S]);
  if (sp->dynamic) parallelFor(S, [&](uint32_t i) {
    const SceneHost& sc = sp->scenes[i];
    if (!sc.dynamic) return;
    const ContactSurface& cs = prep[i].surface;
    for (uint32_t t = 0; t < sc.bpTris; ++t)
      bpTrisH[sc.bpTriOff + t] = make_uint4(sc.vOff + cs.tris[t][0], sc.vOff + cs.tris[t][1], sc.vOff + cs.tris[t][2], i);
    for (uint32_t e = 0; e < sc.bpEdges; ++e)
      bpEdgesH[sc.bpEdgeOff + e] = make_uint2(sc.vOff + cs.edges[e][0], sc.vOff + cs.edges[e][1]);
    for (uint32_t v = 0; v < sc.V; ++v) {
      bpRingH[sc.vOff + v] = make_uint2(ringBase[i] + cs.ringStart[v], cs.ringStart[v + 1] - cs.ringStart[v]);
      bpRowsH[sc.bpRowOff + v] = make_uint4(sc.vOff + v, i, sc.bpTriOff, sc.bpTriOff + sc.bpTris);
    }
    for (size_t k = 0; k < cs.ring.size(); ++k) bpRingIdsH[ringBase[i] + k] = sc.vOff + cs.ring[k];
    for (uint32_t e = 0; e < sc.bpEdges; ++e)
      bpRowsH[sc.bpRowOff + sc.V + e] =
          make_uint4(sc.bpEdgeOff + e, i | 0x80000000u, sc.bpEdgeOff + e + 1, sc.bpEdgeOff + sc.bpEdges);
  });
  // Segmented reduction tables: each scene's elements in fixed chunks.
  std::vector<jgs2::SceneRange> ranges(S);
  std::vector<jgs2::RedBlock> gateTable, convTable;
  for (uint32_t i = 0; i < S; ++i) {
    const SceneHost& sc = sp->scenes[i];
    jgs2::SceneRange& r = ranges[i];
    r.vOff = sc.vOff; r.V = sc.V; r.tOff = sc.tOff; r.T = sc.T;
    r.cOff = sc.cOff; r.C = sc.C; r.hOff = sc.hOff; r.H = sc.H;
    r.kOff = sc.kOff; r.KC = sc.KC;
    r.rowOff = sc.bpRowOff; r.rowCount = sc.dynamic ? sc.bpRows : 0u;
    // A contact-surface scene's gate also takes its listed candidates: the
    // table covers half the list capacity (blocks past the listed count
    // only join the reduction), more stride over it.
    const uint32_t listed = sc.dynamic ? static_cast<uint32_t>(sc.bpCapacity / 2) : 0u;
    const uint32_t n = std::max(std::max(std::max(sc.V, sc.T), std::max(sc.C, sc.H)), std::max(sc.KC, listed));
    r.gateSpan = std::max(n, 1u);
    r.gateBase = static_cast<uint32_t>(gateTable.size());
    for (uint32_t b0 = 0; b0 < std::max(n, 1u); b0 += jgs2::kGateChunk)
      gateTable.push_back({i, b0, std::min(n, b0 + jgs2::kGateChunk), static_cast<uint32_t>(gateTable.size())});
    r.gateBlocks = static_cast<uint32_t>(gateTable.size()) - r.gateBase;
    r.convBase = static_cast<uint32_t>(convTable.size());
    for (uint32_t b0 = 0; b0 < std::max(sc.V, 1u); b0 += jgs2::kConvChunk)
      convTable.push_back({i, b0, std::min(sc.V, b0 + jgs2::kConvChunk), static_cast<uint32_t>(convTable.size())});
    r.convBlocks = static_cast<uint32_t>(convTable.size()) - r.convBase;
  }

  jgs2_status st = JGS2_OK;
  Buffers& b = sp->b;
#define STEP(x) do { st = (x); if (st != JGS2_OK) return bail(st); } while (0)
  STEP(upload(sp, &b.pos[0], pos.data(), nV));
  STEP(upload(sp, &b.pos[1], pos.data(), nV));
  STEP(upload(sp, &b.predicted, pos.data(), nV));
  STEP(upload(sp, &b.old, pos.data(), nV));
  STEP(upload(sp, &b.velocity, vel.data(), nV));
  {
    std::vector<float4> identity(3ull * nV);
    for (uint32_t v = 0; v < nV; ++v) {
#if defined(JGS2_FRAME_QUAT) && JGS2_FRAME_QUAT
      identity[3ull * v] = make_float4(0, 0, 0, 1);  // the identity quaternion
#else
      identity[3ull * v] = make_float4(1, 0, 0, 0);
#endif
      identity[3ull * v + 1] = make_float4(0, 1, 0, 0);
      identity[3ull * v + 2] = make_float4(0, 0, 1, 0);
    }
    STEP(upload(sp, &b.vertexRot, identity.data(), 3ull * nV));
  }
  b.tetRot = nullptr;
  STEP(deviceAlloc(sp, &b.finalUpdate, nV));
  STEP(deviceAlloc(sp, &b.local, 4ull * nV));
  STEP(deviceAlloc(sp, &b.incident, 3ull * nV));
  CUDA_TRY(sp, cudaMemsetAsync(b.finalUpdate, 0, sizeof(float) * nV, sp->stream));
  CUDA_TRY(sp, cudaMemsetAsync(b.local, 0, sizeof(float4) * 4ull * nV, sp->stream));
  CUDA_TRY(sp, cudaMemsetAsync(b.incident, 0, sizeof(float4) * 3ull * nV, sp->stream));
  {
    FrameState fs;
    std::memset(&fs, 0, sizeof(fs));
    fs.localNumericsValid = 1;
    std::vector<FrameState> frames(S, fs);
    STEP(upload(sp, &b.frames, frames.data(), S));
  }
  b.gateBlocks = static_cast<uint32_t>(gateTable.size());
  b.convBlocks = static_cast<uint32_t>(convTable.size());
  b.sceneCount = S;
  b.vertexTotal = static_cast<uint32_t>(V);
  b.tetTotal = static_cast<uint32_t>(T);
  {
    double* gp = nullptr;
    double* cp = nullptr;
    STEP(deviceAlloc(sp, &gp, jgs2::kGatePartialBytes / sizeof(double) * b.gateBlocks));
    STEP(deviceAlloc(sp, &cp, jgs2::kConvPartialBytes / sizeof(double) * b.convBlocks));
    b.gatePartials = gp;
    b.convPartials = cp;
    jgs2::RedBlock* gt = nullptr;
    jgs2::RedBlock* ct = nullptr;
    STEP(upload(sp, &gt, gateTable.data(), gateTable.size()));
    STEP(upload(sp, &ct, convTable.data(), convTable.size()));
    b.gateTable = gt;
    b.convTable = ct;
    jgs2::SceneRange* rg = nullptr;
    STEP(upload(sp, &rg, ranges.data(), ranges.size()));
    b.scenes = rg;
    uint32_t* vs = nullptr;
    STEP(upload(sp, &vs, vertexScene.data(), vertexScene.size()));
    b.vertexScene = vs;
  }
  STEP(deviceAlloc(sp, &b.bodyAccum, 6ull * sp->bodies));
  {
    float4* p = nullptr;
    STEP(upload(sp, &p, rest.data(), nV));
    b.restMass = p;
    uint4* q = nullptr;
    STEP(upload(sp, &q, info.data(), nV));
    b.vinfo = q;
    float4* tt = nullptr;
    STEP(upload(sp, &tt, tets.data(), 4ull * nT));
    b.tets = tt;
    uint32_t* a = nullptr;
    STEP(upload(sp, &a, adjacency.data(), adjacency.size()));
    b.adjacency = a;
    uint4* ch = nullptr;
    STEP(upload(sp, &ch, head.data(), 2 * R));
    b.cubHead = ch;
    float4* cb = nullptr;
    STEP(upload(sp, &cb, reinterpret_cast<const float4*>(basis.data()), 9 * R));
    b.cubBasis = cb;
    b.stiffness = nullptr;
    float4* df = nullptr;
    float4* dt = nullptr;
    STEP(deviceAlloc(sp, &df, nV));
    STEP(deviceAlloc(sp, &dt, nV));
    b.forces = df;
    b.targets = dt;
    CUDA_TRY(sp, cudaMallocHost(reinterpret_cast<void**>(&sp->hForces), sizeof(float4) * std::max<size_t>(1, nV)));
    CUDA_TRY(sp, cudaMallocHost(reinterpret_cast<void**>(&sp->hTargets), sizeof(float4) * std::max<size_t>(1, nV)));
    CUDA_TRY(sp, cudaEventCreateWithFlags(&sp->objectiveUpload, cudaEventDisableTiming));
    CUDA_TRY(sp, cudaEventCreateWithFlags(&sp->readDone, cudaEventDisableTiming));
    std::memcpy(sp->hForces, initialForces.data(), sizeof(float4) * nV);
    std::memcpy(sp->hTargets, initialTargets.data(), sizeof(float4) * nV);
    CUDA_TRY(sp, cudaMemcpyAsync(df, sp->hForces, sizeof(float4) * nV, cudaMemcpyHostToDevice, sp->stream));
    CUDA_TRY(sp, cudaMemcpyAsync(dt, sp->hTargets, sizeof(float4) * nV, cudaMemcpyHostToDevice, sp->stream));
    CUDA_TRY(sp, cudaEventRecord(sp->objectiveUpload, sp->stream));
    sp->objectiveUploadPending = true;
    uint32_t* cl = nullptr;
    STEP(upload(sp, &cl, colors.data(), nV));
    b.colors = cl;
    b.clothTris = b.clothHinges = nullptr;
    b.clothRange = nullptr;
    b.clothIncidence = nullptr;
    if (anyCloth) {
      float4* ct = nullptr;
      float4* ch = nullptr;
      uint4* cr = nullptr;
      uint32_t* ci = nullptr;
      STEP(upload(sp, &ct, clothTris.data(), clothTris.size()));
      STEP(upload(sp, &ch, clothHinges.data(), clothHinges.size()));
      STEP(upload(sp, &cr, clothRange.data(), clothRange.size()));
      STEP(upload(sp, &ci, incidence.data(), incidence.size()));
      b.clothTris = ct;
      b.clothHinges = ch;
      b.clothRange = cr;
      b.clothIncidence = ci;
    }
    b.contactIdx = nullptr;
    b.contactScene = nullptr;
    b.contactState = nullptr;
    b.contactRange = nullptr;
    b.contactIds = nullptr;
    b.activeCount = nullptr;
    b.activeIds = nullptr;
    b.contactFlag = nullptr;
    b.contactGrad = nullptr;
    b.contactCount = nK;
    if (nK) {
      uint4* ki = nullptr;
      uint32_t* ks = nullptr;
      uint2* kr = nullptr;
      uint32_t* kd = nullptr;
      STEP(upload(sp, &ki, contactIdx.data(), nK));
      STEP(upload(sp, &ks, contactScene.data(), nK));
      STEP(upload(sp, &kr, contactRange.data(), nV));
      STEP(upload(sp, &kd, contactIds.data(), contactIds.size()));
      // Empty contact caches (distance -1), zero lagged records, neutral
      // scratch (packIpcContactBuffer, ipc-contact-layout.ts:290-340).
      std::vector<float4> state(7ull * nK, make_float4(0.f, 0.f, 0.f, 0.f));
      for (size_t c = 0; c < nK; ++c) {
        state[7 * c + 0] = make_float4(0.f, 0.f, 0.f, -1.f);
        state[7 * c + 2] = make_float4(0.f, 0.f, 0.f, -1.f);
        state[7 * c + 6] = make_float4(1.f, 0.f, 0.f, 0.f);
      }
      STEP(upload(sp, &b.contactState, state.data(), state.size()));
      STEP(deviceAlloc(sp, &b.activeCount, nV));
      STEP(deviceAlloc(sp, &b.activeIds, contactIds.size()));
      STEP(deviceAlloc(sp, &b.contactFlag, nK));
      STEP(deviceAlloc(sp, &b.contactGrad, nV));
      CUDA_TRY(sp, cudaMemsetAsync(b.activeCount, 0, sizeof(uint32_t) * nV, sp->stream));
      CUDA_TRY(sp, cudaMemsetAsync(b.contactFlag, 0, sizeof(uint32_t) * nK, sp->stream));
      CUDA_TRY(sp, cudaMemsetAsync(b.contactGrad, 0, sizeof(float4) * nV, sp->stream));
      b.contactIdx = ki;
      b.contactScene = ks;
      b.contactRange = kr;
      b.contactIds = kd;
    }
    b.contactDynamic = sp->dynamic ? 1u : 0u;
    if (sp->dynamic) {
      // Device broad phase: static surface data, per-iteration boxes, two
      // candidate lists, the sort's buffers and the status words.
      const uint64_t cap = sp->bpCapacity;
      b.contactCount = static_cast<uint32_t>(cap);
      b.bpRowTotal = static_cast<uint32_t>(bpR);
      b.bpTriTotal = static_cast<uint32_t>(bpT);
      b.bpEdgeTotal = static_cast<uint32_t>(bpE);
      b.bpSentinel = nV;
      b.bpSortPasses = jgs2::broadPhaseSortPasses(nV);
      uint64_t superset = 0;
      for (const SceneHost& sc : sp->scenes) superset += sc.bpSuperset;
      b.bpSuperset = static_cast<uint32_t>(std::min<uint64_t>(superset, 0xffffffffull));
      uint4* rows = nullptr;
      uint4* tris = nullptr;
      uint2* edges = nullptr;
      uint2* ring = nullptr;
      uint32_t* ringIds = nullptr;
      STEP(upload(sp, &rows, bpRowsH.data(), bpRowsH.size()));
      STEP(upload(sp, &tris, bpTrisH.data(), bpTrisH.size()));
      STEP(upload(sp, &edges, bpEdgesH.data(), bpEdgesH.size()));
      STEP(upload(sp, &ring, bpRingH.data(), bpRingH.size()));
      STEP(upload(sp, &ringIds, bpRingIdsH.data(), bpRingIdsH.size()));
      b.bpRows = rows;
      b.bpTris = tris;
      b.bpEdges = edges;
      b.bpRing = ring;
      b.bpRingIds = ringIds;
      STEP(deviceAlloc(sp, &b.bpTriBox, 2 * bpT));
      STEP(deviceAlloc(sp, &b.bpEdgeBox, 2 * bpE));
      STEP(deviceAlloc(sp, &b.bpTriChunk, 2 * ((bpT + 31) / 32)));
      STEP(deviceAlloc(sp, &b.bpEdgeChunk, 2 * ((bpE + 31) / 32)));
      STEP(deviceAlloc(sp, &b.bpTriSuper, 2 * ((bpT + 1023) / 1024)));
      STEP(deviceAlloc(sp, &b.bpEdgeSuper, 2 * ((bpE + 1023) / 1024)));
      for (int l = 0; l < 2; ++l) {
        STEP(deviceAlloc(sp, &sp->dynIdx[l], cap));
        STEP(deviceAlloc(sp, &sp->dynScene[l], cap));
        STEP(deviceAlloc(sp, &sp->dynState[l], 7 * cap));
        STEP(deviceAlloc(sp, &sp->dynFlag[l], cap));
        STEP(deviceAlloc(sp, &sp->dynCols[l], cap));
        STEP(deviceAlloc(sp, &sp->dynRowOff[l], bpR + 1));
        CUDA_TRY(sp, cudaMemsetAsync(sp->dynRowOff[l], 0, sizeof(uint32_t) * (bpR + 1), sp->stream));
        STEP(deviceAlloc(sp, &b.bpKeys[l], 4 * cap));
        STEP(deviceAlloc(sp, &b.bpVals[l], 4 * cap));
      }
      STEP(deviceAlloc(sp, &b.bpHist, 256 * ((4 * cap + 4095) / 4096) + 256));
      STEP(deviceAlloc(sp, &b.bpPinnedMove, nV));
      STEP(deviceAlloc(sp, &b.bpPrev, cap));
      STEP(deviceAlloc(sp, &b.bpSpan, S));
      STEP(deviceAlloc(sp, &b.bpStatus, 4));
      CUDA_TRY(sp, cudaMemsetAsync(b.bpStatus, 0, sizeof(uint32_t) * 4, sp->stream));
      CUDA_TRY(sp, cudaMemsetAsync(b.bpSpan, 0, sizeof(uint2) * S, sp->stream));
      STEP(deviceAlloc(sp, &b.contactRange, nV));
      STEP(deviceAlloc(sp, &b.activeCount, nV));
      STEP(deviceAlloc(sp, &b.contactGrad, nV));
      CUDA_TRY(sp, cudaMemsetAsync(b.activeCount, 0, sizeof(uint32_t) * nV, sp->stream));
      CUDA_TRY(sp, cudaMemsetAsync(b.contactGrad, 0, sizeof(float4) * nV, sp->stream));
      // The first list view; encodeFrame points each iteration at its own.
      b.contactIdx = sp->dynIdx[0];
      b.contactScene = sp->dynScene[0];
      b.contactState = sp->dynState[0];
      b.contactFlag = sp->dynFlag[0];
      b.bpCols = sp->dynCols[0];
      b.bpRowOff = sp->dynRowOff[0];
      b.activeIds = b.bpVals[b.bpSortPasses & 1u];
    }
    STEP(upload(sp, &sp->dColorVertices, byColor.data(), byColor.size()));
    STEP(upload(sp, &sp->dNeedVertices, need.data(), need.size()));
    STEP(upload(sp, &sp->dColorOffsets, sp->colorOffsets.data(), sp->colorOffsets.size()));
    STEP(upload(sp, &sp->dNeedOffsets, sp->needOffsets.data(), sp->needOffsets.size()));
    {
      uint32_t* bar = nullptr;
      STEP(deviceAlloc(sp, &bar, (jgs2::sweepBarrierBytes() + 3) / 4));
      CUDA_TRY(sp, cudaMemsetAsync(bar, 0, jgs2::sweepBarrierBytes(), sp->stream));
      sp->dSweepBarrier = bar;
    }
    STEP(deviceAlloc(sp, &sp->dParams, S));
    sp->hParams.resize(S);
    if (!sp->glob) {
      // Co-rotated path: tet frames, the 144-float rest stiffness of each tet
      // and each tet's scene.
      STEP(deviceAlloc(sp, &b.tetRot, 3ull * nT));
      std::vector<float> stiff(144ull * nT);
      std::vector<uint32_t> tetScene(nT);
      parallelFor(S, [&](uint32_t i) {
        const SceneHost& sc = sp->scenes[i];
        std::memcpy(&stiff[144ull * sc.tOff], prep[i].in->tet_rest_stiffness, sizeof(float) * 144ull * sc.T);
        std::fill(tetScene.begin() + sc.tOff, tetScene.begin() + sc.tOff + sc.T, i);
      });
      float* k = nullptr;
      STEP(upload(sp, &k, stiff.data(), stiff.size()));
      b.stiffness = k;
      uint32_t* ts = nullptr;
      STEP(upload(sp, &ts, tetScene.data(), tetScene.size()));
      b.tetScene = ts;
    }
  }
#undef STEP
  for (uint32_t i = 0; i < S; ++i) sp->hParams[i] = makeParams(sp, i, sp->scenes[i].defaults, false);
  if (!sp->glob) {
    CUDA_TRY(sp, cudaStreamSynchronize(sp->stream));
    return JGS2_OK;
  }
  // GPU preflight of the uploaded pose (validateGpuInitialStableSource,
  // jgs2-solver.ts:820-893): the gate on (posA, posA) must accept in every scene.
  CUDA_TRY(sp, cudaMemcpyAsync(sp->dParams, sp->hParams.data(), sizeof(DevParams) * S, cudaMemcpyHostToDevice,
                               sp->stream));
  jgs2::launchGate(b, sp->dParams, b.pos[0], b.pos[0], sp->stream);
  sp->launches += 1;
  std::vector<FrameState> frames(S);
  CUDA_TRY(sp, cudaMemcpyAsync(frames.data(), b.frames, sizeof(FrameState) * S, cudaMemcpyDeviceToHost, sp->stream));
  ce = cudaStreamSynchronize(sp->stream);
  if (ce != cudaSuccess) { cudaFail(sp, ce, "preflight"); return bail(JGS2_DEVICE_ERROR); }
  for (uint32_t i = 0; i < S; ++i) {
    const float4* control = frames[i].control;
    const uint32_t required = 1u | 2u | 4u;
    const float vb = control[0].w;
    const bool ok = std::isfinite(control[0].x) && std::isfinite(control[0].y) && std::isfinite(control[0].z) &&
                    control[0].x > kDeterminantFloor && control[0].y > kDeterminantFloor &&
                    control[0].z > kDeterminantFloor && vb == std::floor(vb) &&
                    ((static_cast<uint32_t>(vb) & required) == required);
    if (!ok) {
      sp->error = format("The uploaded stable Neo-Hookean source pose%s is not feasible under the production GPU "
                         "f32 determinant calculation; source J=%g, candidate J=%g, accepted J=%g.",
                         S > 1 ? format(" of scene %u", i).c_str() : "", control[0].x, control[0].y, control[0].z);
      return bail(JGS2_INFEASIBLE_INPUT);
    }
  }
  return JGS2_OK;
}

jgs2_status readSceneVec4(Engine* s, uint32_t scene, const float4* dev, float* out, size_t floats,
                          size_t perVertex) {
  const SceneHost& sc = s->scenes[scene];
  if (!out || floats < perVertex * sc.V)
    return fail(s, JGS2_INVALID_ARGUMENT, format("output needs %zu floats.", perVertex * sc.V));
  return readRegion(s, dev + (perVertex / 4) * sc.vOff, sizeof(float) * perVertex * sc.V, out);
}

jgs2_status readSceneGlobalization(Engine* s, uint32_t scene, float* local, size_t localFloats, float* control,
                                   float* history, size_t historyFloats, uint32_t* historyCount) {
  const SceneHost& sc = s->scenes[scene];
  if (!sc.recordsAvailable)
    return fail(s, JGS2_NOT_READY,
                "Globalization diagnostics are unavailable until a stable nonlinear iteration or diagnostic test "
                "kernel has produced records.");
  jgs2_status st = JGS2_OK;
  if (local) {
    if (localFloats < 16ull * sc.V) return fail(s, JGS2_INVALID_ARGUMENT, "local output too small.");
    st = readRegion(s, s->b.local + 4ull * sc.vOff, sizeof(float) * 16ull * sc.V, local);
    if (st != JGS2_OK) return st;
  }
  float4 ctl[4];
  st = readRegion(s, s->b.frames[scene].control, sizeof(ctl), ctl);
  if (st != JGS2_OK) return st;
  if (control) std::memcpy(control, ctl, sizeof(ctl));
  const float raw = ctl[1].w;
  if (!(raw >= 0 && raw <= float(JGS2_HISTORY_CAPACITY) && raw == std::floor(raw)))
    return fail(s, JGS2_DEVICE_ERROR, format("GPU returned invalid globalization history count %g.", raw));
  const uint32_t count = static_cast<uint32_t>(raw);
  if (historyCount) *historyCount = count;
  if (history) {
    if (historyFloats < 32ull * JGS2_HISTORY_CAPACITY) return fail(s, JGS2_INVALID_ARGUMENT, "history output too small.");
    st = readRegion(s, s->b.frames[scene].history, sizeof(float) * 32ull * JGS2_HISTORY_CAPACITY, history);
    if (st != JGS2_OK) return st;
  }
  return JGS2_OK;
}

jgs2_status sceneInfo(Engine* s, uint32_t scene, jgs2_info* out) {
  const SceneHost& sc = s->scenes[scene];
  std::memset(out, 0, sizeof(*out));
  out->vertex_count = sc.V;
  out->tet_count = sc.T;
  out->cubature_k = sc.K;
  out->body_count = sc.bodies;
  out->schedule_color_count = sc.colorCount;
  out->globalization_enabled = s->glob ? 1 : 0;
  out->objective_flags = sc.objectiveFlags;
  out->external_force_vertex_count = sc.forceCount;
  out->quadratic_target_vertex_count = sc.targetCount;
  out->objective_revision = sc.objectiveRevision;
  out->last_submitted_iterations = sc.submittedIterations;
  out->scene_scale = sc.sceneScale;
  out->preprocessing_timestep = sc.preprocessingTimestep;
  out->current_position_buffer = 0;
  out->cloth_triangle_count = sc.C;
  out->contact_candidate_count = sc.KC;
  out->contact_candidate_capacity = 0;
  if (sc.dynamic) {
    // The scene's span of the last iteration's list.
    out->contact_candidate_capacity = static_cast<uint32_t>(sc.bpCapacity);
    uint2 span = make_uint2(0u, 0u);
    if (sc.submittedIterations && readRegion(s, s->b.bpSpan + scene, sizeof(span), &span) == JGS2_OK)
      out->contact_candidate_count = span.y;
  }
  if (sc.recordsAvailable) {
    float4 c1;
    if (readRegion(s, &s->b.frames[scene].control[1], sizeof(c1), &c1) == JGS2_OK)
      out->history_count = static_cast<uint32_t>(c1.w);
  }
  return JGS2_OK;
}

}  // namespace

extern "C" {

uint32_t jgs2_version(void) { return JGS2_ABI_VERSION; }

const char* jgs2_build_string(void) {
  return "jgs2-b200 sm_100a (CUDA " __DATE__ ")";
}

const char* jgs2_global_last_error(void) { return gGlobalError.c_str(); }

void jgs2_default_settings(jgs2_settings* out) {
  if (out) defaults(out);
}

jgs2_status jgs2_resolve_settings(const jgs2_settings* base, const jgs2_settings* overrides, uint32_t mask,
                                  jgs2_settings* out) {
  if (!out) return fail(nullptr, JGS2_INVALID_ARGUMENT, "out is NULL.");
  jgs2_settings d;
  defaults(&d);
  std::string err;
  if (!resolve(base ? *base : d, overrides, mask, out, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  return JGS2_OK;
}

jgs2_status jgs2_validate_input(const jgs2_input* input) {
  std::string err;
  if (!validateInput(input, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  return JGS2_OK;
}

jgs2_status jgs2_minimum_contact_distance(const jgs2_input* input, double cutoff, double* distance) {
  std::string err;
  if (!validateInput(input, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  if (!distance) return fail(nullptr, JGS2_INVALID_ARGUMENT, "distance is NULL.");
  if (!(cutoff >= 0)) return fail(nullptr, JGS2_INVALID_ARGUMENT, "cutoff must be nonnegative.");
  if (input->contact_surface) {
    ContactSurface cs;
    buildContactSurface(input, &cs);
    *distance = surfaceContactDistance(input, cs, cutoff);
  } else {
    const uint64_t nc = uint64_t(input->contact_vertex_triangle_count) + input->contact_edge_edge_count;
    *distance = nc ? staticContactDistance(input) : INFINITY;
  }
  return JGS2_OK;
}

jgs2_status jgs2_evaluate_contact_features(const float* points, const uint32_t* types, uint32_t count, float* out,
                                           uint32_t* fp64_used, int device) {
  if (count == 0) return JGS2_OK;
  if (!points || !types || !out) return fail(nullptr, JGS2_INVALID_ARGUMENT, "points, types and out must not be NULL.");
  for (uint32_t i = 0; i < count; ++i)
    if (types[i] > 1u) return fail(nullptr, JGS2_INVALID_ARGUMENT, format("types[%u] must be 0 or 1.", i));
  if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, JGS2_DEVICE_ERROR, "cudaSetDevice failed.");
  float* dPoints = nullptr;
  float* dOut = nullptr;
  uint32_t* dTypes = nullptr;
  uint32_t* dWide = nullptr;
  cudaError_t e = cudaMalloc(&dPoints, sizeof(float) * 12ull * count);
  if (e == cudaSuccess) e = cudaMalloc(&dOut, sizeof(float) * 9ull * count);
  if (e == cudaSuccess) e = cudaMalloc(&dTypes, sizeof(uint32_t) * count);
  if (e == cudaSuccess) e = cudaMalloc(&dWide, sizeof(uint32_t) * count);
  if (e == cudaSuccess) e = cudaMemcpy(dPoints, points, sizeof(float) * 12ull * count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dTypes, types, sizeof(uint32_t) * count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    jgs2::launchContactFeatures(dPoints, dTypes, count, dOut, dWide, nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dOut, sizeof(float) * 9ull * count, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && fp64_used) e = cudaMemcpy(fp64_used, dWide, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost);
  cudaFree(dPoints);
  cudaFree(dOut);
  cudaFree(dTypes);
  cudaFree(dWide);
  if (e != cudaSuccess)
    return fail(nullptr, JGS2_DEVICE_ERROR, format("contact feature evaluation: %s", cudaGetErrorString(e)));
  return JGS2_OK;
}

jgs2_status jgs2_contact_superset_size(const jgs2_input* input, uint64_t* count) {
  std::string err;
  if (!validateInput(input, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  if (!count) return fail(nullptr, JGS2_INVALID_ARGUMENT, "count is NULL.");
  if (!input->contact_surface) return fail(nullptr, JGS2_INVALID_ARGUMENT, "The input has no contact surface.");
  ContactSurface cs;
  buildContactSurface(input, &cs);
  *count = cs.superset;
  return JGS2_OK;
}

jgs2_status jgs2_build_vertex_coloring(const jgs2_input* input, uint32_t* colors, uint32_t* count) {
  std::string err;
  if (!validateInput(input, &err)) return fail(nullptr, JGS2_INVALID_ARGUMENT, err);
  if (!colors || !count) return fail(nullptr, JGS2_INVALID_ARGUMENT, "output is NULL.");
  const auto c = colorInput(input, count);
  std::memcpy(colors, c.data(), c.size() * sizeof(uint32_t));
  return JGS2_OK;
}

jgs2_status jgs2_create(const jgs2_input* in, const jgs2_settings* settings, uint32_t mask, int device,
                        jgs2_solver** out) {
  if (!out) return fail(nullptr, JGS2_INVALID_ARGUMENT, "out is NULL.");
  *out = nullptr;
  std::vector<PreparedScene> prep(1);
  jgs2_status st = prepareScene(in, settings, mask, true, &prep[0]);
  if (st != JGS2_OK) return st;
  std::unique_ptr<jgs2_solver> s(new jgs2_solver());
  st = buildEngine(s.get(), prep, device);
  if (st != JGS2_OK) return st;
  *out = s.release();
  return JGS2_OK;
}

void jgs2_destroy(jgs2_solver* s) {
  if (!s) return;
  if (!s->destroyed) {
    cudaSetDevice(s->device);
    releaseDevice(s);
    s->destroyed = true;
  }
  delete s;
}

const char* jgs2_last_error(const jgs2_solver* s) { return s ? s->error.c_str() : gGlobalError.c_str(); }

jgs2_status jgs2_get_info(jgs2_solver* s, jgs2_info* out) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  return sceneInfo(s, 0, out);
}

jgs2_status jgs2_get_default_settings(jgs2_solver* s, jgs2_settings* out) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  *out = s->scenes[0].defaults;
  return JGS2_OK;
}

jgs2_status jgs2_get_last_submitted_settings(jgs2_solver* s, jgs2_settings* out) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  *out = s->scenes[0].submitted;
  return JGS2_OK;
}

jgs2_status jgs2_step(jgs2_solver* s, const jgs2_settings* o, uint32_t mask) {
  return stepCommon(s, 1, -1, o, mask, false);
}

jgs2_status jgs2_step_frames(jgs2_solver* s, uint32_t frames, const jgs2_settings* o, uint32_t mask) {
  return stepCommon(s, frames, -1, o, mask, true);
}

jgs2_status jgs2_step_exact_iterations(jgs2_solver* s, uint32_t iterations, const jgs2_settings* o, uint32_t mask) {
  return stepCommon(s, 1, static_cast<int>(iterations), o, mask, false);
}

jgs2_status jgs2_step_frames_exact_iterations(jgs2_solver* s, uint32_t frames, uint32_t iterations,
                                              const jgs2_settings* o, uint32_t mask) {
  return stepCommon(s, frames, static_cast<int>(iterations), o, mask, true);
}

jgs2_status jgs2_step_with_gpu_timestamps(jgs2_solver* s, uint32_t frames, uint32_t iterations,
                                          const jgs2_settings* o, uint32_t mask, jgs2_kernel_profile* out) {
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  KernelProfiler prof;
  jgs2_status st = stepCommon(s, frames, static_cast<int>(iterations), o, mask, true, &prof);
  if (st != JGS2_OK) return st;
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  std::memset(out, 0, sizeof(*out));
  out->kinds = JGS2_PROFILE_KINDS;
  for (int k = 0; k < JGS2_PROFILE_KINDS; ++k)
    std::snprintf(out->names[k], sizeof(out->names[k]), "%s", KernelProfiler::kNames[k]);
  for (size_t i = 0; i < prof.used; ++i) {
    float ms = 0.f;
    CUDA_TRY(s, cudaEventElapsedTime(&ms, prof.pool[i].first, prof.pool[i].second));
    out->milliseconds[prof.kinds[i]] += ms;
    out->launches[prof.kinds[i]] += 1;
  }
  return JGS2_OK;
}

jgs2_status jgs2_sync(jgs2_solver* s) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return checkBroadPhase(s);
}

jgs2_status jgs2_read_oracle_diagnostics(jgs2_solver* s, jgs2_oracle_diagnostics* out, float* vertexRecords,
                                         size_t vertexFloats, float* tetRecords, size_t tetFloats) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  const SceneHost& sc = s->scenes[0];
  const jgs2_settings& set = sc.submitted;
  if ((sc.KC > 0 || sc.dynamic) && set.ipc_barrier_stiffness > 0)
    return fail(s, JGS2_UNSUPPORTED,
                "Exact oracle diagnostics do not yet include IPC contact energy; disable IPC before requesting "
                "this diagnostic.");
  if (vertexRecords && vertexFloats < 36ull * sc.V)
    return fail(s, JGS2_INVALID_ARGUMENT, "vertex_records holds fewer than 36 floats per vertex.");
  if (tetRecords && tetFloats < 4ull * sc.T)
    return fail(s, JGS2_INVALID_ARGUMENT, "tet_records holds fewer than 4 floats per tet.");
  CUDA_TRY(s, cudaSetDevice(s->device));
  if (!s->oracleSummary) {
    if ((st = deviceAlloc(s, &s->oracleTetRot, 3ull * std::max(1u, s->T))) != JGS2_OK) return st;
    if ((st = deviceAlloc(s, &s->oracleTetMetric, std::max(1u, s->T))) != JGS2_OK) return st;
    if ((st = deviceAlloc(s, &s->oracleVertex, 9ull * std::max(1u, s->V))) != JGS2_OK) return st;
    if ((st = deviceAlloc(s, &s->oracleSummary, jgs2::kOracleSummaryWords)) != JGS2_OK) return st;
  }
  jgs2::OracleParams q{};
  const double h = set.timestep;
  q.invDt2 = static_cast<float>(1.0 / (h * h));
  q.floorHeight = set.floor_height;
  q.floorStiffness = set.floor_stiffness;
  q.rotationEpsilon = set.rotation_epsilon;
  q.objectiveFlags = sc.objectiveFlags;
  q.vOff = sc.vOff;
  q.V = sc.V;
  q.tOff = sc.tOff;
  q.T = sc.T;
  q.corotated = s->glob ? 0u : 1u;
  jgs2::launchOracleDiagnostics(s->b, q, s->oracleTetRot, s->oracleTetMetric, s->oracleVertex, s->oracleSummary,
                                s->stream);
  CUDA_TRY(s, cudaGetLastError());
  double sum[jgs2::kOracleSummaryWords];
  st = readRegion(s, s->oracleSummary, sizeof(sum), sum);
  if (st != JGS2_OK) return st;
  if (vertexRecords) {
    st = readRegion(s, s->oracleVertex, sizeof(float) * 36ull * sc.V, vertexRecords);
    if (st != JGS2_OK) return st;
  }
  if (tetRecords) {
    st = readRegion(s, s->oracleTetMetric, sizeof(float) * 4ull * sc.T, tetRecords);
    if (st != JGS2_OK) return st;
  }
  // reduceDiagnostics' closing arithmetic (jgs2-diagnostics.ts:1040-1090).
  jgs2_oracle_diagnostics& d = *out;
  d = jgs2_oracle_diagnostics{};
  d.inertia = sum[0];
  d.elasticity = sum[1];
  d.external_force = sum[2];
  d.quadratic_target = sum[3];
  d.floor_contact = sum[4];
  d.energy = sum[0] + sum[1] + sum[2] + sum[3] + sum[4];
  d.gradient_squared_norm = sum[5];
  d.gradient_norm = std::sqrt(std::max(sum[5], 0.0));
  d.inertia_gradient_norm = std::sqrt(std::max(sum[6], 0.0));
  d.material_gradient_norm = std::sqrt(std::max(sum[7], 0.0));
  d.external_force_gradient_norm = std::sqrt(std::max(sum[8], 0.0));
  d.target_gradient_norm = std::sqrt(std::max(sum[9], 0.0));
  d.contact_gradient_norm = std::sqrt(std::max(sum[10], 0.0));
  d.active_vertex_count = static_cast<uint32_t>(sum[14]);
  d.gradient_valid = sum[14] > 0 ? 1u : 0u;
  d.minimum_deformation_determinant_valid = sc.T > 0 ? 1u : 0u;
  d.minimum_deformation_determinant = sc.T > 0 ? sum[12] : 0.0;
  d.maximum_update = sum[11];
  d.maximum_update_valid = (d.gradient_valid && sum[16] >= 0.5) ? 1u : 0u;
  const bool floorValid = set.floor_stiffness > 0 && d.gradient_valid;
  d.minimum_contact_distance_valid = floorValid ? 1u : 0u;
  d.minimum_contact_distance = floorValid ? sum[13] : 0.0;
  d.active_contact_count = floorValid ? static_cast<uint32_t>(sum[15]) : 0u;
  d.residual_denominator = std::max(1.0, d.inertia_gradient_norm + d.material_gradient_norm +
                                             d.external_force_gradient_norm + d.target_gradient_norm +
                                             d.contact_gradient_norm);
  d.relative_residual = d.gradient_norm / d.residual_denominator;
  bool finite = sum[17] >= 0.5;
  for (double v : {d.energy, d.gradient_norm, d.residual_denominator, d.relative_residual, d.maximum_update,
                   d.minimum_deformation_determinant, d.minimum_contact_distance})
    finite = finite && std::isfinite(v);
  d.finite = finite ? 1u : 0u;
  d.relative_residual_valid = (d.maximum_update_valid && finite) ? 1u : 0u;
  return JGS2_OK;
}

jgs2_status jgs2_read_contact_candidates(jgs2_solver* s, uint32_t* out, uint64_t capacity, uint64_t* count) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!count) return fail(s, JGS2_INVALID_ARGUMENT, "count is NULL.");
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  st = checkBroadPhase(s);
  if (st != JGS2_OK) return st;
  const SceneHost& sc = s->scenes[0];
  const uint4* list = s->b.contactIdx;
  uint64_t n = sc.KC;
  uint64_t first = sc.kOff;
  if (s->dynamic) {
    // The last iteration's list: the one its iteration count's parity picks.
    const uint32_t it = sc.submittedIterations;
    list = s->dynIdx[it ? static_cast<int>((it - 1) & 1u) : 0];
    uint32_t total = 0;
    CUDA_TRY(s, cudaMemcpy(&total, s->b.bpStatus, sizeof(total), cudaMemcpyDeviceToHost));
    n = sc.submittedIterations ? total : 0u;
    first = 0;
  }
  *count = n;
  if (!out || n == 0) return JGS2_OK;
  if (capacity < n) return fail(s, JGS2_INVALID_ARGUMENT, "out holds fewer candidates than were listed.");
  std::vector<uint4> host(n);
  CUDA_TRY(s, cudaMemcpy(host.data(), list + first, sizeof(uint4) * n, cudaMemcpyDeviceToHost));
  for (uint64_t c = 0; c < n; ++c) {
    out[4 * c] = host[c].x - sc.vOff;
    out[4 * c + 1] = host[c].y - sc.vOff;
    out[4 * c + 2] = host[c].z - sc.vOff;
    out[4 * c + 3] = ((host[c].w & 0x7fffffffu) - sc.vOff) | (host[c].w & 0x80000000u);
  }
  return JGS2_OK;
}

jgs2_status jgs2_set_external_force(jgs2_solver* s, uint32_t vertex, const float force[3]) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (vertex >= s->V) return fail(s, JGS2_INVALID_ARGUMENT, format("vertex %u is out of range.", vertex));
  if (!force) return fail(s, JGS2_INVALID_ARGUMENT, "force is NULL.");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(force[k]))
      return fail(s, JGS2_INVALID_ARGUMENT,
                  format("External force %d for vertex %u must be finite after f32 conversion.", k, vertex));
  if (s->pinned[vertex] && (force[0] != 0 || force[1] != 0 || force[2] != 0))
    return fail(s, JGS2_INVALID_ARGUMENT, format("Pinned vertex %u cannot have a nonzero external force.", vertex));
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  SceneHost& sc = s->scenes[0];
  float4& f = s->hForces[vertex];
  sc.forceCount -= forceActive(f) ? 1u : 0u;
  f = make_float4(force[0], force[1], force[2], 0.f);
  sc.forceCount += forceActive(f) ? 1u : 0u;
  return writeObjectives(s, 0, vertex, 1, true, false);
}

jgs2_status jgs2_replace_external_forces(jgs2_solver* s, const float* forces) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!forces) return fail(s, JGS2_INVALID_ARGUMENT, "forces is NULL.");
  // Checked and mirrored in chunks across host threads (a per-frame call on
  // million-vertex solvers); the first failing entry in vertex order is
  // reported, as a sequential pass would, and nothing is mirrored then.
  constexpr uint32_t kChunk = 1u << 16;
  const uint32_t chunks = (s->V + kChunk - 1) / kChunk;
  std::vector<uint64_t> firstBad(chunks, UINT64_MAX);  // 3 v + k, or (V + v) << 2 for a pinned vertex
  parallelFor(chunks, [&](uint32_t c) {
    for (uint32_t v = c * kChunk; v < std::min(s->V, (c + 1) * kChunk); ++v) {
      bool nonzero = false;
      for (int k = 0; k < 3; ++k) {
        if (!std::isfinite(forces[3ull * v + k])) {
          firstBad[c] = 3ull * v + k;
          return;
        }
        nonzero |= forces[3ull * v + k] != 0;
      }
      if (s->pinned[v] && nonzero) {
        firstBad[c] = (uint64_t(s->V) * 3 + v) << 2;
        return;
      }
    }
  });
  for (uint32_t c = 0; c < chunks; ++c) {
    if (firstBad[c] == UINT64_MAX) continue;
    if (firstBad[c] < 3ull * s->V)
      return fail(s, JGS2_INVALID_ARGUMENT, format("External forces[%llu] must be finite after f32 conversion.",
                                                   static_cast<unsigned long long>(firstBad[c])));
    const uint32_t v = static_cast<uint32_t>((firstBad[c] >> 2) - uint64_t(s->V) * 3);
    return fail(s, JGS2_INVALID_ARGUMENT, format("Pinned vertex %u cannot have a nonzero external force.", v));
  }
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  std::vector<uint32_t> active(chunks, 0u);
  parallelFor(chunks, [&](uint32_t c) {
    uint32_t n = 0;
    for (uint32_t v = c * kChunk; v < std::min(s->V, (c + 1) * kChunk); ++v) {
      const float4 f = make_float4(forces[3ull * v], forces[3ull * v + 1], forces[3ull * v + 2], 0.f);
      s->hForces[v] = f;
      n += forceActive(f) ? 1u : 0u;
    }
    active[c] = n;
  });
  uint32_t count = 0;
  for (uint32_t n : active) count += n;
  s->scenes[0].forceCount = count;
  return writeObjectives(s, 0, 0, s->V, true, false);
}

jgs2_status jgs2_clear_external_forces(jgs2_solver* s) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  std::vector<float> zeros(3ull * s->V, 0.f);
  return jgs2_replace_external_forces(s, zeros.data());
}

jgs2_status jgs2_set_quadratic_target(jgs2_solver* s, uint32_t vertex, const float target[3], float stiffness) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (vertex >= s->V) return fail(s, JGS2_INVALID_ARGUMENT, format("vertex %u is out of range.", vertex));
  if (!target) return fail(s, JGS2_INVALID_ARGUMENT, "target is NULL.");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(target[k]))
      return fail(s, JGS2_INVALID_ARGUMENT,
                  format("Quadratic target %d for vertex %u must be finite after f32 conversion.", k, vertex));
  if (!std::isfinite(stiffness))
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("Quadratic-target stiffness for vertex %u must be finite after f32 conversion.", vertex));
  if (stiffness < 0)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("Quadratic-target stiffness for vertex %u must be nonnegative.", vertex));
  if (s->pinned[vertex] && stiffness != 0)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("Pinned vertex %u cannot have a nonzero quadratic-target stiffness.", vertex));
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  SceneHost& sc = s->scenes[0];
  float4& t = s->hTargets[vertex];
  sc.targetCount -= t.w > 0 ? 1u : 0u;
  t = make_float4(target[0], target[1], target[2], stiffness);
  sc.targetCount += t.w > 0 ? 1u : 0u;
  return writeObjectives(s, 0, vertex, 1, false, true);
}

jgs2_status jgs2_replace_quadratic_targets(jgs2_solver* s, const float* positions, const float* stiffnesses) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!positions || !stiffnesses) return fail(s, JGS2_INVALID_ARGUMENT, "targets are NULL.");
  for (uint32_t v = 0; v < s->V; ++v) {
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(positions[3ull * v + k]))
        return fail(s, JGS2_INVALID_ARGUMENT,
                    format("Quadratic target positions[%llu] must be finite after f32 conversion.",
                           static_cast<unsigned long long>(3ull * v + k)));
    if (!std::isfinite(stiffnesses[v]))
      return fail(s, JGS2_INVALID_ARGUMENT,
                  format("Quadratic target stiffnesses[%u] must be finite after f32 conversion.", v));
    if (stiffnesses[v] < 0)
      return fail(s, JGS2_INVALID_ARGUMENT, format("Quadratic target stiffnesses[%u] must be nonnegative.", v));
    if (s->pinned[v] && stiffnesses[v] != 0)
      return fail(s, JGS2_INVALID_ARGUMENT,
                  format("Pinned vertex %u cannot have a nonzero quadratic-target stiffness.", v));
  }
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  uint32_t count = 0;
  for (uint32_t v = 0; v < s->V; ++v) {
    s->hTargets[v] = make_float4(positions[3ull * v], positions[3ull * v + 1], positions[3ull * v + 2], stiffnesses[v]);
    count += stiffnesses[v] > 0 ? 1u : 0u;
  }
  s->scenes[0].targetCount = count;
  return writeObjectives(s, 0, 0, s->V, false, true);
}

jgs2_status jgs2_release_quadratic_target(jgs2_solver* s, uint32_t vertex) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (vertex >= s->V) return fail(s, JGS2_INVALID_ARGUMENT, format("vertex %u is out of range.", vertex));
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  s->scenes[0].targetCount -= s->hTargets[vertex].w > 0 ? 1u : 0u;
  s->hTargets[vertex].w = 0.f;
  return writeObjectives(s, 0, vertex, 1, false, true);
}

jgs2_status jgs2_release_all_quadratic_targets(jgs2_solver* s) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  for (uint32_t v = 0; v < s->V; ++v) s->hTargets[v].w = 0.f;
  s->scenes[0].targetCount = 0;
  return writeObjectives(s, 0, 0, s->V, false, true);
}

jgs2_status jgs2_read_positions(jgs2_solver* s, float* out, size_t floats) {
  if (usable(s) != JGS2_OK) return usable(s);
  return readSceneVec4(s, 0, s->b.pos[0], out, floats, 4);
}

jgs2_status jgs2_read_positions_async(jgs2_solver* s, float* out, size_t floats) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out || floats < 4ull * s->V) return fail(s, JGS2_INVALID_ARGUMENT, format("output needs %u floats.", 4 * s->V));
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaMemcpyAsync(out, s->b.pos[0], sizeof(float4) * s->V, cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(s, cudaEventRecord(s->readDone, s->stream));
  return JGS2_OK;
}

jgs2_status jgs2_wait_reads(jgs2_solver* s) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaEventSynchronize(s->readDone));
  return checkBroadPhase(s);
}

jgs2_status jgs2_read_velocities(jgs2_solver* s, float* out, size_t floats) {
  if (usable(s) != JGS2_OK) return usable(s);
  return readSceneVec4(s, 0, s->b.velocity, out, floats, 4);
}

jgs2_status jgs2_read_predicted_positions(jgs2_solver* s, float* out, size_t floats) {
  if (usable(s) != JGS2_OK) return usable(s);
  const jgs2_status st = readSceneVec4(s, 0, s->b.predicted, out, floats, 4);
  if (st != JGS2_OK) return st;
  // The device copy keeps the distributed inertia weight in w.
  for (uint32_t v = 0; v < s->V; ++v) out[4ull * v + 3] = 1.0f;
  return JGS2_OK;
}

jgs2_status jgs2_read_final_iteration_updates(jgs2_solver* s, float* out, size_t floats) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out || floats < 4ull * s->V) return fail(s, JGS2_INVALID_ARGUMENT, format("output needs %u floats.", 4 * s->V));
  std::vector<float> u(s->V);
  st = readRegion(s, s->b.finalUpdate, sizeof(float) * s->V, u.data());
  if (st != JGS2_OK) return st;
  const float w = s->scenes[0].submittedIterations > 0 ? 1.f : 0.f;
  for (uint32_t v = 0; v < s->V; ++v) {
    out[4ull * v] = u[v];
    out[4ull * v + 1] = 0.f;
    out[4ull * v + 2] = 0.f;
    out[4ull * v + 3] = w;
  }
  return JGS2_OK;
}

jgs2_status jgs2_read_vertex_rotations(jgs2_solver* s, float* out, size_t floats) {
  if (usable(s) != JGS2_OK) return usable(s);
  return readSceneVec4(s, 0, s->b.vertexRot, out, floats, 12);
}

jgs2_status jgs2_read_globalization(jgs2_solver* s, float* local, size_t localFloats, float* control,
                                    float* history, size_t historyFloats, uint32_t* historyCount) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!s->glob)
    return fail(s, JGS2_UNSUPPORTED,
                "Globalization diagnostics are available only for stable Neo-Hookean production solves.");
  return readSceneGlobalization(s, 0, local, localFloats, control, history, historyFloats, historyCount);
}

jgs2_status jgs2_evaluate_assembled_candidate(jgs2_solver* s, const float* source, const float* candidate,
                                              const jgs2_settings* o, uint32_t mask, float* positionsOut,
                                              float* controlOut, float* historyOut) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!s->glob) return fail(s, JGS2_UNSUPPORTED, "Assembled candidate tests require stable globalization.");
  if (!source || !candidate) return fail(s, JGS2_INVALID_ARGUMENT, "Assembled candidate poses must not be NULL.");
  const size_t n = 4ull * s->V;
  for (size_t i = 0; i < n; ++i) {
    if (!std::isfinite(source[i])) return fail(s, JGS2_INVALID_ARGUMENT, "source candidate pose must be finite.");
    if (!std::isfinite(candidate[i]))
      return fail(s, JGS2_INVALID_ARGUMENT, "candidate candidate pose must be finite.");
  }
  jgs2_settings settings;
  std::string err;
  if (!resolve(s->scenes[0].defaults, o, mask, &settings, &err)) return fail(s, JGS2_INVALID_ARGUMENT, err);
  s->hParams[0] = makeParams(s, 0, settings, false);
  const Buffers& b = s->b;
  FrameState* fs = &b.frames[0];
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaMemcpyAsync(s->dParams, &s->hParams[0], sizeof(DevParams), cudaMemcpyHostToDevice, s->stream));
  // posB = source, posA = candidate, predicted = source; local records and
  // the control record cleared (jgs2-solver.ts:2644-2679).
  CUDA_TRY(s, cudaMemcpyAsync(b.pos[1], source, sizeof(float) * n, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaMemcpyAsync(b.pos[0], candidate, sizeof(float) * n, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaMemcpyAsync(b.predicted, source, sizeof(float) * n, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaMemsetAsync(b.local, 0, sizeof(float4) * 4ull * s->V, s->stream));
  CUDA_TRY(s, cudaMemsetAsync(fs->control, 0, sizeof(float4) * 4, s->stream));
  // The sweep aggregates the gate reads, as a cleared record per vertex
  // gives them: status 0 (accepted) with no backtracks and no evaluations,
  // i.e. one skipped trial per vertex and valid numerics.
  const uint32_t aggregates[6] = {0u, 0u, s->V, 0u, 0u, 1u};
  static_assert(offsetof(FrameState, localNumericsValid) - offsetof(FrameState, localFailures) == 20,
                "sweep aggregates are six consecutive words");
  CUDA_TRY(s, cudaMemcpyAsync(&fs->localFailures, aggregates, sizeof(aggregates), cudaMemcpyHostToDevice,
                              s->stream));
  s->launches += jgs2::launchGate(b, s->dParams, b.pos[1], b.pos[0], s->stream);
  s->launches += jgs2::launchConvergence(b, s->dParams, b.pos[1], b.pos[0], false, s->stream);
  CUDA_TRY(s, cudaGetLastError());
  SceneHost& sc = s->scenes[0];
  sc.recordsAvailable = true;
  sc.submitted = settings;
  sc.submittedIterations = 1;
  if (positionsOut) {
    st = readRegion(s, b.pos[0], sizeof(float) * n, positionsOut);
    if (st != JGS2_OK) return st;
  }
  if (controlOut) {
    st = readRegion(s, fs->control, sizeof(float4) * 4, controlOut);
    if (st != JGS2_OK) return st;
  }
  if (historyOut) {
    st = readRegion(s, fs->history, sizeof(float4) * 8, historyOut);
    if (st != JGS2_OK) return st;
  }
  return jgs2_sync(s);
}

// For callers that may not allocate device memory while they run: hosts that
// give the library a fixed device-memory budget up front, and per-frame loops
// where a device allocation would synchronise the device and stall the frame.
// The gate's scratch is a static device array whose address is looked up once
// per device; nothing here calls cudaMalloc or cudaFree.  The address cache
// below lives for the whole process and is keyed by device ordinal only: a
// device reset or a reload of this library in the same process would leave it
// stale, so neither is supported (the header says so).
jgs2_status jgs2_gate_candidate_no_alloc(jgs2_solver* s, const float* source, const float* candidate,
                                         const float* predicted, const jgs2_settings* o, uint32_t mask,
                                         float* control, void* stream) {
  constexpr int kMaxScratchDevices = 64;
  static std::mutex scratchMutex;
  static void* scratchAddress[kMaxScratchDevices] = {};
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!s->glob) return fail(s, JGS2_UNSUPPORTED, "The assembled gate requires stable globalization.");
  if (s->KC > 0 || s->dynamic)
    return fail(s, JGS2_UNSUPPORTED,
                "The no-allocation gate does not evaluate IPC contact energies; use "
                "jgs2_evaluate_assembled_candidate for solvers with contact candidates.");
  if (!source || !candidate || !predicted || !control)
    return fail(s, JGS2_INVALID_ARGUMENT, "The no-allocation gate's device arrays must not be NULL.");
  for (const void* p : {static_cast<const void*>(source), static_cast<const void*>(candidate),
                        static_cast<const void*>(predicted), static_cast<const void*>(control)})
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0)
      return fail(s, JGS2_INVALID_ARGUMENT, "The no-allocation gate's device arrays must be 16-byte aligned.");
  const uint32_t limit = jgs2::gateScratchMaxElements();
  if (std::max(std::max(s->V, s->T), std::max(s->C, s->H)) > limit)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("The no-allocation gate handles at most %u vertices, tetrahedra, cloth triangles and hinges "
                       "(its static scratch holds %u block partials); this solver has %u vertices, %u tetrahedra, "
                       "%u triangles and %u hinges.",
                       limit, jgs2::kGateScratchMaxBlocks, s->V, s->T, s->C, s->H));
  if (s->device < 0 || s->device >= kMaxScratchDevices)
    return fail(s, JGS2_UNSUPPORTED, format("The no-allocation gate supports device ordinals below %d.",
                                            kMaxScratchDevices));
  jgs2_settings settings;
  std::string err;
  if (!resolve(s->scenes[0].defaults, o, mask, &settings, &err)) return fail(s, JGS2_INVALID_ARGUMENT, err);
  const DevParams p = makeParams(s, 0, settings, false);
  CUDA_TRY(s, cudaSetDevice(s->device));
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(scratchMutex);
    if (!scratchAddress[s->device]) {
      void* address = nullptr;
      const cudaError_t e = jgs2::gateScratchAddress(&address);
      if (e != cudaSuccess || !address)
        return cudaFail(s, e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(gate scratch)");
      scratchAddress[s->device] = address;
    }
    scratch = scratchAddress[s->device];
  }
  cudaStream_t launchStream = stream ? static_cast<cudaStream_t>(stream) : s->stream;
  const int launched = jgs2::launchGateScratch(
      s->b, p, reinterpret_cast<const float4*>(predicted), reinterpret_cast<const float4*>(source),
      reinterpret_cast<const float4*>(candidate), s->V, s->T, s->C, s->H, reinterpret_cast<float4*>(control),
      scratch, launchStream);
  if (launched == 0) return fail(s, JGS2_INVALID_ARGUMENT, "The no-allocation gate was given an empty mesh.");
  CUDA_TRY(s, cudaGetLastError());
  s->launches += static_cast<uint64_t>(launched);
  return JGS2_OK;
}

// ---- checkpoint / resume ----------------------------------------------------
// A solver's state between frames, as one self-describing byte image:
// header, then the per-vertex arrays and the frame record.  The frame start
// derives everything else (inertial target, frames, incident systems,
// contact caches and lagged forces) from these, so a solver created from the
// same input and given this image steps exactly as the exporting one would.
namespace {

constexpr char kStateMagic[8] = {'J', 'G', 'S', '2', 'S', 'T', 'A', '1'};
constexpr uint32_t kStateVersion = 1;

struct StateHeader {
  char magic[8];
  uint32_t version, V, T, K, KC, C, H;
  uint32_t objectiveFlags, forceCount, targetCount, objectiveRevision;
  uint32_t submittedIterations, recordsAvailable;
  uint64_t bytes;
  jgs2_settings submitted;
};

struct StateRegion {
  void* dev;
  size_t bytes;
};

std::vector<StateRegion> stateRegions(Engine* s) {
  const size_t V = s->V;
  return {{s->b.pos[0], 16 * V},        {s->b.velocity, 16 * V},  {s->b.old, 16 * V},
          {s->b.predicted, 16 * V},     {s->b.vertexRot, 48 * V}, {s->b.incident, 48 * V},
          {s->b.local, 64 * V},         {s->b.finalUpdate, 4 * V}, {s->b.forces, 16 * V},
          {s->b.targets, 16 * V},       {s->b.frames, sizeof(FrameState)}};
}

size_t stateBytes(Engine* s) {
  size_t n = sizeof(StateHeader);
  for (const StateRegion& r : stateRegions(s)) n += r.bytes;
  return n;
}

}  // namespace

jgs2_status jgs2_export_state(jgs2_solver* s, void* out, size_t capacity, size_t* size) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (s->scenes.size() != 1) return fail(s, JGS2_UNSUPPORTED, "State export covers single-scene solvers.");
  const size_t need = stateBytes(s);
  if (size) *size = need;
  if (!out) return JGS2_OK;
  if (capacity < need) return fail(s, JGS2_INVALID_ARGUMENT, format("The state image needs %zu bytes.", need));
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  st = checkBroadPhase(s);
  if (st != JGS2_OK) return st;
  const SceneHost& sc = s->scenes[0];
  StateHeader h{};
  std::memcpy(h.magic, kStateMagic, sizeof(kStateMagic));
  h.version = kStateVersion;
  h.V = s->V; h.T = s->T; h.K = s->K; h.KC = s->KC; h.C = s->C; h.H = s->H;
  h.objectiveFlags = sc.objectiveFlags;
  h.forceCount = sc.forceCount;
  h.targetCount = sc.targetCount;
  h.objectiveRevision = sc.objectiveRevision;
  h.submittedIterations = sc.submittedIterations;
  h.recordsAvailable = sc.recordsAvailable ? 1u : 0u;
  h.bytes = need;
  h.submitted = sc.submitted;
  unsigned char* p = static_cast<unsigned char*>(out);
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  for (const StateRegion& r : stateRegions(s)) {
    CUDA_TRY(s, cudaMemcpyAsync(p, r.dev, r.bytes, cudaMemcpyDeviceToHost, s->stream));
    p += r.bytes;
  }
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return JGS2_OK;
}

jgs2_status jgs2_import_state(jgs2_solver* s, const void* in, size_t size) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (s->scenes.size() != 1) return fail(s, JGS2_UNSUPPORTED, "State import covers single-scene solvers.");
  if (!in || size < sizeof(StateHeader)) return fail(s, JGS2_INVALID_ARGUMENT, "The state image is too short.");
  StateHeader h;
  std::memcpy(&h, in, sizeof(h));
  if (std::memcmp(h.magic, kStateMagic, sizeof(kStateMagic)) != 0 || h.version != kStateVersion)
    return fail(s, JGS2_INVALID_ARGUMENT, "The state image is not a version-1 JGS2 state image.");
  if (h.V != s->V || h.T != s->T || h.K != s->K || h.KC != s->KC || h.C != s->C || h.H != s->H)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("The state image is of a solver with %u vertices, %u tetrahedra, %u cubature records, %u "
                       "contact candidates, %u triangles and %u hinges; this solver has %u, %u, %u, %u, %u and %u.",
                       h.V, h.T, h.K, h.KC, h.C, h.H, s->V, s->T, s->K, s->KC, s->C, s->H));
  const size_t need = stateBytes(s);
  if (h.bytes != need || size < need)
    return fail(s, JGS2_INVALID_ARGUMENT, format("The state image must hold %zu bytes.", need));
  st = waitObjectiveMirror(s);
  if (st != JGS2_OK) return st;
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  const unsigned char* p = static_cast<const unsigned char*>(in) + sizeof(h);
  for (const StateRegion& r : stateRegions(s)) {
    if (r.dev == s->b.forces) std::memcpy(s->hForces, p, r.bytes);
    if (r.dev == s->b.targets) std::memcpy(s->hTargets, p, r.bytes);
    CUDA_TRY(s, cudaMemcpyAsync(r.dev, p, r.bytes, cudaMemcpyHostToDevice, s->stream));
    p += r.bytes;
  }
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  SceneHost& sc = s->scenes[0];
  sc.objectiveFlags = h.objectiveFlags;
  sc.forceCount = h.forceCount;
  sc.targetCount = h.targetCount;
  sc.objectiveRevision = h.objectiveRevision;
  sc.submittedIterations = h.submittedIterations;
  sc.recordsAvailable = h.recordsAvailable != 0;
  sc.submitted = h.submitted;
  return JGS2_OK;
}

jgs2_status jgs2_device_positions(jgs2_solver* s, void** ptr, void** stream) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (ptr) *ptr = s->b.pos[0];
  if (stream) *stream = s->stream;
  return JGS2_OK;
}

uint64_t jgs2_kernel_launch_count(const jgs2_solver* s) { return s ? s->launches : 0; }

namespace {

jgs2_status startTuning(Engine* s, uint32_t rounds) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (rounds < 1 || rounds > 64)
    return fail(s, JGS2_INVALID_ARGUMENT, format("Autotuning rounds must be 1-64; got %u.", rounds));
  CUDA_TRY(s, cudaSetDevice(s->device));
  for (cudaEvent_t& e : s->tuneEvents)
    if (!e) CUDA_TRY(s, cudaEventCreate(&e));
  for (auto& v : s->tuneMs) v.clear();
  s->tuneRounds = rounds;
  s->tuneLeft = rounds * JGS2_LAUNCH_SHAPES;
  s->tuneNext = 0;
  return JGS2_OK;
}

jgs2_status readShape(Engine* s, jgs2_launch_shape* out) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  *out = jgs2_launch_shape{};
  out->shape = s->b.solveShift;
  CUDA_TRY(s, cudaSetDevice(s->device));
  const uint32_t fit = jgs2::solveGroupsPerBlock(s->K);
  const uint32_t groups = std::max(1u, fit >> s->b.solveShift);
  out->solve_vertices_per_block = fit == 0 ? 0 : groups;
  out->tuning = s->tuneLeft;
  uint32_t fewest = ~0u;
  for (uint32_t c = 0; c < JGS2_LAUNCH_SHAPES; ++c) {
    out->frame_ms[c] = medianMs(s->tuneMs[c]);
    fewest = std::min<uint32_t>(fewest, static_cast<uint32_t>(s->tuneMs[c].size()));
  }
  out->samples = fewest;
  return JGS2_OK;
}

jgs2_status fixShape(Engine* s, uint32_t shape) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (shape >= JGS2_LAUNCH_SHAPES)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("Launch shape must be below %u; got %u.", JGS2_LAUNCH_SHAPES, shape));
  s->b.solveShift = shape;
  s->tuneLeft = 0;
  return JGS2_OK;
}

}  // namespace

jgs2_status jgs2_autotune(jgs2_solver* s, uint32_t rounds) { return startTuning(s, rounds); }
jgs2_status jgs2_get_launch_shape(jgs2_solver* s, jgs2_launch_shape* out) { return readShape(s, out); }
jgs2_status jgs2_set_launch_shape(jgs2_solver* s, uint32_t shape) { return fixShape(s, shape); }

// ---- batches -------------------------------------------------------------------

jgs2_status jgs2_batch_create(const jgs2_input* const* inputs, uint32_t scene_count, const jgs2_settings* settings,
                              const uint32_t* masks, int device, jgs2_batch** out) {
  if (!out) return fail(nullptr, JGS2_INVALID_ARGUMENT, "out is NULL.");
  *out = nullptr;
  if (!inputs || scene_count == 0) return fail(nullptr, JGS2_INVALID_ARGUMENT, "A batch needs at least one scene.");
  // Graph colouring is built only when some scene's default schedule needs it.
  bool colour = false;
  for (uint32_t i = 0; i < scene_count; ++i) {
    jgs2_settings base, resolved;
    defaults(&base);
    std::string err;
    if (resolve(base, settings ? &settings[i] : nullptr, masks ? masks[i] : 0u, &resolved, &err) &&
        resolved.schedule == JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL)
      colour = true;
  }
  std::vector<PreparedScene> prep(scene_count);
  std::vector<jgs2_status> status(scene_count, JGS2_OK);
  parallelFor(scene_count, [&](uint32_t i) {
    status[i] = prepareScene(inputs[i], settings ? &settings[i] : nullptr, masks ? masks[i] : 0u, colour, &prep[i]);
    if (status[i] != JGS2_OK) prep[i].error = gGlobalError;  // this worker's thread-local message
  });
  for (uint32_t i = 0; i < scene_count; ++i) {
    if (status[i] != JGS2_OK) {
      gGlobalError = format("scene %u: %s", i, prep[i].error.c_str());
      return status[i];
    }
  }
  std::unique_ptr<jgs2_batch> s(new jgs2_batch());
  const jgs2_status st = buildEngine(s.get(), prep, device);
  if (st != JGS2_OK) return st;
  *out = s.release();
  return JGS2_OK;
}

void jgs2_batch_destroy(jgs2_batch* s) {
  if (!s) return;
  if (!s->destroyed) {
    cudaSetDevice(s->device);
    releaseDevice(s);
    s->destroyed = true;
  }
  delete s;
}

const char* jgs2_batch_last_error(const jgs2_batch* s) { return s ? s->error.c_str() : gGlobalError.c_str(); }

uint32_t jgs2_batch_scene_count(const jgs2_batch* s) { return s ? static_cast<uint32_t>(s->scenes.size()) : 0u; }

jgs2_status jgs2_batch_step_frames(jgs2_batch* s, uint32_t frames, uint32_t exact_iterations,
                                   const jgs2_settings* overrides, const uint32_t* masks) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (frames < 1 || frames > JGS2_MAX_BATCH_FRAMES)
    return fail(s, JGS2_INVALID_ARGUMENT,
                format("frameCount must be a positive safe integer no greater than %u; got %u.",
                       JGS2_MAX_BATCH_FRAMES, frames));
  const uint32_t S = static_cast<uint32_t>(s->scenes.size());
  std::vector<jgs2_settings> resolved(S);
  uint32_t iterations = exact_iterations;
  for (uint32_t i = 0; i < S; ++i) {
    st = resolveStep(s, i, overrides ? &overrides[i] : nullptr, masks ? masks[i] : 0u, &resolved[i]);
    if (st != JGS2_OK) {
      s->error = format("scene %u: %s", i, s->error.c_str());
      return st;
    }
    if (exact_iterations == 0) {
      // Production stepping: every scene's normalised odd count must agree.
      const uint32_t it = normalizeOdd(resolved[i].iterations);
      if (i == 0) iterations = it;
      else if (it != iterations)
        return fail(s, JGS2_INVALID_ARGUMENT,
                    format("All scenes of one batched production step must run the same number of iterations; "
                           "scene 0 runs %u, scene %u runs %u.", iterations, i, it));
    }
  }
  return runFrames(s, resolved, frames, iterations, exact_iterations == 0);
}

jgs2_status jgs2_batch_sync(jgs2_batch* s) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  CUDA_TRY(s, cudaSetDevice(s->device));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return JGS2_OK;
}

jgs2_status jgs2_batch_get_info(jgs2_batch* s, uint32_t scene, jgs2_info* out) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (scene >= s->scenes.size()) return fail(s, JGS2_INVALID_ARGUMENT, format("scene %u is out of range.", scene));
  if (!out) return fail(s, JGS2_INVALID_ARGUMENT, "out is NULL.");
  return sceneInfo(s, scene, out);
}

jgs2_status jgs2_batch_read_positions(jgs2_batch* s, uint32_t scene, float* out, size_t floats) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (scene >= s->scenes.size()) return fail(s, JGS2_INVALID_ARGUMENT, format("scene %u is out of range.", scene));
  return readSceneVec4(s, scene, s->b.pos[0], out, floats, 4);
}

jgs2_status jgs2_batch_read_velocities(jgs2_batch* s, uint32_t scene, float* out, size_t floats) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (scene >= s->scenes.size()) return fail(s, JGS2_INVALID_ARGUMENT, format("scene %u is out of range.", scene));
  return readSceneVec4(s, scene, s->b.velocity, out, floats, 4);
}

jgs2_status jgs2_batch_read_globalization(jgs2_batch* s, uint32_t scene, float* local, size_t local_floats,
                                          float* control, float* history, size_t history_floats,
                                          uint32_t* history_count) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (scene >= s->scenes.size()) return fail(s, JGS2_INVALID_ARGUMENT, format("scene %u is out of range.", scene));
  return readSceneGlobalization(s, scene, local, local_floats, control, history, history_floats, history_count);
}

jgs2_status jgs2_batch_read_all_positions(jgs2_batch* s, float* out, size_t floats) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (!out || floats < 4ull * s->V)
    return fail(s, JGS2_INVALID_ARGUMENT, format("output needs %llu floats.", 4ull * s->V));
  return readRegion(s, s->b.pos[0], sizeof(float4) * s->V, out);
}

uint64_t jgs2_batch_kernel_launch_count(const jgs2_batch* s) { return s ? s->launches : 0; }
jgs2_status jgs2_batch_autotune(jgs2_batch* s, uint32_t rounds) { return startTuning(s, rounds); }
jgs2_status jgs2_batch_get_launch_shape(jgs2_batch* s, jgs2_launch_shape* out) { return readShape(s, out); }
jgs2_status jgs2_batch_set_launch_shape(jgs2_batch* s, uint32_t shape) { return fixShape(s, shape); }

uint32_t jgs2_batch_vertex_count(const jgs2_batch* s) { return s ? s->V : 0u; }

void* jgs2_batch_stream(const jgs2_batch* s) { return s ? static_cast<void*>(s->stream) : nullptr; }

jgs2_status jgs2_batch_set_scene_active(jgs2_batch* s, uint32_t scene, uint32_t active) {
  jgs2_status st = usable(s);
  if (st != JGS2_OK) return st;
  if (scene >= s->scenes.size()) return fail(s, JGS2_INVALID_ARGUMENT, format("scene %u is out of range.", scene));
  s->scenes[scene].active = active != 0;
  return JGS2_OK;
}

uint64_t jgs2_estimate_device_bytes(const jgs2_input* in) {
  if (!in) return 0;
  const uint64_t V = in->vertex_count, T = in->tet_count, K = in->cubature_k;
  // Per vertex: two position buffers, predicted, velocity, old, frame (3),
  // local records (4), incident system (3), rest/mass, info, force, target
  // (16 bytes each), final update, colour, scene id; per record a 32-byte
  // header and 144 bytes of basis; per tet a 64-byte record, four adjacency
  // entries and a share of the reduction partials; per cloth triangle and
  // hinge a 32-byte record and one incidence entry per vertex, plus a
  // 16-byte incidence range per vertex.
  const uint64_t C = in->cloth ? in->cloth->triangle_count : 0, H = in->cloth ? in->cloth->hinge_count : 0;
  const uint64_t cloth = (C + H) ? V * 16 + C * (32 + 12) + H * (32 + 16) : 0;
  // IPC: per candidate its indices, scene, 7 float4 of state and four
  // incidence and four active entries; per vertex a range and an active count.
  const uint64_t KC = uint64_t(in->contact_vertex_triangle_count) + in->contact_edge_edge_count;
  uint64_t contact = KC ? KC * (16 + 4 + 112 + 32) + V * 12 : 0;
  if (const jgs2_contact_surface* cs = in->contact_surface) {
    // Broad phase: two lists of capacity candidates (indices, scene, state,
    // flag, column) and the sort's four entry buffers; surface data, boxes
    // and rows per triangle and edge (at most three edges per triangle).
    const uint64_t E = 3ull * cs->triangle_count;
    const uint64_t cap = cs->candidate_capacity ? cs->candidate_capacity : 65536 + 16 * (V + E);
    contact = 2 * cap * (16 + 4 + 112 + 4 + 4) + 4 * cap * 16 + cs->triangle_count * (16 + 32) + E * (8 + 32 + 32) +
              V * (8 + 16 + 8 + 8 + 4 + 16) + (4 * cap / 4096 + 1) * 1024;
  }
  return V * (16 * 20 + 12) + V * K * (32 + 144) + T * (64 + 16 + 1) + cloth + contact + (1u << 16);
}

}  // extern "C"
