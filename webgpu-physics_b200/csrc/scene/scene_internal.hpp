// Internal types of the scene builder / precompute library.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "jgs2_scene.h"

namespace jgs2scene {

struct Material {
  double density;
  double young;
  double poisson;
  uint32_t model;  // JGS2_MATERIAL_*
};

// Tetrahedral mesh in the reference's TetrahedralMesh shape
// (src/simulation/cpu/types.ts): xyz positions, four indices per tet.
struct Mesh {
  std::vector<double> positions;    // 3 * V rest positions
  std::vector<uint32_t> tets;       // 4 * T
  std::vector<uint32_t> materials;  // T
  std::vector<uint8_t> fixed;       // V
  std::vector<uint32_t> bodies;     // V
  uint32_t vertexCount() const { return static_cast<uint32_t>(fixed.size()); }
  uint32_t tetCount() const { return static_cast<uint32_t>(materials.size()); }
};

// Rest data per tet (computeRestTetraData, src/simulation/cpu/fem.ts:167-209):
// volume and row-major inverse rest matrix.  The 12x12 linear stiffness is
// recomputed on demand so million-tet scenes need not store it.
struct RestData {
  std::vector<double> volumes;  // T
  std::vector<double> inverseRest;  // 9 * T row-major
};

struct CubatureRecord {
  uint32_t tet = 0xffffffffu;
  double weight = 0.0;
  std::array<double, 36> basis{};  // four row-major 3x3 blocks
};

// Triangle cloth of a scene (SceneDefinition.cloth, src/scenes/index.ts:688-696):
// triangles over scene vertices and one membrane / bending material.
struct Cloth {
  bool present = false;
  std::vector<uint32_t> triangles;  // 3 per triangle, scene vertex ids
  double density = 0, young = 0, poisson = 0, thickness = 0, bending = 0;
};

struct Scene {
  std::string error;
  std::vector<Material> materialTable;
  Mesh mesh;
  Cloth cloth;
  RestData rest;
  bool restValid = false;
  std::vector<double> masses;  // lumped, V
  // Precompute output
  bool precomputed = false;
  double timestep = 0.0;
  uint32_t cubatureK = 0;
  std::vector<uint32_t> recordTets;      // V * K
  std::vector<float> recordWeights;      // V * K
  std::vector<float> recordBasis;        // V * K * 36
  // Initial state / objectives
  std::vector<float> initialPositions;   // 4 * V (empty = rest)
  std::vector<float> initialVelocities;  // 4 * V (empty = none)
  bool pinAtInitial = false;
  std::vector<float> externalForces;     // 3 * V or empty
  std::vector<float> targetPositions;    // 3 * V or empty
  std::vector<float> targetStiffnesses;  // V or empty
  // Packed arrays (owned)
  std::vector<float> packPositions, packVelocities, packRest, packColors;
  std::vector<uint32_t> packInfo, packTetIndices, packAdjacency;
  std::vector<float> packInverseDm, packMeta, packStiffness;
  std::vector<uint32_t> packClothTriangles, packHinges;
  std::vector<float> packClothInverse, packClothAreas, packHingeAngles, packHingeLengths;
  jgs2_cloth_input packCloth{};
  // Static IPC candidates over the boundary surface (tets) and the cloth.
  uint32_t contact = 0;  // JGS2_SCENE_CONTACT_*
  uint64_t contactCapacity = 0;
  std::vector<uint32_t> packContact;
  uint32_t packContactVT = 0, packContactEE = 0;
  std::vector<uint32_t> packSurface;
  jgs2_contact_surface packSurfaceRec{};
};

// ---- small dense helpers (row-major 3x3) ---------------------------------
double det3(const double* m);
// invert3 (src/simulation/cpu/math.ts:11-35); returns false when singular.
bool inv3(const double* m, double* out);
void mul3(const double* a, const double* b, double* out);
void transpose3(const double* a, double* out);
// polarRotation3 (src/simulation/cpu/oracle.ts:182-217), row-major in/out.
void polarRotation3(const double* f, double* r);

// Four material-space shape gradients (computeTetrahedronShapeGradients,
// src/simulation/cpu/fem.ts:68-83), row-major 4x3.
void shapeGradients(const double* inverseRest, double* g);
// Linear co-rotated stiffness (computeLinearTetrahedronStiffness,
// src/simulation/cpu/fem.ts:85-165) from stored rest data.
void linearStiffness(const double* inverseRest, double volume,
                     const Material& material, double* k144);

// Hooke Lame parameters and the stable Neo-Hookean reparameterisation
// (computeStableNeoHookeanParameters, src/simulation/cpu/stable-neo-hookean.ts:68-110).
void hookeLame(const Material& m, double* lambda, double* mu);
void stableLame(const Material& m, double* lambda, double* mu);

// Precompute driver (precompute.cpp).
bool runPrecompute(Scene& scene, const jgs2_precompute_options& options,
                   jgs2_precompute_stats* stats);

}  // namespace jgs2scene
