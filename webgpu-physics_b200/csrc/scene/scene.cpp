// Scene builder: procedural meshes, FEM rest data, lumped masses and the
// jgs2_input packer.  Restates src/simulation/cpu/mesh.ts,
// src/simulation/cpu/fem.ts and src/scenes/index.ts:811-1109 in C++.
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <unordered_map>

#include "scene_internal.hpp"

namespace jgs2scene {

double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

bool inv3(const double* m, double* out) {
  const double determinant = det3(m);
  double scale = 0.0;
  for (int i = 0; i < 9; ++i) scale = std::max(scale, std::fabs(m[i]));
  if (scale == 0.0 || std::fabs(determinant) <= 1e-14 * scale * scale * scale) return false;
  const double s = 1.0 / determinant;
  out[0] = (m[4] * m[8] - m[5] * m[7]) * s;
  out[1] = (m[2] * m[7] - m[1] * m[8]) * s;
  out[2] = (m[1] * m[5] - m[2] * m[4]) * s;
  out[3] = (m[5] * m[6] - m[3] * m[8]) * s;
  out[4] = (m[0] * m[8] - m[2] * m[6]) * s;
  out[5] = (m[2] * m[3] - m[0] * m[5]) * s;
  out[6] = (m[3] * m[7] - m[4] * m[6]) * s;
  out[7] = (m[1] * m[6] - m[0] * m[7]) * s;
  out[8] = (m[0] * m[4] - m[1] * m[3]) * s;
  return true;
}

void mul3(const double* a, const double* b, double* out) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += a[i * 3 + k] * b[k * 3 + j];
      r[i * 3 + j] = v;
    }
  std::memcpy(out, r, sizeof(r));
}

void transpose3(const double* a, double* out) {
  double r[9] = {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]};
  std::memcpy(out, r, sizeof(r));
}

namespace {
constexpr double kPolarEpsilon = 1e-14;   // src/simulation/cpu/oracle.ts:20
constexpr int kPolarIterations = 20;      // src/simulation/cpu/oracle.ts:21

void normalized3(const double* v, const double* fallback, double* out) {
  const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (!(n > kPolarEpsilon) || !std::isfinite(n)) {
    out[0] = fallback[0]; out[1] = fallback[1]; out[2] = fallback[2];
    return;
  }
  out[0] = v[0] / n; out[1] = v[1] / n; out[2] = v[2] / n;
}

void cross3(const double* a, const double* b, double* out) {
  const double x = a[1] * b[2] - a[2] * b[1];
  const double y = a[2] * b[0] - a[0] * b[2];
  const double z = a[0] * b[1] - a[1] * b[0];
  out[0] = x; out[1] = y; out[2] = z;
}

void perpendicularTo(const double* axis, double* out) {
  const double cx[3] = {1, 0, 0}, cy[3] = {0, 1, 0}, fz[3] = {0, 0, 1};
  double c[3];
  cross3(axis, std::fabs(axis[0]) > 0.8 ? cy : cx, c);
  normalized3(c, fz, out);
}

// orthonormalizeRotation (src/simulation/cpu/oracle.ts:140-180).
void orthonormalizeRotation(const double* m, double* out) {
  const double in0[3] = {m[0], m[3], m[6]}, in1[3] = {m[1], m[4], m[7]},
               in2[3] = {m[2], m[5], m[8]};
  const double fx[3] = {1, 0, 0}, fz[3] = {0, 0, 1};
  double c0[3], c1[3], c2[3], perp[3], tmp[3];
  normalized3(in0, fx, c0);
  const double p = c0[0] * in1[0] + c0[1] * in1[1] + c0[2] * in1[2];
  const double cand[3] = {in1[0] - p * c0[0], in1[1] - p * c0[1], in1[2] - p * c0[2]};
  perpendicularTo(c0, perp);
  normalized3(cand, perp, c1);
  cross3(c0, c1, tmp);
  normalized3(tmp, fz, c2);
  if (c2[0] * in2[0] + c2[1] * in2[1] + c2[2] * in2[2] < 0) {
    for (int i = 0; i < 3; ++i) { c1[i] = -c1[i]; c2[i] = -c2[i]; }
  }
  cross3(c2, c0, tmp);
  normalized3(tmp, perp, c1);
  const double r[9] = {c0[0], c1[0], c2[0], c0[1], c1[1], c2[1], c0[2], c1[2], c2[2]};
  std::memcpy(out, r, sizeof(r));
}
}  // namespace

void polarRotation3(const double* f, double* r) {
  double rot[9];
  std::memcpy(rot, f, sizeof(rot));
  for (int it = 0; it < kPolarIterations; ++it) {
    const double d = det3(rot);
    if (!(std::fabs(d) > kPolarEpsilon) || !std::isfinite(d)) break;
    double inv[9];
    if (!inv3(rot, inv)) break;
    double next[9];
    double change = 0.0;
    for (int row = 0; row < 3; ++row)
      for (int col = 0; col < 3; ++col) {
        const int i = row * 3 + col;
        next[i] = 0.5 * (rot[i] + inv[col * 3 + row]);
        change = std::max(change, std::fabs(next[i] - rot[i]));
      }
    std::memcpy(rot, next, sizeof(rot));
    if (change <= 1e-14) break;
  }
  orthonormalizeRotation(rot, r);
}

void shapeGradients(const double* inverseRest, double* g) {
  for (int c = 0; c < 3; ++c) {
    g[3 + c] = inverseRest[c];
    g[6 + c] = inverseRest[3 + c];
    g[9 + c] = inverseRest[6 + c];
    g[c] = -g[3 + c] - g[6 + c] - g[9 + c];
  }
}

void hookeLame(const Material& m, double* lambda, double* mu) {
  *lambda = (m.young * m.poisson) / ((1 + m.poisson) * (1 - 2 * m.poisson));
  *mu = m.young / (2 * (1 + m.poisson));
}

void stableLame(const Material& m, double* lambda, double* mu) {
  double l, u;
  hookeLame(m, &l, &u);
  *mu = (4.0 / 3.0) * u;
  *lambda = l + (5.0 / 6.0) * u;
}

void linearStiffness(const double* inverseRest, double volume, const Material& material,
                     double* k) {
  double g[12];
  shapeGradients(inverseRest, g);
  double B[6 * 12] = {};
  for (int v = 0; v < 4; ++v) {
    const double gx = g[v * 3], gy = g[v * 3 + 1], gz = g[v * 3 + 2];
    const int c = v * 3;
    B[c] = gx;
    B[12 + c + 1] = gy;
    B[24 + c + 2] = gz;
    B[36 + c] = gy;
    B[36 + c + 1] = gx;
    B[48 + c + 1] = gz;
    B[48 + c + 2] = gy;
    B[60 + c] = gz;
    B[60 + c + 2] = gx;
  }
  double lambda, mu;
  hookeLame(material, &lambda, &mu);
  double D[36] = {};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) D[r * 6 + c] = r == c ? lambda + 2 * mu : lambda;
  D[3 * 6 + 3] = mu;
  D[4 * 6 + 4] = mu;
  D[5 * 6 + 5] = mu;
  double DB[6 * 12];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 12; ++c) {
      double v = 0;
      for (int i = 0; i < 6; ++i) v += D[r * 6 + i] * B[i * 12 + c];
      DB[r * 12 + c] = v;
    }
  for (int r = 0; r < 12; ++r)
    for (int c = r; c < 12; ++c) {
      double v = 0;
      for (int i = 0; i < 6; ++i) v += B[i * 12 + r] * DB[i * 12 + c];
      v *= volume;
      k[r * 12 + c] = v;
      k[c * 12 + r] = v;
    }
}

}  // namespace jgs2scene

using namespace jgs2scene;

struct jgs2_scene : public jgs2scene::Scene {};

namespace {

bool fail(jgs2_scene* s, const std::string& message) {
  if (s) s->error = message;
  return false;
}

// orientTetrahedra (src/simulation/cpu/mesh.ts:80-99).
bool orientTets(const std::vector<double>& p, uint32_t* tets, size_t count, std::string* err) {
  for (size_t t = 0; t < count; ++t) {
    uint32_t* q = tets + 4 * t;
    const double* a = &p[3 * q[0]];
    const double m[9] = {p[3 * q[1]] - a[0], p[3 * q[2]] - a[0], p[3 * q[3]] - a[0],
                         p[3 * q[1] + 1] - a[1], p[3 * q[2] + 1] - a[1], p[3 * q[3] + 1] - a[1],
                         p[3 * q[1] + 2] - a[2], p[3 * q[2] + 2] - a[2], p[3 * q[3] + 2] - a[2]};
    const double d = det3(m);
    if (std::fabs(d) <= 1e-14) {
      *err = "Tetrahedron " + std::to_string(t) + " is degenerate.";
      return false;
    }
    if (d < 0) std::swap(q[1], q[2]);
  }
  return true;
}

bool computeRest(Scene& s) {
  if (s.restValid) return true;
  const uint32_t T = s.mesh.tetCount();
  const uint32_t V = s.mesh.vertexCount();
  s.rest.volumes.assign(T, 0.0);
  s.rest.inverseRest.assign(9ull * T, 0.0);
  s.masses.assign(V, 0.0);
  const auto& p = s.mesh.positions;
  for (uint32_t t = 0; t < T; ++t) {
    const uint32_t* q = &s.mesh.tets[4ull * t];
    const double* a = &p[3ull * q[0]];
    // restMatrix (src/simulation/cpu/fem.ts:38-58): columns b-a, c-a, d-a.
    const double m[9] = {p[3ull * q[1]] - a[0], p[3ull * q[2]] - a[0], p[3ull * q[3]] - a[0],
                         p[3ull * q[1] + 1] - a[1], p[3ull * q[2] + 1] - a[1], p[3ull * q[3] + 1] - a[1],
                         p[3ull * q[1] + 2] - a[2], p[3ull * q[2] + 2] - a[2], p[3ull * q[3] + 2] - a[2]};
    const double vol = std::fabs(det3(m)) / 6.0;
    if (!(vol > 1e-14) || !std::isfinite(vol)) {
      s.error = "Cannot assemble a degenerate tetrahedron.";
      return false;
    }
    double inv[9];
    if (!inv3(m, inv)) {
      s.error = "Cannot invert a singular 3 by 3 matrix.";
      return false;
    }
    s.rest.volumes[t] = vol;
    std::memcpy(&s.rest.inverseRest[9ull * t], inv, sizeof(inv));
    // computeLumpedMasses (src/simulation/cpu/fem.ts:211-236).
    const double vm = s.materialTable[s.mesh.materials[t]].density * vol / 4.0;
    for (int l = 0; l < 4; ++l) s.masses[q[l]] += vm;
  }
  // validateAndAddClothMasses (src/simulation/cpu/precompute.ts:44-95): each
  // cloth triangle adds density * thickness * area / 3 to its vertices.
  if (s.cloth.present) {
    const size_t C = s.cloth.triangles.size() / 3;
    for (size_t c = 0; c < C; ++c) {
      const uint32_t* q = &s.cloth.triangles[3 * c];
      double e1[3], e2[3], n[3];
      for (int k = 0; k < 3; ++k) {
        e1[k] = p[3ull * q[1] + k] - p[3ull * q[0] + k];
        e2[k] = p[3ull * q[2] + k] - p[3ull * q[0] + k];
      }
      n[0] = e1[1] * e2[2] - e1[2] * e2[1];
      n[1] = e1[2] * e2[0] - e1[0] * e2[2];
      n[2] = e1[0] * e2[1] - e1[1] * e2[0];
      const double area = 0.5 * std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      if (!(area > 1e-12) || !std::isfinite(area)) {
        s.error = "Cloth triangle " + std::to_string(c) + " must be nondegenerate.";
        return false;
      }
      const double vm = s.cloth.density * s.cloth.thickness * area / 3.0;
      for (int l = 0; l < 3; ++l) s.masses[q[l]] += vm;
    }
  }
  s.restValid = true;
  return true;
}

// ---- cloth rest data (src/simulation/cpu/cloth.ts:107-140, 237-334) --------

double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// assertNondegenerateTriangle (cloth.ts:90-104): twice the area, or -1.
double nondegenerateTwiceArea(const double* e0, const double* e1) {
  double c[3];
  cross3(e0, e1, c);
  const double twiceArea = norm3(c);
  const double d[3] = {e1[0] - e0[0], e1[1] - e0[1], e1[2] - e0[2]};
  const double scale = std::max(norm3(e0), std::max(norm3(e1), norm3(d)));
  if (!(scale > 0) || !(twiceArea > 1e-12 * scale * scale)) return -1.0;
  return twiceArea;
}

// precomputeStVKTriangleRest (cloth.ts:111-140): the intrinsic 2D basis has
// its first axis along rest edge (0, 1); returns the row-major inverse of
// Dm = [[|e01|, x], [0, y]] and the rest area.
bool clothTriangleRest(const double* x0, const double* x1, const double* x2, double inverse[4], double* area) {
  const double e01[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
  const double e02[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
  const double twiceArea = nondegenerateTwiceArea(e01, e02);
  if (twiceArea < 0) return false;
  const double length = norm3(e01);
  const double tangent[3] = {e01[0] / length, e01[1] / length, e01[2] / length};
  double normal[3];
  cross3(e01, e02, normal);
  for (double& c : normal) c /= twiceArea;
  double bitangent[3];
  cross3(normal, tangent, bitangent);
  const double mx = e02[0] * tangent[0] + e02[1] * tangent[1] + e02[2] * tangent[2];
  const double my = e02[0] * bitangent[0] + e02[1] * bitangent[1] + e02[2] * bitangent[2];
  inverse[0] = 1.0 / length;
  inverse[1] = -mx / (length * my);
  inverse[2] = 0.0;
  inverse[3] = 1.0 / my;
  *area = 0.5 * twiceArea;
  return true;
}

// precomputeQuadraticDihedralRest (cloth.ts:316-321) through the angle of
// evaluateSignedDihedral (cloth.ts:237-312) for the oriented hinge
// (0, 1, 2) / (1, 0, 3).
bool clothHingeRest(const double* x0, const double* x1, const double* x2, const double* x3, double* angle,
                    double* edgeLength) {
  const double edge[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
  const double length = norm3(edge);
  if (!(length > 0)) return false;
  const double to2[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
  const double reverse[3] = {-edge[0], -edge[1], -edge[2]};
  const double to3[3] = {x3[0] - x1[0], x3[1] - x1[1], x3[2] - x1[2]};
  const double l0 = nondegenerateTwiceArea(edge, to2);
  const double l1 = nondegenerateTwiceArea(reverse, to3);
  if (l0 < 0 || l1 < 0) return false;
  double n0[3], n1[3], nc[3];
  cross3(edge, to2, n0);
  cross3(reverse, to3, n1);
  for (int k = 0; k < 3; ++k) { n0[k] /= l0; n1[k] /= l1; }
  cross3(n0, n1, nc);
  const double sine = (edge[0] * nc[0] + edge[1] * nc[1] + edge[2] * nc[2]) / length;
  const double cosine = n0[0] * n1[0] + n0[1] * n1[1] + n0[2] * n1[2];
  *angle = std::atan2(sine, cosine);
  *edgeLength = length;
  return true;
}

// extractBoundarySurface (src/simulation/cpu/mesh.ts:364-420): the faces that
// belong to exactly one tetrahedron, each as its sorted vertex triple (the
// candidate enumeration below only needs the vertex sets).
bool boundaryTriangles(const Mesh& m, std::vector<std::array<uint32_t, 3>>* out, std::string* err) {
  std::unordered_map<uint64_t, std::pair<std::array<uint32_t, 3>, int>> faces;
  faces.reserve(m.tets.size());
  for (size_t t = 0; t < m.tets.size() / 4; ++t) {
    const uint32_t* q = &m.tets[4 * t];
    const uint32_t local[4][3] = {{q[1], q[2], q[3]}, {q[0], q[3], q[2]}, {q[0], q[1], q[3]}, {q[0], q[2], q[1]}};
    for (const auto& f : local) {
      std::array<uint32_t, 3> s = {f[0], f[1], f[2]};
      std::sort(s.begin(), s.end());
      // 21 bits per index is enough for the contact scenes (the enumeration
      // is quadratic); larger meshes are rejected.
      if (s[2] >= (1u << 21)) {
        *err = "Contact candidate enumeration takes meshes below 2^21 vertices.";
        return false;
      }
      const uint64_t key = (static_cast<uint64_t>(s[0]) << 42) | (static_cast<uint64_t>(s[1]) << 21) | s[2];
      auto it = faces.find(key);
      if (it == faces.end()) {
        faces.emplace(key, std::make_pair(s, 1));
      } else if (++it->second.second > 2) {
        *err = "Non-manifold face belongs to over two tets.";
        return false;
      }
    }
  }
  for (const auto& kv : faces)
    if (kv.second.second == 1) out->push_back(kv.second.first);
  return true;
}

// buildStaticIpcContactCandidates (src/simulation/cpu/ipc-contact.ts:591-665):
// canonical (sorted, deduplicated) surface triangles and edges; every vertex
// paired with every triangle none of whose vertices is in the vertex's closed
// surface one-ring, then every edge pair (lexicographic order, i < j) whose
// vertices are pairwise outside each other's closed one-rings.  Four indices
// per candidate, vertex-triangle candidates first.
void staticContactCandidates(uint32_t V, std::vector<std::array<uint32_t, 3>> triangles, std::vector<uint32_t>* out,
                             uint32_t* vtCount, uint32_t* eeCount) {
  std::sort(triangles.begin(), triangles.end());
  triangles.erase(std::unique(triangles.begin(), triangles.end()), triangles.end());
  std::vector<std::array<uint32_t, 2>> edges;
  for (const auto& t : triangles) {
    const uint32_t pairs[3][2] = {{t[0], t[1]}, {t[1], t[2]}, {t[2], t[0]}};
    for (const auto& p : pairs) edges.push_back({std::min(p[0], p[1]), std::max(p[0], p[1])});
  }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  std::vector<std::vector<uint32_t>> ring(V);
  for (const auto& e : edges) {
    ring[e[0]].push_back(e[1]);
    ring[e[1]].push_back(e[0]);
  }
  for (auto& r : ring) std::sort(r.begin(), r.end());
  auto closed = [&](uint32_t a, uint32_t b) {
    return a == b || std::binary_search(ring[a].begin(), ring[a].end(), b);
  };
  out->clear();
  uint32_t vt = 0;
  for (uint32_t v = 0; v < V; ++v)
    for (const auto& t : triangles) {
      if (closed(v, t[0]) || closed(v, t[1]) || closed(v, t[2])) continue;
      out->insert(out->end(), {v, t[0], t[1], t[2]});
      vt++;
    }
  uint32_t ee = 0;
  for (size_t i = 0; i < edges.size(); ++i)
    for (size_t j = i + 1; j < edges.size(); ++j) {
      const auto& a = edges[i];
      const auto& b = edges[j];
      if (closed(a[0], b[0]) || closed(a[0], b[1]) || closed(a[1], b[0]) || closed(a[1], b[1])) continue;
      out->insert(out->end(), {a[0], a[1], b[0], b[1]});
      ee++;
    }
  *vtCount = vt;
  *eeCount = ee;
}

// Hinges of buildJGS2GpuClothInput (src/scenes/index.ts:893-933): every
// interior edge shared by two consistently oriented triangles gives one
// hinge (first, second, opposite of the first triangle, opposite of the
// second); an edge with three triangles or opposite windings is an error.
bool buildHinges(const std::vector<uint32_t>& triangles, std::vector<uint32_t>* hinges, std::string* err) {
  struct HalfEdge { uint32_t first, second, opposite; };
  std::unordered_map<uint64_t, HalfEdge> open;
  std::unordered_map<uint64_t, bool> closed;
  auto add = [&](uint32_t a, uint32_t b, uint32_t o) {
    const uint64_t key = (static_cast<uint64_t>(std::min(a, b)) << 32) | std::max(a, b);
    const std::string name = std::to_string(std::min(a, b)) + ":" + std::to_string(std::max(a, b));
    if (closed.count(key)) { *err = "Cloth edge " + name + " is non-manifold."; return false; }
    auto it = open.find(key);
    if (it == open.end()) { open.emplace(key, HalfEdge{a, b, o}); return true; }
    const HalfEdge prev = it->second;
    if (prev.first != b || prev.second != a) {
      *err = "Cloth triangles sharing edge " + name + " must have consistent orientation.";
      return false;
    }
    hinges->insert(hinges->end(), {prev.first, prev.second, prev.opposite, o});
    open.erase(it);
    closed.emplace(key, true);
    return true;
  };
  for (size_t c = 0; c < triangles.size() / 3; ++c) {
    const uint32_t i0 = triangles[3 * c], i1 = triangles[3 * c + 1], i2 = triangles[3 * c + 2];
    if (!add(i0, i1, i2) || !add(i1, i2, i0) || !add(i2, i0, i1)) return false;
  }
  return true;
}

void invalidate(Scene& s) {
  s.restValid = false;
  s.precomputed = false;
}

}  // namespace

extern "C" {

jgs2_scene* jgs2_scene_new(void) { return new (std::nothrow) jgs2_scene(); }

void jgs2_scene_destroy(jgs2_scene* scene) { delete scene; }

const char* jgs2_scene_last_error(const jgs2_scene* scene) {
  return scene ? scene->error.c_str() : "null scene";
}

void jgs2_default_precompute_options(jgs2_precompute_options* out) {
  if (!out) return;
  out->timestep = 1.0 / 60.0;
  out->cubature_k = 6;
  out->method = JGS2_PRECOMPUTE_EXACT;
  out->patch_radius = 2;
  out->threads = 0;
  out->mode_count = 8;
  out->inverse_iterations = 24;
  out->training_amplitude = 0.12;
  out->refinement_passes = 12;
  out->exact_complement = 0;
  out->selection_device = JGS2_SELECTION_AUTO;
}

int32_t jgs2_scene_add_material(jgs2_scene* s, double density, double young, double poisson,
                                uint32_t model) {
  if (!s) return -1;
  // validateMaterial (src/simulation/cpu/fem.ts:13-36) and the stable
  // Poisson range (src/simulation/cpu/stable-neo-hookean.ts:77-86).
  if (!(density > 0) || !std::isfinite(density)) return fail(s, "Material has invalid density."), -1;
  if (!(young > 0) || !std::isfinite(young)) return fail(s, "Material has invalid Young's modulus."), -1;
  if (!(poisson > -1 && poisson < 0.5)) return fail(s, "Material has invalid Poisson ratio."), -1;
  if (model != JGS2_MATERIAL_COROTATED_LINEAR && model != JGS2_MATERIAL_STABLE_NEO_HOOKEAN)
    return fail(s, "Material has invalid model."), -1;
  if (model == JGS2_MATERIAL_STABLE_NEO_HOOKEAN && !(poisson >= 0))
    return fail(s, "Stable Neo-Hookean material requires Poisson ratio in [0, 0.5)."), -1;
  s->materialTable.push_back({density, young, poisson, model});
  return static_cast<int32_t>(s->materialTable.size() - 1);
}

int64_t jgs2_scene_add_cuboid(jgs2_scene* s, const uint32_t cells[3], const double origin[3],
                              const double size[3], uint32_t material, uint32_t body,
                              uint32_t pinned_faces) {
  if (!s || !cells || !origin || !size) return -1;
  for (int i = 0; i < 3; ++i) {
    if (cells[i] < 1) return fail(s, "cells must be positive integers."), -1;
    if (!(size[i] > 0) || !std::isfinite(size[i]))
      return fail(s, "Cuboid dimensions must be finite and positive."), -1;
  }
  if (material >= s->materialTable.size()) return fail(s, "Unknown material id."), -1;
  const uint64_t nx = cells[0], ny = cells[1], nz = cells[2];
  const uint64_t V = (nx + 1) * (ny + 1) * (nz + 1);
  const uint64_t T = nx * ny * nz * 6;
  const uint64_t base = s->mesh.vertexCount();
  if (base + V > 0xfffffff0ull || s->mesh.tetCount() + T > 0xfffffff0ull)
    return fail(s, "Scene exceeds 32-bit index space."), -1;
  std::vector<double> pos(3 * V);
  std::vector<uint8_t> fixed(V);
  const uint64_t sy = nx + 1, sz = sy * (ny + 1);
  for (uint64_t z = 0; z <= nz; ++z)
    for (uint64_t y = 0; y <= ny; ++y)
      for (uint64_t x = 0; x <= nx; ++x) {
        const uint64_t v = x + y * sy + z * sz;
        // generateRegularCuboidMesh vertex placement (mesh.ts:139-147).
        pos[3 * v] = origin[0] + (size[0] * static_cast<double>(x)) / static_cast<double>(nx);
        pos[3 * v + 1] = origin[1] + (size[1] * static_cast<double>(y)) / static_cast<double>(ny);
        pos[3 * v + 2] = origin[2] + (size[2] * static_cast<double>(z)) / static_cast<double>(nz);
        bool f = false;
        if ((pinned_faces & JGS2_FACE_X_MIN) && x == 0) f = true;
        if ((pinned_faces & JGS2_FACE_X_MAX) && x == nx) f = true;
        if ((pinned_faces & JGS2_FACE_Y_MIN) && y == 0) f = true;
        if ((pinned_faces & JGS2_FACE_Y_MAX) && y == ny) f = true;
        if ((pinned_faces & JGS2_FACE_Z_MIN) && z == 0) f = true;
        if ((pinned_faces & JGS2_FACE_Z_MAX) && z == nz) f = true;
        fixed[v] = f ? 1 : 0;
      }
  std::vector<uint32_t> tets(4 * T);
  uint64_t o = 0;
  for (uint64_t z = 0; z < nz; ++z)
    for (uint64_t y = 0; y < ny; ++y)
      for (uint64_t x = 0; x < nx; ++x) {
        auto vi = [&](uint64_t a, uint64_t b, uint64_t c) {
          return static_cast<uint32_t>(a + b * sy + c * sz);
        };
        const uint32_t v000 = vi(x, y, z), v100 = vi(x + 1, y, z), v010 = vi(x, y + 1, z),
                       v110 = vi(x + 1, y + 1, z), v001 = vi(x, y, z + 1),
                       v101 = vi(x + 1, y, z + 1), v011 = vi(x, y + 1, z + 1),
                       v111 = vi(x + 1, y + 1, z + 1);
        // Six tetrahedra around the v000-v111 diagonal (mesh.ts:164-189).
        const uint32_t cell[24] = {v000, v100, v110, v111, v000, v110, v010, v111,
                                   v000, v010, v011, v111, v000, v011, v001, v111,
                                   v000, v001, v101, v111, v000, v101, v100, v111};
        std::memcpy(&tets[o], cell, sizeof(cell));
        o += 24;
      }
  std::string err;
  if (!orientTets(pos, tets.data(), T, &err)) return fail(s, err), -1;
  auto& m = s->mesh;
  m.positions.insert(m.positions.end(), pos.begin(), pos.end());
  for (auto& t : tets) t += static_cast<uint32_t>(base);
  m.tets.insert(m.tets.end(), tets.begin(), tets.end());
  m.materials.insert(m.materials.end(), T, material);
  m.fixed.insert(m.fixed.end(), fixed.begin(), fixed.end());
  m.bodies.insert(m.bodies.end(), V, body);
  invalidate(*s);
  return static_cast<int64_t>(base);
}

int64_t jgs2_scene_add_mesh(jgs2_scene* s, uint32_t vertex_count, const double* positions,
                            uint32_t tet_count, const uint32_t* tets,
                            const uint32_t* tet_materials, uint32_t material,
                            const uint8_t* pinned, uint32_t body) {
  if (!s || !positions || !tets || vertex_count == 0 || tet_count == 0) return -1;
  const uint64_t base = s->mesh.vertexCount();
  std::vector<double> pos(positions, positions + 3ull * vertex_count);
  for (double v : pos)
    if (!std::isfinite(v)) return fail(s, "Mesh positions must be finite."), -1;
  std::vector<uint32_t> q(tets, tets + 4ull * tet_count);
  for (uint32_t v : q)
    if (v >= vertex_count) return fail(s, "Tetrahedron vertex is out of range."), -1;
  std::string err;
  if (!orientTets(pos, q.data(), tet_count, &err)) return fail(s, err), -1;
  for (uint32_t t = 0; t < tet_count; ++t) {
    const uint32_t mid = tet_materials ? tet_materials[t] : material;
    if (mid >= s->materialTable.size()) return fail(s, "Unknown material id."), -1;
  }
  auto& m = s->mesh;
  m.positions.insert(m.positions.end(), pos.begin(), pos.end());
  for (auto& v : q) v += static_cast<uint32_t>(base);
  m.tets.insert(m.tets.end(), q.begin(), q.end());
  for (uint32_t t = 0; t < tet_count; ++t)
    m.materials.push_back(tet_materials ? tet_materials[t] : material);
  for (uint32_t v = 0; v < vertex_count; ++v) m.fixed.push_back(pinned ? (pinned[v] ? 1 : 0) : 0);
  m.bodies.insert(m.bodies.end(), vertex_count, body);
  invalidate(*s);
  return static_cast<int64_t>(base);
}

int64_t jgs2_scene_add_cloth(jgs2_scene* s, uint32_t vertex_count, const double* positions,
                             uint32_t triangle_count, const uint32_t* triangles, const uint8_t* pinned,
                             uint32_t body, double density, double young_modulus, double poisson_ratio,
                             double thickness, double bending_stiffness) {
  if (!s || !positions || !triangles || vertex_count == 0 || triangle_count == 0) return -1;
  // validateAndAddClothMasses (src/simulation/cpu/precompute.ts:44-78).
  if (!(density > 0) || !std::isfinite(density)) return fail(s, "Cloth density must be finite and positive."), -1;
  if (!(young_modulus > 0) || !std::isfinite(young_modulus))
    return fail(s, "Cloth youngModulus must be finite and positive."), -1;
  if (!(thickness > 0) || !std::isfinite(thickness))
    return fail(s, "Cloth thickness must be finite and positive."), -1;
  if (!std::isfinite(poisson_ratio) || poisson_ratio < 0 || poisson_ratio >= 0.5)
    return fail(s, "Cloth poissonRatio must be in [0, 0.5)."), -1;
  if (!std::isfinite(bending_stiffness) || bending_stiffness < 0)
    return fail(s, "Cloth bendingStiffness must be finite and nonnegative."), -1;
  Cloth& c = s->cloth;
  if (c.present && (c.density != density || c.young != young_modulus || c.poisson != poisson_ratio ||
                    c.thickness != thickness || c.bending != bending_stiffness))
    return fail(s, "A scene holds one cloth material; a second sheet must use the same one."), -1;
  const uint64_t base = s->mesh.vertexCount();
  if (base + vertex_count > 0xfffffff0ull) return fail(s, "Scene exceeds 32-bit index space."), -1;
  std::vector<double> pos(positions, positions + 3ull * vertex_count);
  for (double v : pos)
    if (!std::isfinite(v)) return fail(s, "Cloth positions must be finite."), -1;
  std::vector<uint32_t> tri(triangles, triangles + 3ull * triangle_count);
  for (uint32_t t = 0; t < triangle_count; ++t) {
    const uint32_t a = tri[3ull * t], b = tri[3ull * t + 1], d = tri[3ull * t + 2];
    if (a >= vertex_count || b >= vertex_count || d >= vertex_count || a == b || a == d || b == d)
      return fail(s, "Cloth triangle " + std::to_string(t) + " has invalid vertex indices."), -1;
  }
  auto& m = s->mesh;
  m.positions.insert(m.positions.end(), pos.begin(), pos.end());
  for (uint32_t v = 0; v < vertex_count; ++v) m.fixed.push_back(pinned ? (pinned[v] ? 1 : 0) : 0);
  m.bodies.insert(m.bodies.end(), vertex_count, body);
  for (auto& v : tri) v += static_cast<uint32_t>(base);
  c.triangles.insert(c.triangles.end(), tri.begin(), tri.end());
  c.present = true;
  c.density = density;
  c.young = young_modulus;
  c.poisson = poisson_ratio;
  c.thickness = thickness;
  c.bending = bending_stiffness;
  invalidate(*s);
  return static_cast<int64_t>(base);
}

jgs2_status jgs2_scene_set_rest_positions(jgs2_scene* s, const double* positions) {
  if (!s || !positions) return JGS2_INVALID_ARGUMENT;
  const size_t n = 3ull * s->mesh.vertexCount();
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(positions[i])) return fail(s, "Rest positions must be finite."), JGS2_INVALID_ARGUMENT;
  std::vector<double> pos(positions, positions + n);
  std::vector<uint32_t> tets = s->mesh.tets;
  std::string err;
  // transformTetrahedralMesh re-orients the tetrahedra (mesh.ts:272-273).
  if (!orientTets(pos, tets.data(), tets.size() / 4, &err)) return fail(s, err), JGS2_INVALID_ARGUMENT;
  s->mesh.positions = std::move(pos);
  s->mesh.tets = std::move(tets);
  invalidate(*s);
  return JGS2_OK;
}

int64_t jgs2_build_static_contact_candidates(uint32_t vertex_count, const uint32_t* triangles,
                                             uint32_t triangle_count, uint32_t* out, uint64_t capacity,
                                             uint32_t* vertex_triangle_count, uint32_t* edge_edge_count) {
  if ((!triangles && triangle_count) || !vertex_triangle_count || !edge_edge_count) return -1;
  std::vector<std::array<uint32_t, 3>> tri(triangle_count);
  for (uint32_t t = 0; t < triangle_count; ++t) {
    std::array<uint32_t, 3> s = {triangles[3ull * t], triangles[3ull * t + 1], triangles[3ull * t + 2]};
    std::sort(s.begin(), s.end());
    if (s[2] >= vertex_count || s[0] == s[1] || s[1] == s[2]) return -1;
    tri[t] = s;
  }
  std::vector<uint32_t> packed;
  staticContactCandidates(vertex_count, std::move(tri), &packed, vertex_triangle_count, edge_edge_count);
  const uint64_t n = packed.size() / 4;
  if (out && capacity >= n) std::memcpy(out, packed.data(), packed.size() * sizeof(uint32_t));
  return static_cast<int64_t>(n);
}

jgs2_status jgs2_scene_set_contact(jgs2_scene* s, uint32_t mode) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  if (mode > JGS2_SCENE_CONTACT_SURFACE) return fail(s, "Unknown contact mode."), JGS2_INVALID_ARGUMENT;
  s->contact = mode;
  return JGS2_OK;
}

jgs2_status jgs2_scene_set_contact_capacity(jgs2_scene* s, uint64_t capacity) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  s->contactCapacity = capacity;
  return JGS2_OK;
}

uint32_t jgs2_scene_cloth_triangle_count(const jgs2_scene* s) {
  return s ? static_cast<uint32_t>(s->cloth.triangles.size() / 3) : 0;
}

jgs2_status jgs2_scene_set_pinned(jgs2_scene* s, const uint8_t* pinned) {
  if (!s || !pinned) return JGS2_INVALID_ARGUMENT;
  for (uint32_t v = 0; v < s->mesh.vertexCount(); ++v) s->mesh.fixed[v] = pinned[v] ? 1 : 0;
  s->precomputed = false;
  return JGS2_OK;
}

uint32_t jgs2_scene_vertex_count(const jgs2_scene* s) { return s ? s->mesh.vertexCount() : 0; }
uint32_t jgs2_scene_tet_count(const jgs2_scene* s) { return s ? s->mesh.tetCount() : 0; }

jgs2_status jgs2_scene_rest_positions(const jgs2_scene* s, double* out) {
  if (!s || !out) return JGS2_INVALID_ARGUMENT;
  std::memcpy(out, s->mesh.positions.data(), s->mesh.positions.size() * sizeof(double));
  return JGS2_OK;
}

jgs2_status jgs2_scene_precompute(jgs2_scene* s, const jgs2_precompute_options* options,
                                  jgs2_precompute_stats* stats) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  jgs2_precompute_options opt;
  jgs2_default_precompute_options(&opt);
  if (options) opt = *options;
  if (s->mesh.tetCount() == 0) return fail(s, "Scene has no tetrahedra."), JGS2_INVALID_ARGUMENT;
  if (!(opt.timestep > 0) || !std::isfinite(opt.timestep))
    return fail(s, "The timestep must be finite and positive."), JGS2_INVALID_ARGUMENT;
  if (opt.cubature_k < 1) return fail(s, "cubature_k must be positive."), JGS2_INVALID_ARGUMENT;
  if (opt.selection_device > JGS2_SELECTION_AUTO)
    return fail(s, "selection_device must be JGS2_SELECTION_CPU, _GPU or _AUTO."), JGS2_INVALID_ARGUMENT;
  if (opt.method > JGS2_PRECOMPUTE_PATCH) return fail(s, "Unknown precompute method."), JGS2_INVALID_ARGUMENT;
  if (!computeRest(*s)) return JGS2_INVALID_ARGUMENT;
  try {
    if (!runPrecompute(*s, opt, stats)) return JGS2_INVALID_ARGUMENT;
  } catch (const std::bad_alloc&) {
    return fail(s, "Precompute ran out of host memory."), JGS2_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    return fail(s, e.what()), JGS2_INVALID_ARGUMENT;
  }
  s->precomputed = true;
  return JGS2_OK;
}

jgs2_status jgs2_scene_set_initial_state(jgs2_scene* s, const float* positions,
                                         const float* velocities, uint32_t pin_at_initial) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  const size_t V = s->mesh.vertexCount();
  if (positions) s->initialPositions.assign(positions, positions + 4 * V);
  else s->initialPositions.clear();
  if (velocities) s->initialVelocities.assign(velocities, velocities + 4 * V);
  else s->initialVelocities.clear();
  s->pinAtInitial = pin_at_initial != 0;
  return JGS2_OK;
}

jgs2_status jgs2_scene_set_objectives(jgs2_scene* s, const float* forces, const float* targets,
                                      const float* stiffnesses) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  const size_t V = s->mesh.vertexCount();
  if ((targets == nullptr) != (stiffnesses == nullptr))
    return fail(s, "objectives.targetPositions and objectives.targetStiffnesses must be provided together."),
           JGS2_INVALID_ARGUMENT;
  if (forces) s->externalForces.assign(forces, forces + 3 * V); else s->externalForces.clear();
  if (targets) {
    s->targetPositions.assign(targets, targets + 3 * V);
    s->targetStiffnesses.assign(stiffnesses, stiffnesses + V);
  } else {
    s->targetPositions.clear();
    s->targetStiffnesses.clear();
  }
  return JGS2_OK;
}

jgs2_status jgs2_scene_pack(jgs2_scene* s, jgs2_input* out) {
  if (!s || !out) return JGS2_INVALID_ARGUMENT;
  if (!s->precomputed) return fail(s, "Scene precompute has not run."), JGS2_INVALID_ARGUMENT;
  const auto& m = s->mesh;
  const uint32_t V = m.vertexCount(), T = m.tetCount(), K = s->cubatureK;
  // buildAdjacency (src/scenes/index.ts:811-837): incident tets per vertex
  // in ascending tet order.
  std::vector<uint32_t> counts(V, 0), starts(V, 0);
  for (uint32_t v : m.tets) counts[v] += 1;
  uint64_t total = 0;
  for (uint32_t v = 0; v < V; ++v) { starts[v] = static_cast<uint32_t>(total); total += counts[v]; }
  s->packAdjacency.assign(total, 0);
  {
    std::vector<uint32_t> cursor(starts);
    for (uint32_t t = 0; t < T; ++t)
      for (int l = 0; l < 4; ++l) s->packAdjacency[cursor[m.tets[4ull * t + l]]++] = t;
  }
  s->packPositions.assign(4ull * V, 0.f);
  s->packRest.assign(4ull * V, 0.f);
  s->packInfo.assign(4ull * V, 0u);
  s->packColors.assign(4ull * V, 1.f);
  const bool haveInit = s->initialPositions.size() == 4ull * V;
  for (uint32_t v = 0; v < V; ++v) {
    for (int c = 0; c < 3; ++c) {
      const float restValue = static_cast<float>(m.positions[3ull * v + c]);
      const float init = haveInit ? s->initialPositions[4ull * v + c] : restValue;
      s->packPositions[4ull * v + c] = init;
      s->packRest[4ull * v + c] = (s->pinAtInitial && m.fixed[v]) ? init : restValue;
    }
    s->packPositions[4ull * v + 3] = 1.f;
    s->packRest[4ull * v + 3] = static_cast<float>(s->masses[v]);
    s->packInfo[4ull * v] = starts[v];
    s->packInfo[4ull * v + 1] = counts[v];
    s->packInfo[4ull * v + 2] = m.fixed[v];
    s->packInfo[4ull * v + 3] = m.bodies[v];
  }
  if (s->initialVelocities.size() == 4ull * V) {
    s->packVelocities = s->initialVelocities;
    for (uint32_t v = 0; v < V; ++v) s->packVelocities[4ull * v + 3] = 0.f;
  } else {
    s->packVelocities.clear();
  }
  s->packTetIndices = m.tets;
  s->packInverseDm.assign(12ull * T, 0.f);
  s->packMeta.assign(4ull * T, 0.f);
  bool anyCorotated = false;
  for (uint32_t t = 0; t < T; ++t) {
    // Padded column-major inverse Dm (src/scenes/index.ts:1034-1043).
    for (int col = 0; col < 3; ++col)
      for (int row = 0; row < 3; ++row)
        s->packInverseDm[12ull * t + col * 4 + row] =
            static_cast<float>(s->rest.inverseRest[9ull * t + row * 3 + col]);
    const Material& mat = s->materialTable[m.materials[t]];
    double lambda, mu;
    if (mat.model == JGS2_MATERIAL_STABLE_NEO_HOOKEAN) stableLame(mat, &lambda, &mu);
    else { hookeLame(mat, &lambda, &mu); anyCorotated = true; }
    s->packMeta[4ull * t] = static_cast<float>(s->rest.volumes[t]);
    s->packMeta[4ull * t + 1] = static_cast<float>(lambda);
    s->packMeta[4ull * t + 2] = static_cast<float>(mu);
    s->packMeta[4ull * t + 3] = static_cast<float>(mat.model);
  }
  if (anyCorotated) {
    s->packStiffness.assign(144ull * T, 0.f);
    double k[144];
    for (uint32_t t = 0; t < T; ++t) {
      linearStiffness(&s->rest.inverseRest[9ull * t], s->rest.volumes[t],
                      s->materialTable[m.materials[t]], k);
      for (int i = 0; i < 144; ++i) s->packStiffness[144ull * t + i] = static_cast<float>(k[i]);
    }
  } else {
    s->packStiffness.clear();
  }
  // buildJGS2GpuClothInput (src/scenes/index.ts:881-973): rest bases, areas,
  // hinges and rest dihedrals in double, stored as f32.
  const bool cloth = s->cloth.present;
  if (cloth) {
    const auto& tri = s->cloth.triangles;
    const size_t C = tri.size() / 3;
    s->packClothTriangles = tri;
    s->packClothInverse.assign(4 * C, 0.f);
    s->packClothAreas.assign(C, 0.f);
    const auto& p = m.positions;
    for (size_t c = 0; c < C; ++c) {
      double inv[4], area;
      if (!clothTriangleRest(&p[3ull * tri[3 * c]], &p[3ull * tri[3 * c + 1]], &p[3ull * tri[3 * c + 2]], inv, &area))
        return fail(s, "Rest triangle must be nondegenerate."), JGS2_INVALID_ARGUMENT;
      for (int k = 0; k < 4; ++k) s->packClothInverse[4 * c + k] = static_cast<float>(inv[k]);
      s->packClothAreas[c] = static_cast<float>(area);
    }
    std::vector<uint32_t> hinges;
    std::string err;
    if (!buildHinges(tri, &hinges, &err)) return fail(s, err), JGS2_INVALID_ARGUMENT;
    const size_t H = hinges.size() / 4;
    s->packHinges = hinges;
    s->packHingeAngles.assign(H, 0.f);
    s->packHingeLengths.assign(H, 0.f);
    for (size_t h = 0; h < H; ++h) {
      const uint32_t* q = &hinges[4 * h];
      double angle, length;
      if (!clothHingeRest(&p[3ull * q[0]], &p[3ull * q[1]], &p[3ull * q[2]], &p[3ull * q[3]], &angle, &length))
        return fail(s, "First hinge triangle must be nondegenerate."), JGS2_INVALID_ARGUMENT;
      s->packHingeAngles[h] = static_cast<float>(angle);
      s->packHingeLengths[h] = static_cast<float>(length);
    }
    jgs2_cloth_input& ci = s->packCloth;
    std::memset(&ci, 0, sizeof(ci));
    ci.vertex_count = V;
    ci.triangle_count = static_cast<uint32_t>(C);
    ci.hinge_count = static_cast<uint32_t>(H);
    ci.triangle_indices = s->packClothTriangles.data();
    ci.triangle_inverse_rest_bases = s->packClothInverse.data();
    ci.triangle_rest_areas = s->packClothAreas.data();
    ci.hinge_indices = H ? s->packHinges.data() : nullptr;
    ci.hinge_rest_angles = H ? s->packHingeAngles.data() : nullptr;
    ci.hinge_rest_edge_lengths = H ? s->packHingeLengths.data() : nullptr;
    ci.young_modulus = static_cast<float>(s->cloth.young);
    ci.poisson_ratio = static_cast<float>(s->cloth.poisson);
    ci.thickness = static_cast<float>(s->cloth.thickness);
    ci.bending_stiffness = static_cast<float>(s->cloth.bending);
  }
  // Static IPC candidates over the tet boundary and the cloth triangles
  // (surfaceWithCloth, precompute.ts:98-140; buildStaticIpcContactCandidates).
  s->packContact.clear();
  s->packContactVT = s->packContactEE = 0;
  s->packSurface.clear();
  if (s->contact != JGS2_SCENE_CONTACT_NONE) {
    std::vector<std::array<uint32_t, 3>> surface;
    std::string err;
    if (!boundaryTriangles(m, &surface, &err)) return fail(s, err), JGS2_INVALID_ARGUMENT;
    if (cloth)
      for (size_t c = 0; c < s->cloth.triangles.size() / 3; ++c) {
        std::array<uint32_t, 3> t = {s->cloth.triangles[3 * c], s->cloth.triangles[3 * c + 1],
                                     s->cloth.triangles[3 * c + 2]};
        std::sort(t.begin(), t.end());
        surface.push_back(t);
      }
    if (s->contact == JGS2_SCENE_CONTACT_STATIC) {
      staticContactCandidates(V, std::move(surface), &s->packContact, &s->packContactVT, &s->packContactEE);
    } else {
      std::sort(surface.begin(), surface.end());
      surface.erase(std::unique(surface.begin(), surface.end()), surface.end());
      for (const auto& t : surface) s->packSurface.insert(s->packSurface.end(), t.begin(), t.end());
      s->packSurfaceRec = jgs2_contact_surface{};
      s->packSurfaceRec.triangle_count = static_cast<uint32_t>(surface.size());
      s->packSurfaceRec.triangles = s->packSurface.data();
      s->packSurfaceRec.candidate_capacity = s->contactCapacity;
    }
  }
  std::memset(out, 0, sizeof(*out));
  out->cloth = cloth ? &s->packCloth : nullptr;
  out->contact_indices = s->packContact.empty() ? nullptr : s->packContact.data();
  out->contact_vertex_triangle_count = s->packContactVT;
  out->contact_edge_edge_count = s->packContactEE;
  out->contact_surface = s->contact == JGS2_SCENE_CONTACT_SURFACE ? &s->packSurfaceRec : nullptr;
  out->vertex_count = V;
  out->tet_count = T;
  out->cubature_k = K;
  out->positions = s->packPositions.data();
  out->velocities = s->packVelocities.empty() ? nullptr : s->packVelocities.data();
  out->vertex_rest = s->packRest.data();
  out->vertex_colors = s->packColors.data();
  out->vertex_info = s->packInfo.data();
  out->external_forces = s->externalForces.empty() ? nullptr : s->externalForces.data();
  out->target_positions = s->targetPositions.empty() ? nullptr : s->targetPositions.data();
  out->target_stiffnesses = s->targetStiffnesses.empty() ? nullptr : s->targetStiffnesses.data();
  out->tet_indices = s->packTetIndices.data();
  out->tet_inverse_dm = s->packInverseDm.data();
  out->tet_meta = s->packMeta.data();
  out->tet_rest_stiffness = s->packStiffness.empty() ? nullptr : s->packStiffness.data();
  out->adjacency = s->packAdjacency.data();
  out->adjacency_length = s->packAdjacency.size();
  out->cubature_tet_ids = s->recordTets.data();
  out->cubature_weights = s->recordWeights.data();
  out->cubature_basis = s->recordBasis.data();
  return JGS2_OK;
}

}  // extern "C"
