// JGS2 step oracle — TEST INFRASTRUCTURE, not product code.
//
// A CPU restatement of the reference's WGSL step, used only by tests/, by
// __graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline leg.
// It follows the WGSL kernels function by function in the reference's dispatch
// order (src/simulation/gpu/jgs2-solver.ts:2207-2494):
//   predict               jgs2-shader.ts:2660-2692
//   tetPolarRotation      jgs2-shader.ts:2931-2957
//   vertexPolarRotation   jgs2-shader.ts:2959-2989
//   jgs2Solve             jgs2-shader.ts:2991-3487 (+ helpers :1062-2512)
//   assembledVertexEnergy jgs2-shader.ts:3489-3496, 2557-2658
//   candidateTetrahedron  jgs2-shader.ts:3498-3601
//   reduceCandidate       jgs2-shader.ts:3611-3955 (128-lane stride + tree order)
//   applyCandidate        jgs2-shader.ts:3957-3983
//   convergenceGradient   jgs2-shader.ts:3985-4097
//   reduceConvergence     jgs2-shader.ts:4105-4486 (128-lane stride + tree order)
//   copyPosition          jgs2-shader.ts:4488-4496
//   bodyHorizontalCorrection / apply  jgs2-shader.ts:4498-4551
//   finalize              jgs2-shader.ts:4553-4589
// with the stable Neo-Hookean library (stable-neo-hookean-wgsl.ts:14-95) and
// the globalization library (jgs2-globalization-wgsl.ts:26-560).
//
// Scalar = float is the "WGSL-order mirror" (f32 everywhere, the same
// operation order as the shader source, no fused multiply-add); Scalar =
// double is the FP64 run of the same method used for error statements.
// Parity of this restatement with the reference is pinned only at the
// tolerance level: the reference runs in a browser WebGPU stack that cannot
// run here, so bitwise f32 agreement with WGSL is not claimed.
//
// The restatement is pinned to the known answers of the reference's own
// tests, through the test entry points at the end of this file:
// - the stable Neo-Hookean density (stable-neo-hookean.test.ts);
// - the local globalization solve and its shift cases
//   (nonlinear-globalization.test.ts, nonlinear-globalization-gpu.spec.ts);
// - the convergence reduction (nonlinear-iteration.test.ts);
// - the assembled gate (nonlinear-globalization-gpu.spec.ts);
// - IPC barrier, friction and distances (ipc-contact.test.ts);
// - cloth elements (cloth.test.ts);
// - the local system's dense projections (precompute.test.ts,
//   nonlinear-restricted-energy.test.ts);
// - vertex frames, force-free momentum, and the schedule comparison
//   (the e2e specs).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "jgs2.h"

namespace {

template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
V3<T> v3(T x, T y, T z) { return {x, y, z}; }
template <class T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> T comp(V3<T> a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
template <class T> void setComp(V3<T>& a, int i, T v) { (i == 0 ? a.x : (i == 1 ? a.y : a.z)) = v; }

// WGSL mat3x3f: three columns.
template <class T>
struct M3 {
  V3<T> c[3];
};
template <class T> M3<T> zeroM() { return {{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}}; }
template <class T> M3<T> identityM() { return {{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}; }
template <class T> M3<T> operator+(const M3<T>& a, const M3<T>& b) {
  return {{a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]}};
}
template <class T> M3<T> operator-(const M3<T>& a, const M3<T>& b) {
  return {{a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]}};
}
template <class T> M3<T> operator*(T s, const M3<T>& a) { return {{s * a.c[0], s * a.c[1], s * a.c[2]}}; }
template <class T> V3<T> operator*(const M3<T>& m, V3<T> v) {
  return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}
template <class T> M3<T> operator*(const M3<T>& a, const M3<T>& b) {
  return {{a * b.c[0], a * b.c[1], a * b.c[2]}};
}
template <class T> M3<T> transpose(const M3<T>& m) {
  return {{{m.c[0].x, m.c[1].x, m.c[2].x}, {m.c[0].y, m.c[1].y, m.c[2].y}, {m.c[0].z, m.c[1].z, m.c[2].z}}};
}
template <class T> T at(const M3<T>& m, int col, int row) { return comp(m.c[col], row); }
template <class T> M3<T> outerColumns(V3<T> l, V3<T> r) { return {{l * r.x, l * r.y, l * r.z}}; }

template <class T>
struct V4 {
  T x, y, z, w;
};

// ---- constants (jgs2-globalization-wgsl.ts:27-37, jgs2-shader.ts:64-118) ----
constexpr float kF32Max = 3.0e38f;
constexpr float kUnitRoundoff = 0.000000059604644775390625f;
constexpr float kPositionResolutionMultiplier = 8.0f;
constexpr float kRelativeEigenvalueFloor = 0.0000152587890625f;
constexpr float kMaxNormalizedShift = 0.001f;
constexpr float kArmijoC1 = 0.0001f;
constexpr float kBacktrackFactor = 0.5f;
constexpr uint32_t kMaxBacktracks = 12;
constexpr uint32_t kTrialCount = 13;
constexpr float kDeterminantFloor = 0.0001f;
constexpr double kTwoPiOverThree = 2.0943951023931953;
constexpr uint32_t kEmptyTet = 0xffffffffu;
constexpr uint32_t kWorkgroup = 128;
constexpr uint32_t kHistoryCapacity = 64;

enum : uint32_t {
  kStatusAccepted = 0, kStatusPinned = 1, kStatusZeroGradient = 2, kStatusShiftLimit = 3,
  kStatusNonDescent = 4, kStatusLineSearchFailed = 5, kStatusNonfinite = 6, kStatusCholeskyFailed = 7,
};
enum : uint32_t {
  kSourceGeometryValid = 1, kCandidateGeometryValid = 2, kAcceptedMinimumValid = 4,
  kLocalNumericsValid = 8, kValidityMask = 15, kStopLatch = 16, kControlMask = 31,
  kSourceEnergyValid = 16, kCandidateEnergyValid = 32,
  kReductionMask = 1 | 2 | 8 | 16 | 32,
};

template <class T> bool finiteS(T v) { return v == v && std::fabs(v) <= static_cast<T>(kF32Max); }
template <class T> bool finiteV(V3<T> v) { return finiteS(v.x) && finiteS(v.y) && finiteS(v.z); }
template <class T> bool finiteM(const M3<T>& m) { return finiteV(m.c[0]) && finiteV(m.c[1]) && finiteV(m.c[2]); }
template <class T> bool finite4(V4<T> v) { return finiteS(v.x) && finiteS(v.y) && finiteS(v.z) && finiteS(v.w); }
template <class T> T det(const M3<T>& m) { return dot(m.c[0], cross(m.c[1], m.c[2])); }
template <class T> T frob(const M3<T>& a, const M3<T>& b) {
  return dot(a.c[0], b.c[0]) + dot(a.c[1], b.c[1]) + dot(a.c[2], b.c[2]);
}

// ---- stable Neo-Hookean (stable-neo-hookean-wgsl.ts:14-95) ----
template <class T> M3<T> cofactor(const M3<T>& f) {
  return {{cross(f.c[1], f.c[2]), cross(f.c[2], f.c[0]), cross(f.c[0], f.c[1])}};
}
template <class T> M3<T> directionalCofactor(const M3<T>& f, const M3<T>& h) {
  return {{cross(h.c[1], f.c[2]) + cross(f.c[1], h.c[2]), cross(h.c[2], f.c[0]) + cross(f.c[2], h.c[0]),
           cross(h.c[0], f.c[1]) + cross(f.c[0], h.c[1])}};
}
template <class T> T snhEnergy(const M3<T>& f, T lambda, T mu) {
  const T I1 = frob(f, f);
  const T dj = det(f) - T(1);
  return T(0.5) * mu * (I1 - T(3)) - T(0.75) * mu * dj + T(0.5) * lambda * dj * dj -
         T(0.5) * mu * std::log((I1 + T(1)) * T(0.25));
}
template <class T> M3<T> snhPiola(const M3<T>& f, T lambda, T mu) {
  const T I1 = frob(f, f);
  const T den = I1 + T(1);
  const M3<T> cof = cofactor(f);
  const T shear = mu * (T(1) - T(1) / den);
  const T volume = lambda * (det(f) - T(1)) - T(0.75) * mu;
  return shear * f + volume * cof;
}
template <class T> M3<T> snhTangent(const M3<T>& f, const M3<T>& h, T lambda, T mu) {
  const T I1 = frob(f, f);
  const T den = I1 + T(1);
  const M3<T> cof = cofactor(f);
  const M3<T> dcof = directionalCofactor(f, h);
  const T shear = mu * (T(1) - T(1) / den);
  const T dshear = T(2) * mu * frob(f, h) / (den * den);
  const T volume = lambda * (det(f) - T(1)) - T(0.75) * mu;
  const T dvolume = lambda * frob(cof, h);
  return shear * h + dshear * f + dvolume * cof + volume * dcof;
}

// ---- globalization (jgs2-globalization-wgsl.ts) ----
template <class T> M3<T> symmetrize(const M3<T>& m) {
  const T a01 = T(0.5) * (at(m, 0, 1) + at(m, 1, 0));
  const T a02 = T(0.5) * (at(m, 0, 2) + at(m, 2, 0));
  const T a12 = T(0.5) * (at(m, 1, 2) + at(m, 2, 1));
  return {{{m.c[0].x, a01, a02}, {a01, m.c[1].y, a12}, {a02, a12, m.c[2].z}}};
}
template <class T> T maxRelativeAsymmetry(const M3<T>& m) {
  T mx = 0;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) mx = std::max(mx, std::fabs(at(m, c, r)));
  if (!(mx > T(0))) return 0;
  const T d = std::max(std::fabs(at(m, 0, 1) - at(m, 1, 0)),
                       std::max(std::fabs(at(m, 0, 2) - at(m, 2, 0)), std::fabs(at(m, 1, 2) - at(m, 2, 1))));
  return d / mx;
}
template <class T> T frobeniusOverSqrt3(const M3<T>& m) {
  const T me = std::max(std::max(std::max(std::fabs(at(m, 0, 0)), std::fabs(at(m, 1, 1))), std::fabs(at(m, 2, 2))),
                        std::max(std::max(std::fabs(at(m, 0, 1)), std::fabs(at(m, 0, 2))), std::fabs(at(m, 1, 2))));
  if (!(me > T(0))) return 0;
  const T a00 = at(m, 0, 0) / me, a11 = at(m, 1, 1) / me, a22 = at(m, 2, 2) / me;
  const T a01 = at(m, 0, 1) / me, a02 = at(m, 0, 2) / me, a12 = at(m, 1, 2) / me;
  const T sq = a00 * a00 + a11 * a11 + a22 * a22 + T(2) * (a01 * a01 + a02 * a02 + a12 * a12);
  return me * std::sqrt(sq / T(3));
}
template <class T> T minSymmetricEigenvalue(const M3<T>& m) {
  const T a00 = at(m, 0, 0), a11 = at(m, 1, 1), a22 = at(m, 2, 2);
  const T a01 = at(m, 0, 1), a02 = at(m, 0, 2), a12 = at(m, 1, 2);
  const T off = a01 * a01 + a02 * a02 + a12 * a12;
  if (off == T(0)) return std::min(a00, std::min(a11, a22));
  const T mean = (a00 + a11 + a22) / T(3);
  const T d00 = a00 - mean, d11 = a11 - mean, d22 = a22 - mean;
  const T cs = d00 * d00 + d11 * d11 + d22 * d22 + T(2) * off;
  const T ss = std::sqrt(cs / T(6));
  if (!(ss > T(0))) return std::min(a00, std::min(a11, a22));
  const M3<T> nc = {{v3(d00, a01, a02) / ss, v3(a01, d11, a12) / ss, v3(a02, a12, d22) / ss}};
  const T hd = std::min(T(1), std::max(T(-1), T(0.5) * det(nc)));
  const T angle = std::acos(hd) / T(3);
  const T largest = mean + T(2) * ss * std::cos(angle);
  const T smallest = mean + T(2) * ss * std::cos(angle + static_cast<T>(kTwoPiOverThree));
  const T middle = T(3) * mean - largest - smallest;
  return std::min(largest, std::min(middle, smallest));
}

template <class T>
struct SolveResult {
  V3<T> direction{0, 0, 0};
  T gdd = 0, scale = 0, minEig = 0, shift = 0, asym = 0, residual = 0;
  uint32_t status = kStatusNonfinite;
};

template <class T> T scaledLength(V3<T> v) {
  const T mc = std::max(std::fabs(v.x), std::max(std::fabs(v.y), std::fabs(v.z)));
  if (!(mc > T(0))) return 0;
  const V3<T> n = v / mc;
  return mc * std::sqrt(dot(n, n));
}

template <class T> SolveResult<T> globalizationSolve(const M3<T>& hessian, V3<T> gradient, T inertia) {
  SolveResult<T> out;
  if (!finiteM(hessian) || !finiteS(inertia) || !(inertia > T(0))) return out;  // invalid input
  const M3<T> sym = symmetrize(hessian);
  const T lad = std::max(std::fabs(at(sym, 0, 0)), std::max(std::fabs(at(sym, 1, 1)), std::fabs(at(sym, 2, 2))));
  const T scale = std::max(inertia, std::max(lad, frobeniusOverSqrt3(sym)));
  if (!finiteS(scale) || !(scale > T(0))) return out;
  const M3<T> nh = {{sym.c[0] / scale, sym.c[1] / scale, sym.c[2] / scale}};
  const T minEig = minSymmetricEigenvalue(nh);
  if (!finiteS(minEig)) return out;
  const T shift = std::max(T(0), static_cast<T>(kRelativeEigenvalueFloor) - minEig);
  out.scale = scale;
  out.minEig = minEig;
  out.shift = shift;
  out.asym = maxRelativeAsymmetry(hessian);
  if (shift > static_cast<T>(kMaxNormalizedShift)) { out.status = kStatusShiftLimit; return out; }
  if (!finiteV(gradient)) { out.status = kStatusNonfinite; return out; }
  const T gs = std::max(std::fabs(gradient.x), std::max(std::fabs(gradient.y), std::fabs(gradient.z)));
  if (!(gs > T(0))) { out.status = kStatusZeroGradient; return out; }
  M3<T> m = nh;
  m.c[0].x += shift; m.c[1].y += shift; m.c[2].z += shift;
  const V3<T> rhs = (-gradient) / scale;
  if (!finiteV(rhs)) { out.status = kStatusNonfinite; return out; }
  const T p0 = m.c[0].x;
  if (!finiteS(p0) || !(p0 > T(0))) { out.status = kStatusCholeskyFailed; return out; }
  const T l00 = std::sqrt(p0);
  const T l10 = m.c[0].y / l00, l20 = m.c[0].z / l00;
  const T p1 = m.c[1].y - l10 * l10;
  if (!finiteS(p1) || !(p1 > T(0))) { out.status = kStatusCholeskyFailed; return out; }
  const T l11 = std::sqrt(p1);
  const T l21 = (m.c[1].z - l20 * l10) / l11;
  const T p2 = m.c[2].z - l20 * l20 - l21 * l21;
  if (!finiteS(p2) || !(p2 > T(0))) { out.status = kStatusCholeskyFailed; return out; }
  const T l22 = std::sqrt(p2);
  const T y0 = rhs.x / l00;
  const T y1 = (rhs.y - l10 * y0) / l11;
  const T y2 = (rhs.z - l20 * y0 - l21 * y1) / l22;
  const T x2 = y2 / l22;
  const T x1 = (y1 - l21 * x2) / l11;
  const T x0 = (y0 - l10 * x1 - l20 * x2) / l00;
  const V3<T> dir = v3(x0, x1, x2);
  if (!finiteV(dir)) { out.status = kStatusCholeskyFailed; return out; }
  const T gdd = dot(gradient, dir);
  if (!finiteS(gdd)) { out.status = kStatusNonDescent; return out; }
  if (!(gdd < T(0))) { out.gdd = gdd; out.status = kStatusNonDescent; return out; }
  const V3<T> res = m * dir - rhs;
  const T rr = scaledLength(res) / std::max(T(1), scaledLength(rhs));
  if (!finiteS(rr)) { out.gdd = gdd; out.status = kStatusCholeskyFailed; return out; }
  out.direction = dir;
  out.gdd = gdd;
  out.residual = rr;
  out.status = kStatusAccepted;
  return out;
}

template <class T> T logOnePlus(T v) {
  if (std::fabs(v) <= T(0.001)) {
    return v * (T(1) + v * (T(-0.5) + v * (static_cast<T>(0.3333333333333333) + v * (T(-0.25) + T(0.2) * v))));
  }
  return std::log(T(1) + v);
}
template <class T> T determinantDelta(const M3<T>& i, const M3<T>& f) {
  const M3<T> d = f - i;
  return dot(d.c[0], cross(i.c[1], i.c[2])) + dot(i.c[0], cross(d.c[1], i.c[2])) +
         dot(i.c[0], cross(i.c[1], d.c[2])) + dot(d.c[0], cross(d.c[1], i.c[2])) +
         dot(d.c[0], cross(i.c[1], d.c[2])) + dot(i.c[0], cross(d.c[1], d.c[2])) +
         dot(d.c[0], cross(d.c[1], d.c[2]));
}
template <class T> T snhEnergyDelta(const M3<T>& i, const M3<T>& f, T lambda, T mu) {
  const M3<T> dd = f - i;
  const T ii = frob(i, i);
  const T id = frob(dd, f + i);
  const T detd = determinantDelta(i, f);
  const T j0 = det(i), j1 = det(f);
  const T lr = logOnePlus(id / (ii + T(1)));
  return T(0.5) * mu * id - T(0.75) * mu * detd + T(0.5) * lambda * detd * (j1 + j0 - T(2)) - T(0.5) * mu * lr;
}

// ---- IPC contact library (ipc-contact-wgsl.ts:19-472) ----
constexpr float kIpcLengthSquaredFloor = 1.0e-20f;
constexpr float kIpcParallelRelativeEpsilon = 1.0e-6f;
constexpr uint32_t kIpcVertexTriangle = 0, kIpcEdgeEdge = 1;

template <class T>
struct Contact {
  V3<T> pa;
  T distance;
  V3<T> pb;
  T squared;
  V3<T> normal;
  bool valid;
  V4<T> weights;
};

template <class T> V3<T> ipcSafeUnit(V3<T> v, V3<T> fallback) {
  const T l2 = dot(v, v);
  if (finiteS(l2) && l2 > T(kIpcLengthSquaredFloor)) return v * (T(1) / std::sqrt(l2));
  const T f2 = dot(fallback, fallback);
  if (finiteS(f2) && f2 > T(kIpcLengthSquaredFloor)) return fallback * (T(1) / std::sqrt(f2));
  return v3<T>(1, 0, 0);
}
template <class T> V3<T> ipcOrthogonalUnit(V3<T> d) {
  const V3<T> a = v3(std::fabs(d.x), std::fabs(d.y), std::fabs(d.z));
  V3<T> axis = v3<T>(1, 0, 0);
  if (a.y <= a.x && a.y <= a.z) axis = v3<T>(0, 1, 0);
  else if (a.z <= a.x && a.z <= a.y) axis = v3<T>(0, 0, 1);
  return ipcSafeUnit(cross(d, axis), v3<T>(1, 0, 0));
}
template <class T> Contact<T> ipcInvalidContact() {
  return {v3<T>(0, 0, 0), T(0), v3<T>(0, 0, 0), T(0), v3<T>(1, 0, 0), false, {0, 0, 0, 0}};
}
template <class T> bool finite4v(V4<T> v) { return finiteS(v.x) && finiteS(v.y) && finiteS(v.z) && finiteS(v.w); }
template <class T> Contact<T> ipcMakeContact(V3<T> pa, V3<T> pb, V4<T> w, V3<T> fallback) {
  if (!finiteV(pa) || !finiteV(pb) || !finite4v(w)) return ipcInvalidContact<T>();
  const V3<T> gap = pa - pb;
  const T sq = dot(gap, gap);
  if (!finiteS(sq) || sq < T(0)) return ipcInvalidContact<T>();
  return {pa, std::sqrt(sq), pb, sq, ipcSafeUnit(gap, fallback), true, w};
}
template <class T> T clamp01(T v) { return std::min(std::max(v, T(0)), T(1)); }
template <class T>
struct SegmentPoint { V3<T> point; T parameter; T squared; };
template <class T> SegmentPoint<T> ipcClosestOnSegment(V3<T> q, V3<T> s, V3<T> e) {
  const V3<T> edge = e - s;
  const T l2 = dot(edge, edge);
  T t = 0;
  if (finiteS(l2) && l2 > T(kIpcLengthSquaredFloor)) t = clamp01(dot(q - s, edge) / l2);
  const V3<T> p = s + t * edge;
  const V3<T> d = q - p;
  return {p, t, dot(d, d)};
}
template <class T> Contact<T> ipcPointTriangle(V3<T> p, V3<T> t0, V3<T> t1, V3<T> t2) {
  const V3<T> e01 = t1 - t0, e02 = t2 - t0, e12 = t2 - t1;
  const T s01 = dot(e01, e01), s02 = dot(e02, e02), s12 = dot(e12, e12);
  const T largest = std::max(s01, std::max(s02, s12));
  const V3<T> an = cross(e01, e02);
  const T a2 = dot(an, an);
  const T threshold = std::max(T(kIpcLengthSquaredFloor) * T(kIpcLengthSquaredFloor),
                               T(kIpcParallelRelativeEpsilon) * largest * largest);
  V3<T> longest = e01;
  if (s02 > s01 && s02 >= s12) longest = e02;
  else if (s12 > s01 && s12 > s02) longest = e12;
  const V3<T> fallback = ipcSafeUnit(an, ipcOrthogonalUnit(longest));
  if (finiteS(a2) && a2 > threshold) {
    const T d00 = s01, d01 = dot(e01, e02), d11 = s02;
    const V3<T> po = p - t0;
    const T d20 = dot(po, e01), d21 = dot(po, e02);
    const T den = d00 * d11 - d01 * d01;
    const T b1 = (d11 * d20 - d01 * d21) / den;
    const T b2 = (d00 * d21 - d01 * d20) / den;
    const T b0 = T(1) - b1 - b2;
    if (b0 >= T(0) && b1 >= T(0) && b2 >= T(0)) {
      const V3<T> closest = b0 * t0 + b1 * t1 + b2 * t2;
      return ipcMakeContact(p, closest, V4<T>{T(1), -b0, -b1, -b2}, fallback);
    }
  }
  const SegmentPoint<T> c01 = ipcClosestOnSegment(p, t0, t1);
  const SegmentPoint<T> c12 = ipcClosestOnSegment(p, t1, t2);
  const SegmentPoint<T> c20 = ipcClosestOnSegment(p, t2, t0);
  SegmentPoint<T> best = c01;
  V3<T> bary = v3<T>(T(1) - c01.parameter, c01.parameter, T(0));
  if (c12.squared < best.squared) { best = c12; bary = v3<T>(T(0), T(1) - c12.parameter, c12.parameter); }
  if (c20.squared < best.squared) { best = c20; bary = v3<T>(c20.parameter, T(0), T(1) - c20.parameter); }
  return ipcMakeContact(p, best.point, V4<T>{T(1), -bary.x, -bary.y, -bary.z}, fallback);
}
template <class T> Contact<T> ipcEdgeEdge(V3<T> a0, V3<T> a1, V3<T> b0, V3<T> b1) {
  const V3<T> da = a1 - a0, db = b1 - b0, off = a0 - b0;
  const T la = dot(da, da), lb = dot(db, db);
  const T scale = std::max(la, lb);
  const T degenerate = std::max(T(kIpcLengthSquaredFloor), T(kIpcParallelRelativeEpsilon) * scale);
  const bool aDeg = !(la > degenerate), bDeg = !(lb > degenerate);
  T pa = 0, pb = 0;
  if (aDeg && !bDeg) {
    pb = clamp01(dot(db, off) / lb);
  } else if (!aDeg) {
    const T projA = dot(da, off);
    if (bDeg) {
      pa = clamp01(-projA / la);
    } else {
      const T coupling = dot(da, db);
      const T projB = dot(db, off);
      const T den = la * lb - coupling * coupling;
      const T parallel = T(kIpcParallelRelativeEpsilon) * la * lb;
      if (den > parallel) pa = clamp01((coupling * projB - projA * lb) / den);
      const T pbu = (coupling * pa + projB) / lb;
      if (pbu < T(0)) {
        pb = 0;
        pa = clamp01(-projA / la);
      } else if (pbu > T(1)) {
        pb = 1;
        pa = clamp01((coupling - projA) / la);
      } else {
        pb = pbu;
      }
    }
  }
  const V3<T> pointA = a0 + pa * da, pointB = b0 + pb * db;
  const V3<T> longest = lb > la ? db : da;
  const V3<T> fallback = ipcSafeUnit(cross(da, db), ipcOrthogonalUnit(longest));
  return ipcMakeContact(pointA, pointB, V4<T>{T(1) - pa, pa, -(T(1) - pb), -pb}, fallback);
}
template <class T> bool ipcBarrierActive(T d, T dHat) {
  return finiteS(d) && finiteS(dHat) && d > T(0) && d < dHat;
}
template <class T> T ipcBarrier(T d, T dHat) {
  if (!ipcBarrierActive(d, dHat)) return 0;
  const T o = d - dHat;
  const T lr = std::log(d) - std::log(dHat);
  return -(o * o) * lr;
}
template <class T> T ipcBarrier1(T d, T dHat) {
  if (!ipcBarrierActive(d, dHat)) return 0;
  const T o = d - dHat;
  const T lr = std::log(d) - std::log(dHat);
  return T(-2) * o * lr - o * o / d;
}
template <class T> T ipcBarrier2(T d, T dHat) {
  if (!ipcBarrierActive(d, dHat)) return 0;
  const T o = d - dHat;
  const T lr = std::log(d) - std::log(dHat);
  return T(-2) * lr - T(4) * o / d + o * o / (d * d);
}
template <class T> T ipcNormalGradientScalar(T w, T kappa, T b1) {
  if (!finiteS(w) || !finiteS(kappa) || !finiteS(b1) || kappa < T(0)) return 0;
  return w * kappa * b1;
}
template <class T> T ipcPsdScalar(T w, T kappa, T b2) {
  if (!finiteS(w) || !finiteS(kappa) || !finiteS(b2) || kappa <= T(0) || w == T(0) || b2 <= T(0)) return 0;
  const T s = kappa * w * w * b2;
  if (!finiteS(s)) return static_cast<T>(kF32Max);
  return s;
}
template <class T> M3<T> ipcPsdNormalHessian(V3<T> n, T s) {
  const V3<T> u = ipcSafeUnit(n, v3<T>(1, 0, 0));
  const T k = std::max(s, T(0));
  return {{k * u.x * u, k * u.y * u, k * u.z * u}};
}
template <class T> T ipcSafeStepCap(T src, T dMin, T L, T safety) {
  if (!finiteS(src) || !finiteS(dMin) || !finiteS(L) || !finiteS(safety) || dMin < T(0) || src <= dMin ||
      L < T(0))
    return 0;
  if (L == T(0)) return 1;
  return clamp01(clamp01(safety) * (src - dMin) / L);
}
template <class T> T ipcFrictionF1(T s, T eps) {
  const T n = std::max(s, T(0));
  if (!(eps > T(0)) || n >= eps) return n > T(0) ? T(1) : T(0);
  const T u = n / eps;
  return u * (T(2) - u);
}
template <class T> T ipcFrictionDissipation(T slip, T eps, T mu, T lambda) {
  if (!finiteS(slip) || !finiteS(eps) || !finiteS(mu) || !finiteS(lambda)) return 0;
  const T n = std::max(slip, T(0));
  const T scale = std::max(mu, T(0)) * std::max(lambda, T(0));
  if (!(eps > T(0))) return scale * n;
  if (n < eps) {
    const T u = n / eps;
    return scale * eps * u * u * (T(1) - u / T(3));
  }
  return scale * (n - eps / T(3));
}
// ipcAabbDistanceLowerBound (jgs2-shader.ts:520-548).
template <class T> T ipcAabbLowerBound(uint32_t type, V3<T> p0, V3<T> p1, V3<T> p2, V3<T> p3) {
  auto vmin = [](V3<T> a, V3<T> b) { return v3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); };
  auto vmax = [](V3<T> a, V3<T> b) { return v3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)); };
  V3<T> gap = v3<T>(0, 0, 0);
  if (type == kIpcVertexTriangle) {
    const V3<T> lo = vmin(p1, vmin(p2, p3)), hi = vmax(p1, vmax(p2, p3));
    gap = vmax(vmax(lo - p0, p0 - hi), v3<T>(0, 0, 0));
  } else {
    const V3<T> lo0 = vmin(p0, p1), hi0 = vmax(p0, p1), lo1 = vmin(p2, p3), hi1 = vmax(p2, p3);
    gap = vmax(vmax(lo1 - hi0, lo0 - hi1), v3<T>(0, 0, 0));
  }
  return std::sqrt(dot(gap, gap));
}
// ipcContactFromPositions (jgs2-shader.ts:564-592): a separated contact at
// the AABB lower bound when that bound reaches the threshold.
template <class T>
Contact<T> ipcContactFromPositions(uint32_t type, V3<T> p0, V3<T> p1, V3<T> p2, V3<T> p3, T threshold) {
  const T lb = ipcAabbLowerBound(type, p0, p1, p2, p3);
  if (finiteS(lb) && lb >= threshold) return {v3<T>(0, 0, 0), lb, v3<T>(0, 0, 0), lb * lb, v3<T>(1, 0, 0), true, {0, 0, 0, 0}};
  if (type == kIpcVertexTriangle) return ipcPointTriangle(p0, p1, p2, p3);
  return ipcEdgeEdge(p0, p1, p2, p3);
}

// ---- the oracle solver ----------------------------------------------------

struct Settings {
  uint32_t schedule, iterations;
  float timestep, gravity[3], floorHeight, floorStiffness, velocityDamping, regularization,
      rotationEpsilon, maxStep, residualTolerance, normalizedUpdateTolerance,
      contactTangentialDamping, contactMargin, ipcActivation, ipcStiffness;
  bool horizontalBodyCorrection;
};

template <class T>
struct Oracle {
  uint32_t V = 0, Tn = 0, K = 0, bodyCount = 1;
  bool glob = true;
  // static
  std::vector<V4<T>> restMass;  // rest xyz, mass
  std::vector<uint32_t> info;   // 4V
  std::vector<uint32_t> tetIdx; // 4T
  std::vector<M3<T>> invDm;     // T
  std::vector<V4<T>> meta;      // T
  std::vector<T> stiffness;     // 144 T (co-rotated only)
  std::vector<uint32_t> adjacency;
  std::vector<uint32_t> cubTet;
  std::vector<T> cubW, cubBasis;
  std::vector<V4<T>> objectives;  // 2V
  uint32_t objectiveFlags = 0;
  std::vector<uint32_t> colors;
  uint32_t colorCount = 1;
  T sceneScale = 1;
  // dynamic
  std::vector<V3<T>> posA, posB, predicted, velocity, old;
  std::vector<M3<T>> vertexRot, tetRot;
  std::vector<V4<T>> finalUpdate, local, tetGlob, vertexEnergy, conv;
  V4<T> control[4];
  std::vector<V4<T>> history;
  // per-dispatch state ("uniforms")
  std::vector<V3<T>>* src = nullptr;
  std::vector<V3<T>>* tgt = nullptr;
  int activeColor = -1;
  bool stopEnabled = false;
  Settings st{};
  T dt = 0, invDt = 0, invDt2 = 0;

  bool pinned(uint32_t v) const { return info[4 * v + 2] != 0; }
  bool forceEnabled() const { return (objectiveFlags & 1u) != 0; }
  bool targetEnabled() const { return (objectiveFlags & 2u) != 0; }

  static uint32_t controlBits(T packed) {
    if (!finiteS(packed) || packed < T(0) || packed > T(kControlMask) || packed != std::floor(packed)) return 0;
    return static_cast<uint32_t>(packed);
  }
  static uint32_t validityBits(T packed) { return controlBits(packed) & kValidityMask; }
  bool latched() const {
    if (!stopEnabled) return false;
    return (controlBits(control[0].w) & kStopLatch) != 0;
  }
  static bool finiteNonnegInt(T v, T maximum) {
    return finiteS(v) && v >= T(0) && v <= maximum && v == std::floor(v);
  }

  V3<T> safeNormalize(V3<T> v, V3<T> fallback) const {
    const T sq = dot(v, v);
    const T eps = static_cast<T>(st.rotationEpsilon);
    if (sq > eps * eps && sq < T(1.0e30)) return v * (T(1) / std::sqrt(sq));
    return fallback;
  }
  V3<T> perpendicularTo(V3<T> axis) const {
    V3<T> c = v3<T>(1, 0, 0);
    if (std::fabs(axis.x) > T(0.8)) c = v3<T>(0, 1, 0);
    return safeNormalize(cross(axis, c), v3<T>(0, 0, 1));
  }
  M3<T> orthonormalize(const M3<T>& m) const {
    const V3<T> c0 = safeNormalize(m.c[0], v3<T>(1, 0, 0));
    const V3<T> c1c = m.c[1] - c0 * dot(c0, m.c[1]);
    V3<T> c1 = safeNormalize(c1c, perpendicularTo(c0));
    V3<T> c2 = safeNormalize(cross(c0, c1), v3<T>(0, 0, 1));
    if (dot(c2, m.c[2]) < T(0)) { c1 = -c1; c2 = -c2; }
    c1 = safeNormalize(cross(c2, c0), perpendicularTo(c0));
    return {{c0, c1, c2}};
  }
  M3<T> polar(const M3<T>& m) const {
    M3<T> r = m;
    for (int it = 0; it < 7; ++it) {
      const T d = det(r);
      const T mag = std::fabs(d);
      if (!(mag > static_cast<T>(st.rotationEpsilon)) || mag > T(1.0e20)) break;
      const T recip = T(1) / d;
      const M3<T> it2 = recip * M3<T>{{cross(r.c[1], r.c[2]), cross(r.c[2], r.c[0]), cross(r.c[0], r.c[1])}};
      r = T(0.5) * (r + it2);
    }
    return orthonormalize(r);
  }

  const uint32_t* tetIndices(uint32_t t) const { return &tetIdx[4 * t]; }
  static uint32_t slotOf(const uint32_t* q, uint32_t v) {
    if (q[0] == v) return 0;
    if (q[1] == v) return 1;
    if (q[2] == v) return 2;
    if (q[3] == v) return 3;
    return 4;
  }
  bool stableTet(uint32_t t) const { return meta[t].w >= T(0.5); }
  M3<T> deformationAt(uint32_t t, const std::vector<V3<T>>& x) const {
    const uint32_t* q = tetIndices(t);
    const V3<T> p0 = x[q[0]];
    const M3<T> ds = {{x[q[1]] - p0, x[q[2]] - p0, x[q[3]] - p0}};
    return ds * invDm[t];
  }
  void shapeGradients(uint32_t t, V3<T> g[4]) const {
    const M3<T> rows = transpose(invDm[t]);
    g[1] = rows.c[0]; g[2] = rows.c[1]; g[3] = rows.c[2];
    g[0] = -g[1] - g[2] - g[3];
  }
  void stableGradientAt(uint32_t t, const std::vector<V3<T>>& x, V3<T> out[4]) const {
    const M3<T> P = snhPiola(deformationAt(t, x), meta[t].y, meta[t].z);
    V3<T> g[4];
    shapeGradients(t, g);
    for (int l = 0; l < 4; ++l) out[l] = meta[t].x * (P * g[l]);
  }
  void stableHessianProduct(uint32_t t, const V3<T> dir[4], V3<T> out[4]) const {
    V3<T> g[4];
    shapeGradients(t, g);
    M3<T> dF = zeroM<T>();
    for (int l = 0; l < 4; ++l) dF = dF + M3<T>{{dir[l] * g[l].x, dir[l] * g[l].y, dir[l] * g[l].z}};
    const M3<T> s = snhTangent(deformationAt(t, *src), dF, meta[t].y, meta[t].z);
    for (int l = 0; l < 4; ++l) out[l] = meta[t].x * (s * g[l]);
  }
  M3<T> stableLocalHessian(uint32_t t, uint32_t slot) const {
    V3<T> g[4];
    shapeGradients(t, g);
    const V3<T> gr = g[slot];
    const M3<T> F = deformationAt(t, *src);
    M3<T> out;
    for (int c = 0; c < 3; ++c) {
      V3<T> axis = v3<T>(0, 0, 0);
      setComp(axis, c, T(1));
      const M3<T> d = {{axis * gr.x, axis * gr.y, axis * gr.z}};
      out.c[c] = meta[t].x * (snhTangent(F, d, meta[t].y, meta[t].z) * gr);
    }
    return out;
  }
  M3<T> stiffnessBlock(uint32_t t, uint32_t rv, uint32_t cv) const {
    const T* k = &stiffness[144ull * t];
    const uint32_t r0 = rv * 3, c0 = cv * 3;
    M3<T> m;
    for (int c = 0; c < 3; ++c)
      m.c[c] = v3(k[(r0) * 12 + c0 + c], k[(r0 + 1) * 12 + c0 + c], k[(r0 + 2) * 12 + c0 + c]);
    return m;
  }
  void tetGradient(uint32_t t, V3<T> out[4]) const {
    if (stableTet(t)) { stableGradientAt(t, *src, out); return; }
    const uint32_t* q = tetIndices(t);
    V3<T> cur[4], rest[4];
    for (int l = 0; l < 4; ++l) {
      cur[l] = (*src)[q[l]];
      rest[l] = v3(restMass[q[l]].x, restMass[q[l]].y, restMass[q[l]].z);
    }
    const V3<T> cc = T(0.25) * (cur[0] + cur[1] + cur[2] + cur[3]);
    const V3<T> rc = T(0.25) * (rest[0] + rest[1] + rest[2] + rest[3]);
    const M3<T> R = tetRot[t];
    const M3<T> Rt = transpose(R);
    V3<T> disp[4];
    for (int l = 0; l < 4; ++l) disp[l] = Rt * (cur[l] - cc) - (rest[l] - rc);
    for (int r = 0; r < 4; ++r) {
      V3<T> lg = v3<T>(0, 0, 0);
      for (int c = 0; c < 4; ++c) lg = lg + stiffnessBlock(t, r, c) * disp[c];
      out[r] = R * lg;
    }
  }
  M3<T> cubBlock(size_t record, int l) const {
    const T* b = &cubBasis[36 * record + 9 * l];
    return {{v3(b[0], b[3], b[6]), v3(b[1], b[4], b[7]), v3(b[2], b[5], b[8])}};
  }
  void currentBasis(size_t record, uint32_t v, const uint32_t* q, M3<T> basis[4]) const {
    const M3<T> Rst = transpose(vertexRot[v]);
    for (int l = 0; l < 4; ++l) basis[l] = vertexRot[q[l]] * cubBlock(record, l) * Rst;
  }
  M3<T> exactTrialF(uint32_t t, uint32_t v, V3<T> d) const {
    const uint32_t slot = slotOf(tetIndices(t), v);
    if (slot >= 4) return deformationAt(t, *src);
    V3<T> g[4];
    shapeGradients(t, g);
    return deformationAt(t, *src) + outerColumns(d, g[slot]);
  }
  M3<T> projectedTrialF(uint32_t t, const M3<T> basis[4], V3<T> d) const {
    V3<T> g[4];
    shapeGradients(t, g);
    M3<T> r = deformationAt(t, *src);
    for (int l = 0; l < 4; ++l) r = r + outerColumns(basis[l] * d, g[l]);
    return r;
  }
  static T quadraticDelta(V3<T> base, V3<T> target, V3<T> d, T w) {
    const V3<T> r = base - target;
    return w * (dot(r, d) + T(0.5) * dot(d, d));
  }
  V3<T> force(uint32_t v) const {
    if (forceEnabled()) return v3(objectives[2 * v].x, objectives[2 * v].y, objectives[2 * v].z);
    return v3<T>(0, 0, 0);
  }
  V4<T> targetRecord(uint32_t v) const {
    if (targetEnabled()) return objectives[2 * v + 1];
    return {0, 0, 0, 0};
  }
  T objectiveDelta(uint32_t v, V3<T> base, V3<T> d) const {
    T r = 0;
    if (forceEnabled()) r -= dot(force(v), d);
    if (targetEnabled()) {
      const V4<T> t = targetRecord(v);
      if (t.w > T(0)) r += quadraticDelta(base, v3(t.x, t.y, t.z), d, t.w);
    }
    return r;
  }
  V3<T> objectiveGradient(uint32_t v, V3<T> p) const {
    V3<T> r = v3<T>(0, 0, 0);
    if (forceEnabled()) r = r - force(v);
    if (targetEnabled()) {
      const V4<T> t = targetRecord(v);
      if (t.w > T(0)) r = r + t.w * (p - v3(t.x, t.y, t.z));
    }
    return r;
  }
  T floorDelta(T baseY, T dY) const {
    const T k = st.floorStiffness, h = st.floorHeight;
    if (!(k > T(0))) return 0;
    const T i = std::min(T(0), baseY - h);
    const T f = std::min(T(0), baseY + dY - h);
    return T(0.5) * k * (f - i) * (f + i);
  }
  T materialDelta(uint32_t t, const M3<T>& i, const M3<T>& f) const {
    return meta[t].x * snhEnergyDelta(i, f, meta[t].y, meta[t].z);
  }
  uint32_t incidentCount(uint32_t v) const { return std::max(info[4 * v + 1], 1u); }
  T distributedInertiaWeight(uint32_t v) const {
    if (pinned(v)) return 0;
    return restMass[v].w * invDt2 / T(incidentCount(v));
  }
  V3<T> distributedInertiaGradient(uint32_t v) const {
    return distributedInertiaWeight(v) * ((*src)[v] - predicted[v]);
  }
  V3<T> distributedObjectiveGradient(uint32_t v) const {
    if (pinned(v)) return v3<T>(0, 0, 0);
    return objectiveGradient(v, (*src)[v]) / T(incidentCount(v));
  }
  T distributedTargetStiffness(uint32_t v) const {
    if (pinned(v)) return 0;
    return targetRecord(v).w / T(incidentCount(v));
  }
  T distributedObjectiveDelta(uint32_t v, V3<T> base, V3<T> d) const {
    if (pinned(v)) return 0;
    return objectiveDelta(v, base, d) / T(incidentCount(v));
  }

  // ---- triangle cloth (jgs2-shader.ts:1225-1844; cloth-layout.ts:88-452) ----
  uint32_t C = 0, H = 0;
  std::vector<uint32_t> clothTri;            // 3C
  std::vector<V4<T>> clothInv;               // C: row-major inverse rest basis (x y / z w)
  std::vector<T> clothArea;                  // C
  std::vector<uint32_t> hingeIdx;            // 4H
  std::vector<T> hingeAngle, hingeLength;    // H
  T clothLambda = 0, clothMu = 0, clothThickness = 0, clothBending = 0;
  // Vertex-to-element CSR in ascending element order (buildIncidentElementCsr,
  // cloth-layout.ts:198-223).
  std::vector<uint32_t> triRows, triElems, hingeRows, hingeElems;

  static V3<T> clothAt(const std::vector<V3<T>>& x, uint32_t q, uint32_t ov, V3<T> op) {
    return q == ov ? op : x[q];
  }
  static uint32_t triSlot(const uint32_t* q, uint32_t v) {
    if (q[0] == v) return 0;
    if (q[1] == v) return 1;
    if (q[2] == v) return 2;
    return 3;
  }
  // clothTriangleShapeGradient (jgs2-shader.ts:1536-1547).
  static void triShapeGradient(const V4<T>& inv, uint32_t l, T* gx, T* gy) {
    if (l == 1) { *gx = inv.x; *gy = inv.y; return; }
    if (l == 2) { *gx = inv.z; *gy = inv.w; return; }
    *gx = -inv.x - inv.z;
    *gy = -inv.y - inv.w;
  }
  struct Membrane {
    T energy;
    V3<T> d0, d1;
    T s0, s1, s2;
    V3<T> g[3];
  };
  // clothMembraneEvaluationAt (jgs2-shader.ts:1549-1608).
  Membrane membraneAt(uint32_t c, const std::vector<V3<T>>& x, uint32_t ov, V3<T> op) const {
    const uint32_t* q = &clothTri[3ull * c];
    const V3<T> x0 = clothAt(x, q[0], ov, op);
    const V3<T> e01 = clothAt(x, q[1], ov, op) - x0;
    const V3<T> e02 = clothAt(x, q[2], ov, op) - x0;
    const V4<T> inv = clothInv[c];
    Membrane m;
    m.d0 = e01 * inv.x + e02 * inv.z;
    m.d1 = e01 * inv.y + e02 * inv.w;
    const T e00 = T(0.5) * (dot(m.d0, m.d0) - T(1));
    const T e01s = T(0.5) * dot(m.d0, m.d1);
    const T e11 = T(0.5) * (dot(m.d1, m.d1) - T(1));
    const T trace = e00 + e11;
    m.s0 = T(2) * clothMu * e00 + clothLambda * trace;
    m.s1 = T(2) * clothMu * e01s;
    m.s2 = T(2) * clothMu * e11 + clothLambda * trace;
    const V3<T> p0 = m.d0 * m.s0 + m.d1 * m.s1;
    const V3<T> p1 = m.d0 * m.s1 + m.d1 * m.s2;
    const T aw = clothArea[c] * clothThickness;
    for (uint32_t l = 0; l < 3; ++l) {
      T gx, gy;
      triShapeGradient(inv, l, &gx, &gy);
      m.g[l] = aw * (p0 * gx + p1 * gy);
    }
    const T density = clothMu * (e00 * e00 + T(2) * e01s * e01s + e11 * e11) + T(0.5) * clothLambda * trace * trace;
    m.energy = aw * density;
    return m;
  }
  // clothMembraneLocalHessian (jgs2-shader.ts:1610-1660) at the source pose.
  M3<T> membraneLocalHessian(uint32_t c, uint32_t slot) const {
    const Membrane ev = membraneAt(c, *src, 0xffffffffu, v3<T>(0, 0, 0));
    T gx, gy;
    triShapeGradient(clothInv[c], slot, &gx, &gy);
    const T aw = clothArea[c] * clothThickness;
    M3<T> r;
    for (int k = 0; k < 3; ++k) {
      V3<T> axis = v3<T>(0, 0, 0);
      setComp(axis, k, T(1));
      const V3<T> f0 = axis * gx, f1 = axis * gy;
      const T de00 = gx * comp(ev.d0, k);
      const T de01 = T(0.5) * (gx * comp(ev.d1, k) + gy * comp(ev.d0, k));
      const T de11 = gy * comp(ev.d1, k);
      const T dtr = de00 + de11;
      const T ds0 = T(2) * clothMu * de00 + clothLambda * dtr;
      const T ds1 = T(2) * clothMu * de01;
      const T ds2 = T(2) * clothMu * de11 + clothLambda * dtr;
      const V3<T> dp0 = f0 * ev.s0 + f1 * ev.s1 + ev.d0 * ds0 + ev.d1 * ds1;
      const V3<T> dp1 = f0 * ev.s1 + f1 * ev.s2 + ev.d0 * ds1 + ev.d1 * ds2;
      r.c[k] = aw * (dp0 * gx + dp1 * gy);
    }
    return T(0.5) * (r + transpose(r));
  }
  // clothTriangleRawNormalAt (jgs2-shader.ts:1662-1690).
  V3<T> triangleNormalAt(uint32_t c, const std::vector<V3<T>>& x, uint32_t ov, V3<T> op) const {
    const uint32_t* q = &clothTri[3ull * c];
    const V3<T> x0 = clothAt(x, q[0], ov, op);
    return cross(clothAt(x, q[1], ov, op) - x0, clothAt(x, q[2], ov, op) - x0);
  }
  struct Dihedral {
    T angle;
    bool valid;
    V3<T> g[4];
  };
  static T length3(V3<T> v) { return std::sqrt(dot(v, v)); }
  static V3<T> normalizedDifferential(V3<T> unit, T len, V3<T> d) { return (d - unit * dot(unit, d)) / len; }
  // clothDihedralEvaluationAt (jgs2-shader.ts:1702-1813): atan2 of
  // (t . (n0 x n1), n0 . n1) and its analytic differential per coordinate.
  Dihedral dihedralAt(uint32_t h, const std::vector<V3<T>>& x, uint32_t ov, V3<T> op) const {
    const uint32_t* q = &hingeIdx[4ull * h];
    V3<T> p[4];
    for (int l = 0; l < 4; ++l) p[l] = clothAt(x, q[l], ov, op);
    Dihedral out{0, false, {}};
    for (auto& g : out.g) g = v3<T>(0, 0, 0);
    const V3<T> edge = p[1] - p[0];
    const T edgeLength = length3(edge);
    const V3<T> to2 = p[2] - p[0];
    const V3<T> rev = -edge;
    const V3<T> to3 = p[3] - p[1];
    const V3<T> n0r = cross(edge, to2), n1r = cross(rev, to3);
    const T nl0 = length3(n0r), nl1 = length3(n1r);
    const T es0 = std::max(edgeLength, std::max(length3(to2), length3(to2 - edge)));
    const T es1 = std::max(edgeLength, std::max(length3(to3), length3(to3 - rev)));
    const bool geometryValid = finiteS(edgeLength) && edgeLength > T(0) && finiteS(nl0) && finiteS(nl1) &&
                               nl0 > T(1.0e-12) * es0 * es0 && nl1 > T(1.0e-12) * es1 * es1;
    if (!geometryValid) return out;
    const V3<T> t = edge / edgeLength;
    const V3<T> n0 = n0r / nl0, n1 = n1r / nl1;
    const V3<T> nc = cross(n0, n1);
    const T sine = dot(t, nc), cosine = dot(n0, n1);
    const T den = sine * sine + cosine * cosine;
    if (!finiteS(den) || !(den > T(0))) return out;
    for (int coord = 0; coord < 12; ++coord) {
      const int dv = coord / 3, axis = coord % 3;
      V3<T> deltas[4];
      for (auto& d : deltas) d = v3<T>(0, 0, 0);
      setComp(deltas[dv], axis, T(1));
      const V3<T> dEdge = deltas[1] - deltas[0];
      const V3<T> dt = normalizedDifferential(t, edgeLength, dEdge);
      const V3<T> dTo2 = deltas[2] - deltas[0];
      const V3<T> dTo3 = deltas[3] - deltas[1];
      const V3<T> dn0r = cross(dEdge, to2) + cross(edge, dTo2);
      const V3<T> dn1r = cross(-dEdge, to3) + cross(rev, dTo3);
      const V3<T> dn0 = normalizedDifferential(n0, nl0, dn0r);
      const V3<T> dn1 = normalizedDifferential(n1, nl1, dn1r);
      const T dcos = dot(dn0, n1) + dot(n0, dn1);
      const T dsin = dot(dt, nc) + dot(t, cross(dn0, n1) + cross(n0, dn1));
      setComp(out.g[dv], axis, (cosine * dsin - sine * dcos) / den);
    }
    const T angle = std::atan2(sine, cosine);
    bool fin = finiteS(angle);
    for (auto& g : out.g) fin = fin && finiteV(g);
    if (!fin) {
      for (auto& g : out.g) g = v3<T>(0, 0, 0);
      return out;
    }
    out.angle = angle;
    out.valid = true;
    return out;
  }
  // clothWrappedAngleDifference (jgs2-shader.ts:1815-1818).
  static T wrappedAngleDifference(T angle, T reference) {
    const T d = angle - reference;
    return std::atan2(std::sin(d), std::cos(d));
  }
  // clothBendingEnergyAt (jgs2-shader.ts:1820-1836).
  T bendingEnergyAt(uint32_t h, const std::vector<V3<T>>& x, uint32_t ov, V3<T> op) const {
    const Dihedral e = dihedralAt(h, x, ov, op);
    if (!e.valid) return static_cast<T>(kF32Max);
    const T diff = wrappedAngleDifference(e.angle, hingeAngle[h]);
    const T ws = clothBending * hingeLength[h];
    return T(0.5) * ws * diff * diff;
  }
  // Membrane and bending gradient (and, with hess, the local Hessian) of
  // vertex v at the source pose: the cloth loops of jgs2Solve
  // (jgs2-shader.ts:3113-3186).
  void clothLocal(uint32_t v, const std::vector<V3<T>>& x, V3<T>* grad, M3<T>* hess) const {
    if (C == 0) return;
    for (uint32_t k = triRows[v]; k < triRows[v + 1]; ++k) {
      const uint32_t c = triElems[k];
      const uint32_t slot = triSlot(&clothTri[3ull * c], v);
      if (slot >= 3) continue;
      *grad = *grad + membraneAt(c, x, 0xffffffffu, v3<T>(0, 0, 0)).g[slot];
      if (hess) *hess = *hess + membraneLocalHessian(c, slot);
    }
    for (uint32_t k = hingeRows[v]; k < hingeRows[v + 1]; ++k) {
      const uint32_t h = hingeElems[k];
      const uint32_t slot = slotOf(&hingeIdx[4ull * h], v);
      if (slot >= 4) continue;
      const Dihedral d = dihedralAt(h, x, 0xffffffffu, v3<T>(0, 0, 0));
      if (!d.valid) {
        const T m = static_cast<T>(kF32Max);
        *grad = *grad + v3<T>(m, m, m);
        continue;
      }
      const T diff = wrappedAngleDifference(d.angle, hingeAngle[h]);
      const T ws = clothBending * hingeLength[h];
      const V3<T> ag = d.g[slot];
      *grad = *grad + ws * diff * ag;
      if (hess) *hess = *hess + ws * outerColumns(ag, ag);
    }
  }

  // ---- IPC contact (jgs2-shader.ts:233-874, 2694-2929) ----
  uint32_t NC = 0, NVT = 0;
  std::vector<uint32_t> cIdx;                  // 4 per candidate
  std::vector<uint32_t> cRows, cIds;           // vertex -> incident candidates (CSR)
  std::vector<uint32_t> activeCount, activeIds;  // per-iteration active rows (capacity of cIds)
  std::vector<V4<T>> srcC, srcW, tgtC, tgtW, lagN, lagW, scratch;
  T contactAlpha = 1;
  bool contactFixed = false;
  T ipcMinDistance = 0, ipcFriction = 0, ipcEpsilon = 0, ipcSafety = 0;  // fixed at create

  uint32_t cType(uint32_t c) const { return c < NVT ? kIpcVertexTriangle : kIpcEdgeEdge; }
  T dHat() const { return static_cast<T>(st.ipcActivation); }
  T kappa() const { return static_cast<T>(st.ipcStiffness); }
  // ipcEnabled (jgs2-shader.ts:458-464).
  bool ipcEnabled() const { return glob && NC > 0 && kappa() > T(0) && dHat() > ipcMinDistance; }
  // ipcContactRoundingReach / ipcBarrierBroadPhaseThreshold / ipcActiveContactReach (:505-518).
  T roundingReach() const {
    return std::max(std::max(sceneScale, dHat()), T(1.0e-12)) * T(kUnitRoundoff) * T(kPositionResolutionMultiplier);
  }
  T broadPhaseThreshold() const { return dHat() + roundingReach(); }
  T activeReach() const { return dHat() + T(2) * (std::max(static_cast<T>(st.maxStep), T(0)) + roundingReach()); }

  Contact<T> contactAt(uint32_t c, const std::vector<V3<T>>& x, T threshold, uint32_t ov = 0xffffffffu,
                       V3<T> op = v3<T>(0, 0, 0)) const {
    const uint32_t* q = &cIdx[4ull * c];
    return ipcContactFromPositions(cType(c), clothAt(x, q[0], ov, op), clothAt(x, q[1], ov, op),
                                   clothAt(x, q[2], ov, op), clothAt(x, q[3], ov, op), threshold);
  }
  static void storeCache(std::vector<V4<T>>& cc, std::vector<V4<T>>& cw, uint32_t c, const Contact<T>& k) {
    const bool valid = k.valid && finiteS(k.distance) && k.distance >= T(0) && finiteV(k.normal) && finite4v(k.weights);
    cc[c] = valid ? V4<T>{k.normal.x, k.normal.y, k.normal.z, k.distance} : V4<T>{0, 0, 0, T(-1)};
    cw[c] = valid ? k.weights : V4<T>{0, 0, 0, 0};
  }
  // ipcCachedContact (:408-437).
  static Contact<T> cached(const V4<T>& nd, const V4<T>& w) {
    const bool valid = nd.w >= T(0) && finite4v(nd) && finite4v(w);
    const T d = valid ? nd.w : T(0);
    return {v3<T>(0, 0, 0), d, v3<T>(0, 0, 0), d * d, valid ? v3(nd.x, nd.y, nd.z) : v3<T>(1, 0, 0), valid,
            valid ? w : V4<T>{0, 0, 0, 0}};
  }
  Contact<T> sourceCache(uint32_t c) const { return cached(srcC[c], srcW[c]); }
  Contact<T> targetCache(uint32_t c) const { return cached(tgtC[c], tgtW[c]); }
  static T weightFor(const uint32_t* q, V4<T> w, uint32_t v) {
    T r = 0;
    if (q[0] == v) r += w.x;
    if (q[1] == v) r += w.y;
    if (q[2] == v) r += w.z;
    if (q[3] == v) r += w.w;
    return r;
  }
  // ipcWeightedDisplacement (:686-708): displacement since the frame start.
  V3<T> weightedDisplacement(uint32_t c, V4<T> w, const std::vector<V3<T>>& x, uint32_t ov, V3<T> op) const {
    const uint32_t* q = &cIdx[4ull * c];
    V3<T> r = v3<T>(0, 0, 0);
    r = r + w.x * (clothAt(x, q[0], ov, op) - old[q[0]]);
    r = r + w.y * (clothAt(x, q[1], ov, op) - old[q[1]]);
    r = r + w.z * (clothAt(x, q[2], ov, op) - old[q[2]]);
    r = r + w.w * (clothAt(x, q[3], ov, op) - old[q[3]]);
    return r;
  }
  // ipcCandidateEnergyFromContact (:710-741).
  T candidateEnergy(uint32_t c, const Contact<T>& k, const std::vector<V3<T>>& x, uint32_t ov, V3<T> op) const {
    if (!k.valid || !(k.distance > ipcMinDistance)) return static_cast<T>(kF32Max);
    T e = kappa() * ipcBarrier(k.distance, dHat());
    const V4<T> lag = lagN[c];
    if (ipcFriction > T(0) && lag.w > T(0)) {
      const V3<T> n = ipcSafeUnit(v3(lag.x, lag.y, lag.z), k.normal);
      const V3<T> rel = weightedDisplacement(c, lagW[c], x, ov, op);
      const V3<T> tang = rel - n * dot(n, rel);
      const T slipVelocity = std::sqrt(dot(tang, tang)) * invDt;
      e += dt * ipcFrictionDissipation(slipVelocity, ipcEpsilon, ipcFriction, lag.w);
    }
    return e;
  }
  uint32_t energyOwner(const uint32_t* q) const {
    for (int l = 0; l < 4; ++l)
      if (!pinned(q[l])) return q[l];
    return q[0];
  }
  // ipcOwnedEnergy (:751-781); useTarget selects the target contact cache
  // (ipcCachedContactAt, :439-449).
  T ownedEnergy(uint32_t v, const std::vector<V3<T>>& x, bool useTarget) const {
    if (!ipcEnabled()) return 0;
    T r = 0;
    for (uint32_t k = 0; k < activeCount[v]; ++k) {
      const uint32_t c = activeIds[cRows[v] + k];
      const Contact<T> contact = useTarget ? targetCache(c) : sourceCache(c);
      if (!contact.valid) return static_cast<T>(kF32Max);
      const bool barrier = ipcBarrierActive(contact.distance, dHat());
      const bool friction = ipcFriction > T(0) && lagN[c].w > T(0);
      if (!barrier && !friction) continue;
      if (energyOwner(&cIdx[4ull * c]) != v) continue;
      const T e = candidateEnergy(c, contact, x, 0xffffffffu, v3<T>(0, 0, 0));
      if (!finiteS(e)) return static_cast<T>(kF32Max);
      r += e;
    }
    return r;
  }
  // ipcLocalContribution (:788-869): barrier gradient and PSD normal block,
  // lagged friction gradient and tangential block.
  void contactLocal(uint32_t v, const std::vector<V3<T>>& x, bool fresh, V3<T>* grad, M3<T>* hess) const {
    if (!ipcEnabled()) return;
    for (uint32_t k = 0; k < activeCount[v]; ++k) {
      const uint32_t c = activeIds[cRows[v] + k];
      const uint32_t* q = &cIdx[4ull * c];
      const Contact<T> contact = fresh ? contactAt(c, x, dHat()) : sourceCache(c);
      if (!contact.valid) continue;
      const bool barrier = ipcBarrierActive(contact.distance, dHat());
      const V4<T> lag = lagN[c];
      const bool friction = ipcFriction > T(0) && lag.w > T(0);
      if (!barrier && !friction) continue;
      if (weightFor(q, V4<T>{1, 1, 1, 1}, v) == T(0)) continue;
      const T w = weightFor(q, contact.weights, v);
      if (w != T(0) && barrier) {
        const T b1 = ipcBarrier1(contact.distance, dHat()), b2 = ipcBarrier2(contact.distance, dHat());
        *grad = *grad + ipcNormalGradientScalar(w, kappa(), b1) * contact.normal;
        if (hess) *hess = *hess + ipcPsdNormalHessian(contact.normal, ipcPsdScalar(w, kappa(), b2));
      }
      const T lw = weightFor(q, lagW[c], v);
      if (friction && lw != T(0)) {
        const V3<T> n = ipcSafeUnit(v3(lag.x, lag.y, lag.z), contact.normal);
        const V3<T> rel = weightedDisplacement(c, lagW[c], x, 0xffffffffu, v3<T>(0, 0, 0));
        const V3<T> tang = rel - n * dot(n, rel);
        const T slip = std::sqrt(dot(tang, tang));
        const T slipVelocity = slip * invDt;
        const T scale = ipcFriction * lag.w;
        V3<T> dir = v3<T>(0, 0, 0);
        if (slip > T(1.0e-12)) dir = tang / slip;
        const T f1 = ipcFrictionF1(slipVelocity, ipcEpsilon);
        *grad = *grad + lw * scale * f1 * dir;
        if (hess) {
          const M3<T> projector = identityM<T>() - ipcPsdNormalHessian(n, T(1));
          T curvature = T(2) * scale / std::max(ipcEpsilon * dt, T(1.0e-12));
          if (slip > T(1.0e-12)) curvature = scale * f1 / slip;
          *hess = *hess + (lw * lw * std::max(curvature, T(0))) * projector;
        }
      }
    }
  }
  bool pinnedMotionExceeds(uint32_t c, T bound) const {
    const uint32_t* q = &cIdx[4ull * c];
    for (int l = 0; l < 4; ++l) {
      if (!pinned(q[l])) continue;
      const V3<T> d = v3(restMass[q[l]].x, restMass[q[l]].y, restMass[q[l]].z) - (*src)[q[l]];
      const T len = std::sqrt(dot(d, d));
      if (!finiteV(d) || !finiteS(len) || len > bound) return true;
    }
    return false;
  }
  // lagContact (:2712-2740), at the accepted pose.
  void lagContact() {
    for (uint32_t c = 0; c < NC; ++c) {
      const Contact<T> k = contactAt(c, posA, broadPhaseThreshold());
      storeCache(srcC, srcW, c, k);
      V4<T> force{0, 0, 0, 0}, w{0, 0, 0, 0};
      if (k.valid && k.distance > ipcMinDistance) {
        const T f = std::max(T(0), -kappa() * ipcBarrier1(k.distance, dHat()));
        if (finiteS(f)) { force = {k.normal.x, k.normal.y, k.normal.z, f}; w = k.weights; }
      }
      lagN[c] = force;
      lagW[c] = w;
      scratch[c] = {1, 0, 0, 0};
    }
    contactAlpha = 1;
  }
  // buildActiveContactRows (:2742-2782).
  void buildActiveRows() {
    const bool bounded = st.maxStep > 0;
    const T reach = activeReach();
    for (uint32_t v = 0; v < V; ++v) {
      uint32_t n = 0;
      for (uint32_t k = cRows[v]; k < cRows[v + 1]; ++k) {
        const uint32_t c = cIds[k];
        const Contact<T> contact = sourceCache(c);
        const bool friction = ipcFriction > T(0) && lagN[c].w > T(0);
        const bool pinnedMotion = pinnedMotionExceeds(c, std::max(static_cast<T>(st.maxStep), T(0)));
        if (!contact.valid || !bounded || contact.distance <= reach || friction || pinnedMotion)
          activeIds[cRows[v] + n++] = c;
      }
      activeCount[v] = n;
    }
  }
  // candidateContactStep (:2784-2847) + reduceContactStep (:2870-2907).
  void contactStepAndReduce() {
    if (latched()) {
      for (uint32_t c = 0; c < NC; ++c) scratch[c] = {1, 0, 0, 1};
    } else {
      for (uint32_t c = 0; c < NC; ++c) {
        const uint32_t* q = &cIdx[4ull * c];
        V3<T> d[4];
        for (int l = 0; l < 4; ++l) d[l] = (*tgt)[q[l]] - (*src)[q[l]];
        T L = 0;
        if (cType(c) == kIpcVertexTriangle)
          L = length3(d[0]) + std::max(length3(d[1]), std::max(length3(d[2]), length3(d[3])));
        else
          L = std::max(length3(d[0]), length3(d[1])) + std::max(length3(d[2]), length3(d[3]));
        Contact<T> source = sourceCache(c);
        bool fullStepSafe = source.valid && finiteS(L) && source.distance - L > ipcMinDistance;
        if (!fullStepSafe) {
          source = contactAt(c, *src, static_cast<T>(kF32Max));
          fullStepSafe = source.valid && finiteS(L) && source.distance - L > ipcMinDistance;
        }
        const bool trialValid = finiteV(d[0]) && finiteV(d[1]) && finiteV(d[2]) && finiteV(d[3]);
        const bool valid = source.valid && trialValid && source.distance > ipcMinDistance && finiteS(L);
        T alpha = 0;
        if (valid) alpha = fullStepSafe ? T(1) : ipcSafeStepCap(source.distance, ipcMinDistance, L, ipcSafety);
        scratch[c] = {alpha, source.valid ? source.distance : T(0), trialValid ? source.distance : T(0),
                      valid ? T(1) : T(0)};
      }
    }
    reduceContactStep();
  }
  void reduceContactStep() {
    T minimum = 1;
    bool all = true;
    for (uint32_t c = 0; c < NC; ++c) {
      const V4<T> s = scratch[c];
      const bool valid = s.w == T(1) && finiteS(s.x) && finiteS(s.y) && finiteS(s.z);
      minimum = std::min(minimum, valid ? s.x : T(0));
      all = all && valid;
    }
    contactAlpha = all ? clamp01(minimum) : T(0);
  }
  // applyContactStep (:2909-2917).
  void applyContactStep() {
    if (latched()) return;
    const T a = clamp01(contactAlpha);
    for (uint32_t v = 0; v < V; ++v) (*tgt)[v] = (*src)[v] + a * ((*tgt)[v] - (*src)[v]);
  }
  // validateContactStep (:2849-2868).
  void validateContactStep() {
    for (uint32_t c = 0; c < NC; ++c) {
      const Contact<T> k = contactAt(c, *tgt, broadPhaseThreshold());
      storeCache(tgtC, tgtW, c, k);
      const bool valid = k.valid && finiteS(k.distance) && k.distance > ipcMinDistance;
      const T d = valid ? k.distance : T(0);
      scratch[c] = {1, d, d, valid ? T(1) : T(0)};
    }
    reduceContactStep();
  }
  // promoteAcceptedContactCache (:2694-2710).
  void promoteContacts() {
    if (!(control[1].x == T(1) && finiteS(contactAlpha) && contactAlpha > T(0))) return;
    srcC = tgtC;
    srcW = tgtW;
  }

  struct Geometry { T minimum; bool valid; };
  Geometry restrictedMinimumDeterminant(uint32_t v, V3<T> d) const {
    T minimum = static_cast<T>(kF32Max);
    const V4<T> pre = control[0];
    const uint32_t bits = validityBits(pre.w);
    if ((bits & kAcceptedMinimumValid) != 0 && finiteS(pre.z)) minimum = pre.z;
    // IPC: a trial that brings an active candidate within the minimum
    // distance is infeasible (jgs2-shader.ts:1997-2038).
    if (ipcEnabled()) {
      const V3<T> trial = (*src)[v] + d;
      const T dl = length3(d);
      for (uint32_t k = 0; k < activeCount[v]; ++k) {
        const uint32_t c = activeIds[cRows[v] + k];
        const Contact<T> source = activeColor >= 0 ? contactAt(c, *src, dHat()) : sourceCache(c);
        if (!source.valid) return {0, false};
        if (source.distance - dl > ipcMinDistance) continue;
        if (weightFor(&cIdx[4ull * c], V4<T>{1, 1, 1, 1}, v) == T(0)) continue;
        const Contact<T> trialContact = contactAt(c, *src, dHat(), v, trial);
        if (!trialContact.valid) return {0, false};
        if (!(trialContact.distance > ipcMinDistance)) return {0, true};
      }
    }
    const uint32_t start = info[4 * v], count = info[4 * v + 1];
    for (uint32_t a = 0; a < count; ++a) {
      const uint32_t t = adjacency[start + a];
      const T j = det(exactTrialF(t, v, d));
      if (!finiteS(j)) return {0, false};
      minimum = std::min(minimum, j);
    }
    for (uint32_t s = 0; s < K; ++s) {
      const size_t rec = static_cast<size_t>(v) * K + s;
      const uint32_t t = cubTet[rec];
      const T w = cubW[rec];
      if (t == kEmptyTet || t >= Tn || !(w > T(0))) continue;
      M3<T> basis[4];
      currentBasis(rec, v, tetIndices(t), basis);
      const T j = det(projectedTrialF(t, basis, d));
      if (!finiteS(j)) return {0, false};
      minimum = std::min(minimum, j);
    }
    // Cloth: signed relative area stretch of each incident triangle at the
    // source and the trial pose (jgs2-shader.ts:2067-2116).
    if (C != 0) {
      const V3<T> trial = (*src)[v] + d;
      for (uint32_t k = triRows[v]; k < triRows[v + 1]; ++k) {
        const uint32_t c = triElems[k];
        if (triSlot(&clothTri[3ull * c], v) >= 3) continue;
        const V3<T> sn = triangleNormalAt(c, *src, 0xffffffffu, v3<T>(0, 0, 0));
        const V3<T> tn = triangleNormalAt(c, *src, v, trial);
        const T twice = T(2) * clothArea[c];
        const T ss = length3(sn) / twice;
        const T tm = length3(tn) / twice;
        const T ts = dot(sn, tn) > T(0) ? tm : -tm;
        if (!(twice > T(0)) || !finiteS(ss) || !finiteS(ts)) return {0, false};
        minimum = std::min(minimum, std::min(ss, ts));
      }
    }
    return {minimum, true};
  }
  T restrictedEnergyDelta(uint32_t v, V3<T> d) const {
    const V3<T> sp = (*src)[v];
    const T inertia = restMass[v].w * invDt2;
    T result = quadraticDelta(sp, predicted[v], d, inertia) + floorDelta(sp.y, d.y);
    if (objectiveFlags != 0) result += objectiveDelta(v, sp, d);
    // IPC barrier and lagged friction deltas (jgs2-shader.ts:2137-2196).
    if (ipcEnabled()) {
      const V3<T> trial = sp + d;
      const T dl = length3(d);
      for (uint32_t k = 0; k < activeCount[v]; ++k) {
        const uint32_t c = activeIds[cRows[v] + k];
        const Contact<T> source = activeColor >= 0 ? contactAt(c, *src, dHat()) : sourceCache(c);
        if (!source.valid) return static_cast<T>(kF32Max);
        const bool friction = ipcFriction > T(0) && lagN[c].w > T(0);
        const bool barrierMayChange = source.distance - dl < dHat();
        if (!barrierMayChange && !friction) continue;
        if (weightFor(&cIdx[4ull * c], V4<T>{1, 1, 1, 1}, v) == T(0)) continue;
        Contact<T> trialContact = {v3<T>(0, 0, 0), dHat(), v3<T>(0, 0, 0), dHat() * dHat(), v3<T>(1, 0, 0), true,
                                   {0, 0, 0, 0}};
        if (barrierMayChange) trialContact = contactAt(c, *src, dHat(), v, trial);
        const T se = candidateEnergy(c, source, *src, 0xffffffffu, v3<T>(0, 0, 0));
        const T te = candidateEnergy(c, trialContact, *src, v, trial);
        result += te - se;
      }
    }
    const uint32_t start = info[4 * v], count = info[4 * v + 1];
    for (uint32_t a = 0; a < count; ++a) {
      const uint32_t t = adjacency[start + a];
      result += materialDelta(t, deformationAt(t, *src), exactTrialF(t, v, d));
    }
    // Cloth membrane and bending deltas of the incident elements
    // (jgs2-shader.ts:2207-2263).
    if (C != 0) {
      const V3<T> trial = sp + d;
      for (uint32_t k = triRows[v]; k < triRows[v + 1]; ++k) {
        const uint32_t c = triElems[k];
        if (triSlot(&clothTri[3ull * c], v) >= 3) continue;
        result += membraneAt(c, *src, v, trial).energy - membraneAt(c, *src, 0xffffffffu, v3<T>(0, 0, 0)).energy;
      }
      for (uint32_t k = hingeRows[v]; k < hingeRows[v + 1]; ++k) {
        const uint32_t h = hingeElems[k];
        if (slotOf(&hingeIdx[4ull * h], v) >= 4) continue;
        result += bendingEnergyAt(h, *src, v, trial) - bendingEnergyAt(h, *src, 0xffffffffu, v3<T>(0, 0, 0));
      }
    }
    for (uint32_t s = 0; s < K; ++s) {
      const size_t rec = static_cast<size_t>(v) * K + s;
      const uint32_t t = cubTet[rec];
      const T w = cubW[rec];
      if (t == kEmptyTet || t >= Tn || !(w > T(0))) continue;
      const uint32_t* q = tetIndices(t);
      M3<T> basis[4];
      currentBasis(rec, v, q, basis);
      const M3<T> initial = deformationAt(t, *src);
      const M3<T> projected = projectedTrialF(t, basis, d);
      T comp = materialDelta(t, initial, projected);
      for (int l = 0; l < 4; ++l)
        comp += quadraticDelta((*src)[q[l]], predicted[q[l]], basis[l] * d, distributedInertiaWeight(q[l]));
      if (objectiveFlags != 0)
        for (int l = 0; l < 4; ++l) comp += distributedObjectiveDelta(q[l], (*src)[q[l]], basis[l] * d);
      const uint32_t ss = slotOf(q, v);
      if (ss < 4) {
        comp -= materialDelta(t, initial, exactTrialF(t, v, d));
        comp -= quadraticDelta(sp, predicted[v], d, distributedInertiaWeight(v));
        if (objectiveFlags != 0) comp -= distributedObjectiveDelta(v, sp, d);
      }
      result += w * comp;
    }
    return result;
  }
  M3<T> cubatureHessian(uint32_t t, const M3<T> basis[4]) const {
    M3<T> out;
    if (stableTet(t)) {
      for (int c = 0; c < 3; ++c) {
        V3<T> dir[4], prod[4];
        for (int l = 0; l < 4; ++l) dir[l] = basis[l].c[c];
        stableHessianProduct(t, dir, prod);
        V3<T> col = v3<T>(0, 0, 0);
        for (int r = 0; r < 3; ++r) {
          T e = 0;
          for (int l = 0; l < 4; ++l) e += dot(basis[l].c[r], prod[l]);
          setComp(col, r, e);
        }
        out.c[c] = col;
      }
      return out;
    }
    const M3<T> R = tetRot[t], Rt = transpose(R);
    for (int c = 0; c < 3; ++c) {
      V3<T> ld[4], wp[4];
      for (int l = 0; l < 4; ++l) ld[l] = Rt * basis[l].c[c];
      for (int r = 0; r < 4; ++r) {
        V3<T> lp = v3<T>(0, 0, 0);
        for (int cv = 0; cv < 4; ++cv) lp = lp + stiffnessBlock(t, r, cv) * ld[cv];
        wp[r] = R * lp;
      }
      V3<T> col = v3<T>(0, 0, 0);
      for (int r = 0; r < 3; ++r) {
        T e = 0;
        for (int l = 0; l < 4; ++l) e += dot(basis[l].c[r], wp[l]);
        setComp(col, r, e);
      }
      out.c[c] = col;
    }
    return out;
  }

  void storeLocal(uint32_t v, V3<T> dir, T alpha, T minEig, T scale, T dshift, T nshift, T dE, T bound,
                  T gdd, T res, T minDet, uint32_t back, uint32_t evals, uint32_t status) {
    local[4 * v] = {dir.x, dir.y, dir.z, alpha};
    local[4 * v + 1] = {minEig, scale, dshift, nshift};
    local[4 * v + 2] = {dE, bound, gdd, res};
    local[4 * v + 3] = {minDet, T(back), T(evals), T(status)};
  }
  T implicitEnergyAt(const std::vector<V3<T>>& x, uint32_t v, bool useTargetCache = false) const {
    const bool pin = pinned(v);
    const V3<T> p = x[v];
    T e = 0;
    if (!pin) {
      const T inertia = restMass[v].w * invDt2;
      const V3<T> r = p - predicted[v];
      e += T(0.5) * inertia * dot(r, r);
    }
    if (objectiveFlags != 0 && !pin) {
      if (forceEnabled()) e -= dot(force(v), p);
      if (targetEnabled()) {
        const V4<T> t = targetRecord(v);
        if (t.w > T(0)) {
          const V3<T> r = p - v3(t.x, t.y, t.z);
          e += T(0.5) * t.w * dot(r, r);
        }
      }
    }
    if (!pin && st.floorStiffness > 0) {
      const T pen = std::min(T(0), p.y - static_cast<T>(st.floorHeight));
      e += T(0.5) * static_cast<T>(st.floorStiffness) * pen * pen;
    }
    // Each cloth element's energy is owned by its lowest vertex index, pinned
    // or not (jgs2-shader.ts:2585-2642).
    if (C != 0) {
      for (uint32_t k = triRows[v]; k < triRows[v + 1]; ++k) {
        const uint32_t c = triElems[k];
        const uint32_t* q = &clothTri[3ull * c];
        if (v != std::min(q[0], std::min(q[1], q[2]))) continue;
        const T twice = T(2) * clothArea[c];
        const T stretch = length3(triangleNormalAt(c, x, 0xffffffffu, v3<T>(0, 0, 0))) / twice;
        if (!(twice > T(0)) || !finiteS(stretch) || !(stretch > T(kDeterminantFloor))) return static_cast<T>(kF32Max);
        e += membraneAt(c, x, 0xffffffffu, v3<T>(0, 0, 0)).energy;
      }
      for (uint32_t k = hingeRows[v]; k < hingeRows[v + 1]; ++k) {
        const uint32_t h = hingeElems[k];
        const uint32_t* q = &hingeIdx[4ull * h];
        if (v != std::min(std::min(q[0], q[1]), std::min(q[2], q[3]))) continue;
        e += bendingEnergyAt(h, x, 0xffffffffu, v3<T>(0, 0, 0));
      }
    }
    e += ownedEnergy(v, x, useTargetCache);
    return e;
  }
  void storeAssembledVertexEnergy(uint32_t v) {
    // The candidate pose reads the target contact cache unless the contact
    // step collapsed to zero (ipcCachedContactAt, jgs2-shader.ts:439-449).
    const bool target = src != tgt && contactAlpha != T(0);
    const T se = implicitEnergyAt(*src, v, false), ce = implicitEnergyAt(*tgt, v, target);
    const bool sv = finiteS(se), cv = finiteS(ce);
    vertexEnergy[v] = {sv ? se : T(0), cv ? ce : T(0), sv ? T(1) : T(0), cv ? T(1) : T(0)};
  }

  // ---- kernels ----
  void predict() {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) {
      const uint32_t v = static_cast<uint32_t>(i);
      const V3<T> o = posA[v];
      old[v] = o;
      V3<T> p = v3(restMass[v].x, restMass[v].y, restMass[v].z);
      if (!pinned(v)) {
        const V3<T> dv = static_cast<T>(st.velocityDamping) * velocity[v];
        p = o + dt * dv + dt * dt * v3<T>(st.gravity[0], st.gravity[1], st.gravity[2]);
      } else {
        velocity[v] = v3<T>(0, 0, 0);
      }
      predicted[v] = p;
      posB[v] = glob ? o : p;
      finalUpdate[v] = {0, 0, 0, 0};
    }
    if (glob)
      for (auto& c : control) c = {0, 0, 0, 0};
  }
  void tetPolarRotation() {
    if (latched()) return;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < Tn; ++i) {
      const uint32_t t = static_cast<uint32_t>(i);
      if (stableTet(t)) { tetRot[t] = identityM<T>(); continue; }
      tetRot[t] = polar(deformationAt(t, *src));
    }
  }
  void vertexPolarRotation() {
    if (latched()) return;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) {
      const uint32_t v = static_cast<uint32_t>(i);
      const uint32_t start = info[4 * v], count = info[4 * v + 1];
      if (count == 0) { vertexRot[v] = identityM<T>(); continue; }
      M3<T> avg = zeroM<T>();
      T total = 0;
      for (uint32_t a = 0; a < count; ++a) {
        const uint32_t t = adjacency[start + a];
        avg = avg + meta[t].x * deformationAt(t, *src);
        total += meta[t].x;
      }
      avg = total > T(0) ? (T(1) / total) * avg : identityM<T>();
      vertexRot[v] = polar(avg);
    }
  }
  void solveVertex(uint32_t v) {
    if (latched()) { (*tgt)[v] = (*src)[v]; return; }
    if (activeColor >= 0 && colors[v] != static_cast<uint32_t>(activeColor)) return;
    if (pinned(v)) {
      (*tgt)[v] = v3(restMass[v].x, restMass[v].y, restMass[v].z);
      finalUpdate[v] = {0, 0, 0, 1};
      if (glob) {
        storeLocal(v, v3<T>(0, 0, 0), 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, kStatusPinned);
        storeAssembledVertexEnergy(v);
      }
      return;
    }
    const V3<T> position = (*src)[v];
    if (glob) {
      const V4<T> pre = control[0];
      const uint32_t bits = validityBits(pre.w);
      const bool amv = (bits & kAcceptedMinimumValid) != 0 && finiteS(pre.z);
      if (!(amv && pre.z > T(kDeterminantFloor))) {
        (*tgt)[v] = (*src)[v];
        finalUpdate[v] = {0, 0, 0, 1};
        storeLocal(v, v3<T>(0, 0, 0), 0, 0, 0, 0, 0, 0, 0, 0, 0, amv ? pre.z : T(0), 0, 0,
                   amv ? kStatusLineSearchFailed : kStatusNonfinite);
        storeAssembledVertexEnergy(v);
        return;
      }
    }
    const T inertia = restMass[v].w * invDt2;
    V3<T> gradient = inertia * (position - predicted[v]);
    M3<T> hessian = inertia * identityM<T>();
    if (objectiveFlags != 0) gradient = gradient + objectiveGradient(v, position);
    if (targetEnabled()) hessian = hessian + targetRecord(v).w * identityM<T>();
    const uint32_t start = info[4 * v], count = info[4 * v + 1];
    for (uint32_t a = 0; a < count; ++a) {
      const uint32_t t = adjacency[start + a];
      const uint32_t slot = slotOf(tetIndices(t), v);
      if (slot >= 4) continue;
      V3<T> tg[4];
      tetGradient(t, tg);
      gradient = gradient + tg[slot];
      if (stableTet(t)) hessian = hessian + stableLocalHessian(t, slot);
      else hessian = hessian + tetRot[t] * stiffnessBlock(t, slot, slot) * transpose(tetRot[t]);
    }
    clothLocal(v, *src, &gradient, &hessian);
    if (st.floorStiffness > 0 && position.y < static_cast<T>(st.floorHeight)) {
      gradient.y += static_cast<T>(st.floorStiffness) * (position.y - static_cast<T>(st.floorHeight));
      hessian.c[1].y += static_cast<T>(st.floorStiffness);
    }
    contactLocal(v, *src, activeColor >= 0, &gradient, &hessian);
    for (uint32_t s = 0; s < K; ++s) {
      const size_t rec = static_cast<size_t>(v) * K + s;
      const uint32_t t = cubTet[rec];
      const T w = cubW[rec];
      if (t == kEmptyTet || t >= Tn || !(w > T(0))) continue;
      const uint32_t* q = tetIndices(t);
      M3<T> basis[4];
      currentBasis(rec, v, q, basis);
      V3<T> tg[4];
      tetGradient(t, tg);
      V3<T> pg = v3<T>(0, 0, 0);
      for (int l = 0; l < 4; ++l) pg = pg + transpose(basis[l]) * (tg[l] + distributedInertiaGradient(q[l]));
      if (objectiveFlags != 0)
        for (int l = 0; l < 4; ++l) pg = pg + transpose(basis[l]) * distributedObjectiveGradient(q[l]);
      M3<T> ph = cubatureHessian(t, basis);
      M3<T> ih = zeroM<T>();
      for (int l = 0; l < 4; ++l) ih = ih + distributedInertiaWeight(q[l]) * (transpose(basis[l]) * basis[l]);
      ph = ph + ih;
      if (targetEnabled()) {
        M3<T> oh = zeroM<T>();
        for (int l = 0; l < 4; ++l) oh = oh + distributedTargetStiffness(q[l]) * (transpose(basis[l]) * basis[l]);
        ph = ph + oh;
      }
      const uint32_t ss = slotOf(q, v);
      if (ss < 4) {
        pg = pg - (tg[ss] + distributedInertiaGradient(v));
        if (objectiveFlags != 0) pg = pg - distributedObjectiveGradient(v);
        if (stableTet(t))
          ph = ph - (stableLocalHessian(t, ss) + distributedInertiaWeight(v) * identityM<T>());
        else
          ph = ph - (tetRot[t] * stiffnessBlock(t, ss, ss) * transpose(tetRot[t]) +
                     distributedInertiaWeight(v) * identityM<T>());
        if (targetEnabled()) ph = ph - distributedTargetStiffness(v) * identityM<T>();
      }
      gradient = gradient + w * pg;
      hessian = hessian + w * ph;
    }
    if (glob) {
      const SolveResult<T> dr = globalizationSolve(hessian, gradient, inertia);
      uint32_t status = kStatusNonfinite;
      const V3<T> full = position + dr.direction;
      const V3<T> fullD = full - position;
      const T scs = std::max(std::fabs(position.x), std::max(std::fabs(position.y), std::fabs(position.z)));
      const T resolution = std::max(sceneScale, std::max(scs, T(1.0e-12))) * static_cast<T>(kUnitRoundoff) *
                           static_cast<T>(kPositionResolutionMultiplier);
      const bool below = dr.status == kStatusAccepted && finiteV(full) && finiteV(fullD) &&
                         scaledLength(fullD) <= resolution;
      if (dr.status == kStatusAccepted) status = below ? kStatusZeroGradient : kStatusLineSearchFailed;
      else if (dr.status == kStatusZeroGradient) status = kStatusZeroGradient;
      else if (dr.status == kStatusShiftLimit) status = kStatusShiftLimit;
      else if (dr.status == kStatusCholeskyFailed) status = kStatusCholeskyFailed;
      else if (dr.status == kStatusNonDescent) status = kStatusNonDescent;
      T alpha = 0, acceptedDelta = 0, bound = 0, minTrialDet = 0;
      uint32_t backtracks = 0, evals = 0;
      V3<T> acceptedD = v3<T>(0, 0, 0), acceptedP = position;
      if (dr.status == kStatusAccepted && !below) {
        T ta = 1;
        const T dl = scaledLength(dr.direction);
        const T maxStep = st.maxStep;
        if (maxStep > T(0) && dl > maxStep) ta = maxStep / dl;
        for (uint32_t b = 0; b <= kMaxBacktracks; ++b) {
          const V3<T> nominal = ta * dr.direction;
          const V3<T> tp = position + nominal;
          const V3<T> td = tp - position;
          if (!finiteV(tp) || !finiteV(td)) { status = kStatusNonfinite; minTrialDet = 0; backtracks = b; break; }
          const T tl = scaledLength(td);
          if (maxStep > T(0) && tl > maxStep) { ta *= T(kBacktrackFactor); continue; }
          if (tl <= resolution) { status = kStatusZeroGradient; minTrialDet = 0; backtracks = b; break; }
          const T gd = dot(gradient, td);
          if (!finiteS(gd)) { status = kStatusNonfinite; minTrialDet = 0; backtracks = b; break; }
          if (!(gd < T(0))) { status = kStatusZeroGradient; minTrialDet = 0; backtracks = b; break; }
          const Geometry geo = restrictedMinimumDeterminant(v, td);
          if (!geo.valid) { status = kStatusNonfinite; minTrialDet = 0; backtracks = b; break; }
          minTrialDet = geo.minimum;
          if (geo.minimum > T(kDeterminantFloor)) {
            const T de = restrictedEnergyDelta(v, td);
            evals += 1;
            if (!finiteS(de)) { status = kStatusNonfinite; backtracks = b; break; }
            const T tb = T(kArmijoC1) * gd;
            if (de <= tb) {
              alpha = ta; acceptedDelta = de; bound = tb; backtracks = b; status = kStatusAccepted;
              acceptedD = td; acceptedP = tp;
              break;
            }
          }
          ta *= T(kBacktrackFactor);
        }
        if (status == kStatusLineSearchFailed) backtracks = kMaxBacktracks;
      }
      (*tgt)[v] = acceptedP;
      finalUpdate[v] = {scaledLength(acceptedD), 0, 0, 1};
      storeLocal(v, dr.direction, alpha, dr.minEig * dr.scale, dr.scale, dr.shift * dr.scale, dr.shift,
                 acceptedDelta, bound, dr.gdd, dr.residual, minTrialDet, backtracks, evals, status);
      storeAssembledVertexEnergy(v);
      return;
    }
    // Legacy co-rotated path: regularizedSolve (jgs2-shader.ts:2479-2512).
    const T ds = std::max(T(1), std::max(std::fabs(at(hessian, 0, 0)),
                                         std::max(std::fabs(at(hessian, 1, 1)), std::fabs(at(hessian, 2, 2)))));
    const T shift = std::max(static_cast<T>(st.regularization) * ds, T(1.0e-9));
    const T a00 = at(hessian, 0, 0) + shift, a11 = at(hessian, 1, 1) + shift, a22 = at(hessian, 2, 2) + shift;
    const T a01 = T(0.5) * (at(hessian, 0, 1) + at(hessian, 1, 0));
    const T a02 = T(0.5) * (at(hessian, 0, 2) + at(hessian, 2, 0));
    const T a12 = T(0.5) * (at(hessian, 1, 2) + at(hessian, 2, 1));
    const V3<T> rhs = -gradient;
    const T l00 = std::sqrt(std::max(a00, shift));
    const T l10 = a01 / l00, l20 = a02 / l00;
    const T l11 = std::sqrt(std::max(a11 - l10 * l10, shift));
    const T l21 = (a12 - l20 * l10) / l11;
    const T l22 = std::sqrt(std::max(a22 - l20 * l20 - l21 * l21, shift));
    const T y0 = rhs.x / l00, y1 = (rhs.y - l10 * y0) / l11, y2 = (rhs.z - l20 * y0 - l21 * y1) / l22;
    const T x2 = y2 / l22, x1 = (y1 - l21 * x2) / l11, x0 = (y0 - l10 * x1 - l20 * x2) / l00;
    V3<T> delta = v3(x0, x1, x2);
    const T sq = dot(delta, delta);
    if (!(sq >= T(0) && sq < T(1.0e30))) delta = v3<T>(0, 0, 0);
    const T dls = dot(delta, delta);
    const T maxStep = st.maxStep;
    if (maxStep > T(0) && dls > maxStep * maxStep) delta = delta * (maxStep * (T(1) / std::sqrt(dls)));
    (*tgt)[v] = position + delta;
    finalUpdate[v] = {std::sqrt(dot(delta, delta)), 0, 0, 1};
  }
  void solveAll() {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < V; ++i) solveVertex(static_cast<uint32_t>(i));
  }
  void assembledVertexEnergyAll() {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) storeAssembledVertexEnergy(static_cast<uint32_t>(i));
  }
  void candidateTetrahedron() {
    if (latched()) return;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < Tn; ++i) {
      const uint32_t t = static_cast<uint32_t>(i);
      const M3<T> sf = deformationAt(t, *src), cf = deformationAt(t, *tgt);
      const T sj = det(sf), cj = det(cf);
      const bool sgv = finiteS(sj), cgv = finiteS(cj);
      T se = 0, ce = 0;
      bool sev = false, cev = false;
      if (sgv && sj > T(kDeterminantFloor)) { se = meta[t].x * snhEnergy(sf, meta[t].y, meta[t].z); sev = finiteS(se); }
      if (cgv && cj > T(kDeterminantFloor)) { ce = meta[t].x * snhEnergy(cf, meta[t].y, meta[t].z); cev = finiteS(ce); }
      tetGlob[2 * t] = {sgv ? sj : T(0), cgv ? cj : T(0), sgv ? T(1) : T(0), cgv ? T(1) : T(0)};
      tetGlob[2 * t + 1] = {sev ? se : T(0), cev ? ce : T(0), sev ? T(1) : T(0), cev ? T(1) : T(0)};
    }
    // Cloth triangles follow the tets: signed area stretch as geometry, and
    // neutral energy lanes (jgs2-shader.ts:3507-3549).
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
      const uint32_t c = static_cast<uint32_t>(i);
      const V3<T> sn = triangleNormalAt(c, *src, 0xffffffffu, v3<T>(0, 0, 0));
      const V3<T> cn = triangleNormalAt(c, *tgt, 0xffffffffu, v3<T>(0, 0, 0));
      const T twice = T(2) * clothArea[c];
      const T ss = length3(sn) / twice;
      const T cm = length3(cn) / twice;
      const T cs = dot(sn, cn) > T(0) ? cm : -cm;
      const bool sgv = twice > T(0) && finiteV(sn) && finiteS(ss);
      const bool cgv = twice > T(0) && finiteV(cn) && finiteS(cs);
      const size_t e = static_cast<size_t>(Tn) + c;
      tetGlob[2 * e] = {sgv ? ss : T(0), cgv ? cs : T(0), sgv ? T(1) : T(0), cgv ? T(1) : T(0)};
      tetGlob[2 * e + 1] = {0, 0, 1, 1};
    }
  }
  static bool localFailure(uint32_t s) {
    return s == kStatusShiftLimit || s == kStatusNonDescent || s == kStatusLineSearchFailed ||
           s == kStatusNonfinite || s == kStatusCholeskyFailed;
  }
  struct CandLane {
    T minDet[2];
    T energy[2];
    T maxShift;
    uint32_t failures, maxBacktracks, skipped, evals, bits;
  };
  static void addEnergy(CandLane& r, int which, T value, bool valid) {
    const uint32_t bit = which == 0 ? kSourceEnergyValid : kCandidateEnergyValid;
    if (valid) {
      const T sum = r.energy[which] + value;
      if (finiteS(sum)) r.energy[which] = sum;
      else { r.energy[which] = 0; r.bits &= ~bit; }
    } else {
      r.bits &= ~bit;
    }
  }
  void reduceCandidate() {
    std::vector<CandLane> lanes(kWorkgroup);
    for (uint32_t lane = 0; lane < kWorkgroup; ++lane) {
      CandLane r{{T(kF32Max), T(kF32Max)}, {0, 0}, 0, 0, 0, 0, 0, kReductionMask};
      for (uint32_t t = lane; t < Tn + C; t += kWorkgroup) {
        const V4<T> g = tetGlob[2 * t], e = tetGlob[2 * t + 1];
        const bool sgv = g.z == T(1) && finiteS(g.x), cgv = g.w == T(1) && finiteS(g.y);
        if (sgv) r.minDet[0] = std::min(r.minDet[0], g.x); else r.bits &= ~kSourceGeometryValid;
        if (cgv) r.minDet[1] = std::min(r.minDet[1], g.y); else r.bits &= ~kCandidateGeometryValid;
        addEnergy(r, 0, e.x, e.z == T(1) && finiteS(e.x));
        addEnergy(r, 1, e.y, e.w == T(1) && finiteS(e.y));
      }
      for (uint32_t v = lane; v < V; v += kWorkgroup) {
        const V4<T> l0 = local[4 * v], l1 = local[4 * v + 1], l2 = local[4 * v + 2], l3 = local[4 * v + 3];
        bool lnv = finite4(l0) && finite4(l1) && finite4(l2) && finite4(l3);
        const bool sv = finiteNonnegInt(l3.w, T(kStatusCholeskyFailed));
        uint32_t status = kStatusNonfinite;
        if (sv) status = static_cast<uint32_t>(l3.w);
        lnv = lnv && sv && status != kStatusNonfinite;
        if (localFailure(status)) r.failures += 1;
        if (finiteS(l1.w) && l1.w >= T(0)) r.maxShift = std::max(r.maxShift, l1.w); else lnv = false;
        const bool bv = finiteNonnegInt(l3.y, T(kMaxBacktracks));
        const bool ev = finiteNonnegInt(l3.z, T(kTrialCount));
        uint32_t back = 0, evals = 0;
        if (bv) back = static_cast<uint32_t>(l3.y); else lnv = false;
        if (ev) evals = static_cast<uint32_t>(l3.z); else lnv = false;
        r.maxBacktracks = std::max(r.maxBacktracks, back);
        r.evals += evals;
        uint32_t trials = 0;
        if (status == kStatusAccepted) trials = back + 1;
        else if (status == kStatusLineSearchFailed && back == kMaxBacktracks) trials = kTrialCount;
        else if (status == kStatusZeroGradient && back > 0) trials = back;
        else if (status == kStatusNonfinite) { trials = back; if (l3.x > T(kDeterminantFloor)) trials += 1; }
        r.skipped += trials - std::min(trials, evals);
        if (!lnv) r.bits &= ~kLocalNumericsValid;
        const V4<T> ve = vertexEnergy[v];
        addEnergy(r, 0, ve.x, ve.z == T(1) && finiteS(ve.x));
        addEnergy(r, 1, ve.y, ve.w == T(1) && finiteS(ve.y));
      }
      lanes[lane] = r;
    }
    for (uint32_t stride = kWorkgroup / 2; stride >= 1; stride /= 2) {
      for (uint32_t lane = 0; lane < stride; ++lane) {
        CandLane l = lanes[lane];
        const CandLane& r = lanes[lane + stride];
        l.minDet[0] = std::min(l.minDet[0], r.minDet[0]);
        l.minDet[1] = std::min(l.minDet[1], r.minDet[1]);
        for (int w = 0; w < 2; ++w) {
          const T sum = l.energy[w] + r.energy[w];
          if (finiteS(sum)) l.energy[w] = sum;
          else { l.energy[w] = 0; l.bits &= ~(w == 0 ? kSourceEnergyValid : kCandidateEnergyValid); }
        }
        l.maxShift = std::max(l.maxShift, r.maxShift);
        l.failures += r.failures;
        l.maxBacktracks = std::max(l.maxBacktracks, r.maxBacktracks);
        l.skipped += r.skipped;
        l.evals += r.evals;
        l.bits &= r.bits;
        lanes[lane] = l;
      }
    }
    if (latched()) return;
    const CandLane& a = lanes[0];
    uint32_t bits = a.bits;
    if (Tn == 0) bits &= ~(kSourceGeometryValid | kCandidateGeometryValid);
    const bool sgv = (bits & kSourceGeometryValid) != 0, cgv = (bits & kCandidateGeometryValid) != 0;
    const bool sev = (bits & kSourceEnergyValid) != 0, cev = (bits & kCandidateEnergyValid) != 0;
    const T sm = a.minDet[0], cm = a.minDet[1];
    const bool accepted = (sgv && sm > T(kDeterminantFloor)) && (cgv && cm > T(kDeterminantFloor));
    const T am = accepted ? cm : sm;
    const bool amv = accepted ? cgv : sgv;
    const T ae = accepted ? a.energy[1] : a.energy[0];
    const bool aev = accepted ? cev : sev;
    if (amv) bits |= kAcceptedMinimumValid;
    uint32_t historyIndex = 0;
    const T packed = control[1].w;
    if (finiteNonnegInt(packed, T(kHistoryCapacity))) historyIndex = static_cast<uint32_t>(packed);
    else bits &= ~kLocalNumericsValid;
    const uint32_t cbits = bits & kValidityMask;
    control[0] = {sgv ? sm : T(0), cgv ? cm : T(0), amv ? am : T(0), T(cbits)};
    control[1] = {accepted ? T(1) : T(0), accepted ? T(0) : T(1), T(a.failures), T(historyIndex)};
    control[2] = {sev ? a.energy[0] : T(0), cev ? a.energy[1] : T(0), aev ? ae : T(0), (sev && cev) ? T(1) : T(0)};
    control[3] = {a.maxShift, T(a.maxBacktracks), T(a.skipped), T(a.evals)};
  }
  void applyCandidate() {
    if (latched()) return;
    const bool accepted = control[1].x == T(1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) {
      const uint32_t v = static_cast<uint32_t>(i);
      if (!accepted) {
        (*tgt)[v] = (*src)[v];
        finalUpdate[v] = {0, 0, 0, 1};
        continue;
      }
      finalUpdate[v] = {scaledLength((*tgt)[v] - (*src)[v]), 0, 0, 1};
    }
  }
  void convergenceGradient() {
    if (latched()) return;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) {
      const uint32_t v = static_cast<uint32_t>(i);
      V4<T>* base = &conv[5 * v];
      if (pinned(v)) {
        for (int c = 0; c < 5; ++c) base[c] = {0, 0, 0, 0};
        continue;
      }
      const V3<T> p = (*tgt)[v];
      const V3<T> inertia = restMass[v].w * invDt2 * (p - predicted[v]);
      V3<T> ef = v3<T>(0, 0, 0), tgr = v3<T>(0, 0, 0);
      if (objectiveFlags != 0) {
        if (forceEnabled()) ef = -force(v);
        if (targetEnabled()) {
          const V4<T> t = targetRecord(v);
          if (t.w > T(0)) tgr = t.w * (p - v3(t.x, t.y, t.z));
        }
      }
      V3<T> material = v3<T>(0, 0, 0);
      const uint32_t start = info[4 * v], count = info[4 * v + 1];
      for (uint32_t a = 0; a < count; ++a) {
        const uint32_t t = adjacency[start + a];
        const uint32_t slot = slotOf(tetIndices(t), v);
        if (slot < 4) {
          V3<T> g[4];
          stableGradientAt(t, *tgt, g);
          material = material + g[slot];
        }
      }
      clothLocal(v, *tgt, &material, nullptr);
      V3<T> contact = v3<T>(0, 0, 0);
      if (st.floorStiffness > 0 && p.y < static_cast<T>(st.floorHeight))
        contact.y = static_cast<T>(st.floorStiffness) * (p.y - static_cast<T>(st.floorHeight));
      contactLocal(v, *tgt, false, &contact, nullptr);
      base[0] = {inertia.x, inertia.y, inertia.z, 0};
      base[1] = {material.x, material.y, material.z, 0};
      base[2] = {ef.x, ef.y, ef.z, 0};
      base[3] = {tgr.x, tgr.y, tgr.z, 0};
      base[4] = {contact.x, contact.y, contact.z, 0};
    }
  }
  struct ConvLane {
    T ch[6];  // four first channels, final x, final y
    T maxUpdate;
    uint32_t valid;
  };
  void reduceConvergence() {
    std::vector<ConvLane> lanes(kWorkgroup);
    auto comp3 = [&](uint32_t v, int c) { const V4<T> q = conv[5 * v + c]; return v3(q.x, q.y, q.z); };
    for (uint32_t lane = 0; lane < kWorkgroup; ++lane) {
      ConvLane r{{0, 0, 0, 0, 0, 0}, 0, 1};
      for (uint32_t v = lane; v < V; v += kWorkgroup) {
        V3<T> total = v3<T>(0, 0, 0);
        bool tv = true;
        for (int c = 0; c < 5; ++c) {
          const V3<T> raw = comp3(v, c);
          const bool ok = finiteV(raw);
          const V3<T> val = ok ? raw : v3<T>(0, 0, 0);
          const T sc = std::max(std::fabs(val.x), std::max(std::fabs(val.y), std::fabs(val.z)));
          r.ch[c] = std::max(r.ch[c], sc);
          total = total + val;
          tv = tv && ok;
        }
        tv = tv && finiteV(total);
        if (tv) r.ch[5] = std::max(r.ch[5], std::max(std::fabs(total.x), std::max(std::fabs(total.y), std::fabs(total.z))));
        else r.valid = 0;
        const T u = finalUpdate[v].x;
        if (finiteS(u) && u >= T(0)) r.maxUpdate = std::max(r.maxUpdate, u);
        else r.valid = 0;
      }
      lanes[lane] = r;
    }
    for (uint32_t stride = kWorkgroup / 2; stride >= 1; stride /= 2)
      for (uint32_t lane = 0; lane < stride; ++lane) {
        ConvLane& l = lanes[lane];
        const ConvLane& r = lanes[lane + stride];
        for (int c = 0; c < 6; ++c) l.ch[c] = std::max(l.ch[c], r.ch[c]);
        l.maxUpdate = std::max(l.maxUpdate, r.maxUpdate);
        l.valid &= r.valid;
      }
    const ConvLane scales = lanes[0];
    for (uint32_t lane = 0; lane < kWorkgroup; ++lane) {
      ConvLane r{{0, 0, 0, 0, 0, 0}, 0, 1};
      for (uint32_t v = lane; v < V; v += kWorkgroup) {
        V3<T> total = v3<T>(0, 0, 0);
        bool tv = true;
        for (int c = 0; c < 5; ++c) {
          const V3<T> raw = comp3(v, c);
          const bool ok = finiteV(raw);
          const V3<T> val = ok ? raw : v3<T>(0, 0, 0);
          const T sc = scales.ch[c];
          T sq = 0;
          if (ok && sc > T(0)) { const V3<T> n = val / sc; sq = dot(n, n); }
          const bool sqv = finiteS(sq) && sq >= T(0);
          const T sum = r.ch[c] + sq;
          if (sqv && finiteS(sum)) r.ch[c] = sum;
          else { r.ch[c] = 0; r.valid = 0; }
          total = total + val;
          tv = tv && ok;
        }
        tv = tv && finiteV(total);
        T ts = 0;
        if (tv && scales.ch[5] > T(0)) { const V3<T> n = total / scales.ch[5]; ts = dot(n, n); }
        const T tss = r.ch[5] + ts;
        if (tv && finiteS(ts) && ts >= T(0) && finiteS(tss)) r.ch[5] = tss;
        else { r.ch[5] = 0; r.valid = 0; }
      }
      lanes[lane] = r;
    }
    for (uint32_t stride = kWorkgroup / 2; stride >= 1; stride /= 2)
      for (uint32_t lane = 0; lane < stride; ++lane) {
        ConvLane& l = lanes[lane];
        const ConvLane& r = lanes[lane + stride];
        for (int c = 0; c < 6; ++c) {
          const T s = l.ch[c] + r.ch[c];
          if (finiteS(s)) l.ch[c] = s;
          else { l.ch[c] = 0; l.valid = 0; }
        }
        l.valid &= r.valid;
      }
    if (latched()) return;
    const ConvLane& sums = lanes[0];
    T norms[5];
    for (int c = 0; c < 5; ++c) norms[c] = scales.ch[c] * std::sqrt(sums.ch[c]);
    const T gnorm = scales.ch[5] * std::sqrt(sums.ch[5]);
    bool cnv = scales.valid == 1 && sums.valid == 1;
    for (int c = 0; c < 5; ++c) cnv = cnv && finiteS(norms[c]) && norms[c] >= T(0);
    const T den = std::max(T(1), norms[0] + norms[1] + norms[2] + norms[3] + norms[4]);
    const T rel = gnorm / den;
    const bool rnv = cnv && finiteS(gnorm) && gnorm >= T(0) && finiteS(den) && den >= T(1) && finiteS(rel) && rel >= T(0);
    const bool ssv = finiteS(sceneScale) && sceneScale >= T(0);
    const T nmu = scales.maxUpdate / std::max(ssv ? sceneScale : T(1.0e-12), T(1.0e-12));
    const bool unv = scales.valid == 1 && ssv && finiteS(scales.maxUpdate) && scales.maxUpdate >= T(0) &&
                     finiteS(nmu) && nmu >= T(0);
    const V4<T> geometry = control[0];
    const uint32_t cb = validityBits(geometry.w);
    const bool sgv = (cb & kSourceGeometryValid) != 0 && finiteS(geometry.x);
    const bool cgv = (cb & kCandidateGeometryValid) != 0 && finiteS(geometry.y);
    const bool amv = (cb & kAcceptedMinimumValid) != 0 && finiteS(geometry.z);
    const bool lnv = (cb & kLocalNumericsValid) != 0;
    const V4<T> acc = control[1];
    const bool aav = finiteNonnegInt(acc.x, T(1)), arv = finiteNonnegInt(acc.y, T(1));
    const bool lfv = finiteNonnegInt(acc.z, T(V));
    const bool hiv = finiteNonnegInt(acc.w, T(kHistoryCapacity));
    const bool aa = aav && acc.x == T(1), ar = arv && acc.y == T(1);
    uint32_t failures = 0, hi = 0;
    if (lfv) failures = static_cast<uint32_t>(acc.z);
    if (hiv) hi = static_cast<uint32_t>(acc.w);
    const V4<T> cm = control[3];
    const bool cmv = finiteS(cm.x) && cm.x >= T(0) && finiteNonnegInt(cm.y, T(kMaxBacktracks)) &&
                     finiteNonnegInt(cm.z, T(V) * T(kTrialCount)) && finiteNonnegInt(cm.w, T(V) * T(kTrialCount));
    const bool fin = rnv && unv && sgv && cgv && amv && lnv && aav && arv && lfv && hiv && cmv;
    const bool rs = fin && rel <= static_cast<T>(st.residualTolerance);
    const bool us = fin && nmu <= static_cast<T>(st.normalizedUpdateTolerance);
    const bool conv_ = rs && us && aa && !ar && failures == 0;
    if (hiv && hi < kHistoryCapacity) {
      V4<T>* h = &history[8 * hi];
      h[0] = control[0];
      h[1] = {acc.x, acc.y, acc.z, ar ? T(1) : T(0)};
      h[2] = control[2];
      h[3] = {cnv ? norms[0] : T(0), cnv ? norms[1] : T(0), cnv ? norms[2] : T(0), cnv ? norms[3] : T(0)};
      h[4] = {cnv ? norms[4] : T(0), rnv ? gnorm : T(0), rnv ? den : T(0), rnv ? rel : T(0)};
      h[5] = {unv ? scales.maxUpdate : T(0), unv ? nmu : T(0), rs ? T(1) : T(0), us ? T(1) : T(0)};
      h[6] = {conv_ ? T(1) : T(0), fin ? T(1) : T(0), T(hi), cmv ? cm.x : T(0)};
      h[7] = {cmv ? cm.y : T(0), cmv ? cm.z : T(0), cmv ? cm.w : T(0), T(1)};
    }
    control[1].w = T(hi + 1);
    if (conv_ && stopEnabled) control[0].w = T(cb | kStopLatch);
  }
  void copyPosition() {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) (*tgt)[i] = (*src)[i];
  }
  void bodyCorrection() {
    std::vector<T> corr(2 * bodyCount, T(0));
    for (uint32_t b = 0; b < bodyCount; ++b) {
      T total = 0, sx = 0, sz = 0, px = 0, pz = 0;
      bool hasPinned = false;
      for (uint32_t v = 0; v < V; ++v) {
        if (info[4 * v + 3] != b) continue;
        hasPinned = hasPinned || pinned(v);
        const T m = std::max(restMass[v].w, T(0));
        total += m;
        sx += m * posA[v].x; sz += m * posA[v].z;
        px += m * predicted[v].x; pz += m * predicted[v].z;
      }
      if (!hasPinned && total > T(0)) { corr[2 * b] = (px - sx) / total; corr[2 * b + 1] = (pz - sz) / total; }
    }
    for (uint32_t v = 0; v < V; ++v) {
      if (pinned(v)) continue;
      const uint32_t b = info[4 * v + 3];
      if (b >= bodyCount) continue;
      posA[v].x += corr[2 * b];
      posA[v].z += corr[2 * b + 1];
    }
  }
  void finalize() {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < V; ++i) {
      const uint32_t v = static_cast<uint32_t>(i);
      if (pinned(v)) {
        if (!glob) posA[v] = v3(restMass[v].x, restMass[v].y, restMass[v].z);
        velocity[v] = v3<T>(0, 0, 0);
        continue;
      }
      V3<T> vel = (posA[v] - old[v]) * invDt;
      if (st.floorStiffness > 0 && st.contactTangentialDamping > 0 &&
          posA[v].y <= static_cast<T>(st.floorHeight) + static_cast<T>(st.contactMargin)) {
        const T s = std::exp(-static_cast<T>(st.contactTangentialDamping) * dt);
        vel.x *= s;
        vel.z *= s;
      }
      velocity[v] = vel;
    }
  }
  void bind(std::vector<V3<T>>* s, std::vector<V3<T>>* t, int color) { src = s; tgt = t; activeColor = color; }

  // encodeFrame (src/simulation/gpu/jgs2-solver.ts:2207-2494), IPC/cloth off.
  void frame(uint32_t iterations) {
    // contactEnabled (jgs2-solver.ts:2213-2214).
    const bool contact = ipcEnabled();
    bind(&posA, &posA, -1);
    predict();
    if (contact) lagContact();
    if (glob) {
      candidateTetrahedron();
      reduceCandidate();
    }
    for (uint32_t it = 0; it < iterations; ++it) {
      std::vector<V3<T>>* s = (it % 2 == 0) ? &posB : &posA;
      std::vector<V3<T>>* t = (it % 2 == 0) ? &posA : &posB;
      bind(s, t, -1);
      if (contact) buildActiveRows();
      if (st.schedule == JGS2_SCHEDULE_GRAPH_COLORED_GAUSS_SEIDEL) {
        copyPosition();
        for (uint32_t c = 0; c < colorCount; ++c) {
          bind(t, t, static_cast<int>(c));
          tetPolarRotation();
          vertexPolarRotation();
          solveAll();
        }
        bind(s, t, -1);
        if (glob && !contact) assembledVertexEnergyAll();
      } else {
        tetPolarRotation();
        vertexPolarRotation();
        solveAll();
      }
      if (contact) {
        // Safe-step scaling of the candidate, exact validation of the scaled
        // pose (a failure restores the source), then the assembled energies
        // of the final pair (jgs2-solver.ts:2340-2393).
        contactStepAndReduce();
        applyContactStep();
        validateContactStep();
        applyContactStep();
        assembledVertexEnergyAll();
      }
      if (glob) {
        candidateTetrahedron();
        reduceCandidate();
        applyCandidate();
        if (contact) promoteContacts();
        convergenceGradient();
        reduceConvergence();
      }
    }
    if (iterations % 2 == 0) {
      bind(&posB, &posA, -1);
      copyPosition();
    }
    if (st.horizontalBodyCorrection) {
      bind(&posA, &posA, -1);
      bodyCorrection();
    }
    bind(&posA, &posA, -1);
    finalize();
  }
};

// buildGreedyVertexColoring (src/simulation/cpu/vertex-coloring.ts:20-110)
// over the conflict groups of buildJGS2InputVertexColoring
// (src/simulation/gpu/jgs2-solver.ts:308-367).
// computeJGS2InitialDynamicSceneScale (src/simulation/gpu/jgs2-solver.ts:732-768):
// the diagonal of the unpinned vertices' bounding box, in double; 1e-12
// (JGS2_DEGENERATE_DYNAMIC_SCENE_SCALE, :160) when no vertex is free or the box
// has no finite positive extent.
double initialDynamicSceneScale(const float* positions, const uint32_t* info, uint32_t V) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  uint32_t dyn = 0;
  for (uint32_t v = 0; v < V; ++v) {
    if (info[4ull * v + 2] != 0) continue;
    dyn++;
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], static_cast<double>(positions[4ull * v + k]));
      hi[k] = std::max(hi[k], static_cast<double>(positions[4ull * v + k]));
    }
  }
  const double diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                (hi[2] - lo[2]) * (hi[2] - lo[2]));
  return dyn > 0 && std::isfinite(diag) && diag > 0 ? diag : 1e-12;
}

std::vector<uint32_t> greedyColoring(const jgs2_input* in, uint32_t* countOut) {
  const uint32_t V = in->vertex_count;
  std::vector<std::vector<uint32_t>> adj(V);
  auto addGroup = [&](const uint32_t* g, int n) {
    uint32_t uniq[8];
    int u = 0;
    for (int i = 0; i < n; ++i) {
      bool seen = false;
      for (int j = 0; j < u; ++j) seen |= uniq[j] == g[i];
      if (!seen) uniq[u++] = g[i];
    }
    for (int a = 0; a < u; ++a)
      for (int b = a + 1; b < u; ++b) {
        adj[uniq[a]].push_back(uniq[b]);
        adj[uniq[b]].push_back(uniq[a]);
      }
  };
  for (uint32_t t = 0; t < in->tet_count; ++t) addGroup(&in->tet_indices[4ull * t], 4);
  for (uint32_t v = 0; v < V; ++v)
    for (uint32_t s = 0; s < in->cubature_k; ++s) {
      const size_t r = static_cast<size_t>(v) * in->cubature_k + s;
      const uint32_t t = in->cubature_tet_ids[r];
      if (t == kEmptyTet || in->cubature_weights[r] <= 0) continue;
      uint32_t g[5] = {v, in->tet_indices[4ull * t], in->tet_indices[4ull * t + 1], in->tet_indices[4ull * t + 2],
                       in->tet_indices[4ull * t + 3]};
      addGroup(g, 5);
    }
  if (in->cloth) {
    for (uint32_t c = 0; c < in->cloth->triangle_count; ++c) addGroup(&in->cloth->triangle_indices[3ull * c], 3);
    for (uint32_t h = 0; h < in->cloth->hinge_count; ++h) addGroup(&in->cloth->hinge_indices[4ull * h], 4);
  }
  if (in->contact_indices) {
    const uint64_t nc = uint64_t(in->contact_vertex_triangle_count) + in->contact_edge_edge_count;
    for (uint64_t c = 0; c < nc; ++c) addGroup(&in->contact_indices[4 * c], 4);
  }
  std::vector<uint32_t> colors(V, 0xffffffffu), stamp(V + 1, 0);
  uint32_t count = 0, st = 0;
  for (uint32_t v = 0; v < V; ++v) {
    st += 1;
    for (uint32_t n : adj[v])
      if (colors[n] != 0xffffffffu) stamp[colors[n]] = st;
    uint32_t c = 0;
    while (c < count && stamp[c] == st) c += 1;
    colors[v] = c;
    count = std::max(count, c + 1);
  }
  *countOut = count;
  return colors;
}

struct Handle {
  bool dbl = false;
  Oracle<float> f;
  Oracle<double> d;
  std::string error;
};

template <class T>
void initOracle(Oracle<T>& o, const jgs2_input* in) {
  o.V = in->vertex_count;
  o.Tn = in->tet_count;
  o.K = in->cubature_k;
  const uint32_t V = o.V, Tn = o.Tn;
  o.restMass.resize(V);
  o.info.assign(in->vertex_info, in->vertex_info + 4ull * V);
  uint32_t maxBody = 0;
  for (uint32_t v = 0; v < V; ++v) {
    o.restMass[v] = {in->vertex_rest[4 * v], in->vertex_rest[4 * v + 1], in->vertex_rest[4 * v + 2],
                     in->vertex_rest[4 * v + 3]};
    maxBody = std::max(maxBody, o.info[4 * v + 3]);
  }
  o.bodyCount = maxBody + 1;
  o.tetIdx.assign(in->tet_indices, in->tet_indices + 4ull * Tn);
  o.invDm.resize(Tn);
  o.meta.resize(Tn);
  uint32_t stable = 0;
  for (uint32_t t = 0; t < Tn; ++t) {
    const float* m = &in->tet_inverse_dm[12ull * t];
    o.invDm[t] = {{v3<T>(m[0], m[1], m[2]), v3<T>(m[4], m[5], m[6]), v3<T>(m[8], m[9], m[10])}};
    o.meta[t] = {in->tet_meta[4 * t], in->tet_meta[4 * t + 1], in->tet_meta[4 * t + 2], in->tet_meta[4 * t + 3]};
    stable += in->tet_meta[4 * t + 3] == 1.0f ? 1 : 0;
  }
  o.glob = stable == Tn;
  if (in->tet_rest_stiffness) o.stiffness.assign(in->tet_rest_stiffness, in->tet_rest_stiffness + 144ull * Tn);
  o.adjacency.assign(in->adjacency, in->adjacency + in->adjacency_length);
  const size_t R = static_cast<size_t>(V) * o.K;
  o.cubTet.assign(in->cubature_tet_ids, in->cubature_tet_ids + R);
  o.cubW.assign(in->cubature_weights, in->cubature_weights + R);
  o.cubBasis.assign(in->cubature_basis, in->cubature_basis + 36 * R);
  o.objectives.assign(2ull * V, {0, 0, 0, 0});
  uint32_t forces = 0, targets = 0;
  for (uint32_t v = 0; v < V; ++v) {
    if (in->external_forces) {
      o.objectives[2 * v] = {in->external_forces[3 * v], in->external_forces[3 * v + 1], in->external_forces[3 * v + 2], 0};
      if (in->external_forces[3 * v] != 0 || in->external_forces[3 * v + 1] != 0 || in->external_forces[3 * v + 2] != 0)
        forces++;
    }
    if (in->target_positions) {
      o.objectives[2 * v + 1] = {in->target_positions[3 * v], in->target_positions[3 * v + 1],
                                 in->target_positions[3 * v + 2], in->target_stiffnesses[v]};
      if (in->target_stiffnesses[v] > 0) targets++;
    } else {
      o.objectives[2 * v + 1] = {in->positions[4 * v], in->positions[4 * v + 1], in->positions[4 * v + 2], 0};
    }
  }
  o.objectiveFlags = (forces ? 1u : 0u) | (targets ? 2u : 0u);
  o.sceneScale = static_cast<T>(static_cast<float>(initialDynamicSceneScale(in->positions, o.info.data(), V)));
  o.posA.resize(V);
  for (uint32_t v = 0; v < V; ++v)
    o.posA[v] = v3<T>(in->positions[4 * v], in->positions[4 * v + 1], in->positions[4 * v + 2]);
  o.posB = o.posA;
  o.predicted = o.posA;
  o.old = o.posA;
  o.velocity.assign(V, v3<T>(0, 0, 0));
  if (in->velocities)
    for (uint32_t v = 0; v < V; ++v)
      o.velocity[v] = v3<T>(in->velocities[4 * v], in->velocities[4 * v + 1], in->velocities[4 * v + 2]);
  o.vertexRot.assign(V, identityM<T>());
  o.tetRot.assign(Tn, identityM<T>());
  o.finalUpdate.assign(V, {0, 0, 0, 0});
  o.local.assign(4ull * V, {0, 0, 0, 0});
  if (const jgs2_cloth_input* cl = in->cloth) {
    // packJGS2GpuClothArena (cloth-layout.ts:335-452): plane-stress Lame
    // parameters formed in double and stored as f32, incidence CSR rows.
    o.C = cl->triangle_count;
    o.H = cl->hinge_count;
    o.clothTri.assign(cl->triangle_indices, cl->triangle_indices + 3ull * o.C);
    o.clothInv.resize(o.C);
    o.clothArea.resize(o.C);
    for (uint32_t c = 0; c < o.C; ++c) {
      const float* b = &cl->triangle_inverse_rest_bases[4ull * c];
      o.clothInv[c] = {b[0], b[1], b[2], b[3]};
      o.clothArea[c] = cl->triangle_rest_areas[c];
    }
    o.hingeIdx.assign(cl->hinge_indices, cl->hinge_indices + 4ull * o.H);
    o.hingeAngle.resize(o.H);
    o.hingeLength.resize(o.H);
    for (uint32_t h = 0; h < o.H; ++h) {
      o.hingeAngle[h] = cl->hinge_rest_angles[h];
      o.hingeLength[h] = cl->hinge_rest_edge_lengths[h];
    }
    const double E = cl->young_modulus, nu = cl->poisson_ratio;
    o.clothLambda = static_cast<T>(static_cast<float>(E * nu / (1 - nu * nu)));
    o.clothMu = static_cast<T>(static_cast<float>(E / (2 * (1 + nu))));
    o.clothThickness = cl->thickness;
    o.clothBending = cl->bending_stiffness;
    auto csr = [&](const std::vector<uint32_t>& idx, uint32_t width, std::vector<uint32_t>& rows,
                   std::vector<uint32_t>& elems) {
      rows.assign(V + 1, 0);
      for (uint32_t q : idx) rows[q + 1] += 1;
      for (uint32_t v = 0; v < V; ++v) rows[v + 1] += rows[v];
      elems.assign(idx.size(), 0);
      std::vector<uint32_t> cursor(rows.begin(), rows.end() - 1);
      for (size_t e = 0; e < idx.size() / width; ++e)
        for (uint32_t l = 0; l < width; ++l) elems[cursor[idx[e * width + l]]++] = static_cast<uint32_t>(e);
    };
    csr(o.clothTri, 3, o.triRows, o.triElems);
    csr(o.hingeIdx, 4, o.hingeRows, o.hingeElems);
  }
  // Static IPC candidates (packIpcContactBuffer and
  // packIpcIncidentCandidateAdjacency, ipc-contact-layout.ts:190-342):
  // empty contact caches, zero lagged records, incidence CSR.
  o.NVT = in->contact_indices ? in->contact_vertex_triangle_count : 0;
  o.NC = in->contact_indices ? in->contact_vertex_triangle_count + in->contact_edge_edge_count : 0;
  o.cIdx.assign(in->contact_indices, in->contact_indices + 4ull * o.NC);
  o.cRows.assign(V + 1, 0);
  for (uint32_t q : o.cIdx) o.cRows[q + 1] += 1;
  for (uint32_t v = 0; v < V; ++v) o.cRows[v + 1] += o.cRows[v];
  o.cIds.assign(o.cIdx.size(), 0);
  {
    std::vector<uint32_t> cursor(o.cRows.begin(), o.cRows.end() - 1);
    for (uint32_t c = 0; c < o.NC; ++c)
      for (int l = 0; l < 4; ++l) o.cIds[cursor[o.cIdx[4ull * c + l]]++] = c;
  }
  o.activeCount.assign(V, 0);
  o.activeIds.assign(o.cIds.size(), 0);
  o.srcC.assign(o.NC, {0, 0, 0, T(-1)});
  o.tgtC.assign(o.NC, {0, 0, 0, T(-1)});
  o.srcW.assign(o.NC, {0, 0, 0, 0});
  o.tgtW.assign(o.NC, {0, 0, 0, 0});
  o.lagN.assign(o.NC, {0, 0, 0, 0});
  o.lagW.assign(o.NC, {0, 0, 0, 0});
  o.scratch.assign(o.NC, {1, 0, 0, 0});
  o.tetGlob.assign(2ull * (Tn + o.C), {0, 0, 0, 0});
  o.vertexEnergy.assign(V, {0, 0, 0, 0});
  o.conv.assign(5ull * V, {0, 0, 0, 0});
  for (auto& c : o.control) c = {0, 0, 0, 0};
  o.history.assign(8ull * kHistoryCapacity, {0, 0, 0, 0});
  o.colors = greedyColoring(in, &o.colorCount);
}

template <class T>
void applySettings(Oracle<T>& o, const jgs2_settings* s, bool stop) {
  o.st.schedule = s->schedule;
  o.st.iterations = s->iterations;
  o.st.timestep = s->timestep;
  for (int k = 0; k < 3; ++k) o.st.gravity[k] = s->gravity[k];
  o.st.floorHeight = s->floor_height;
  o.st.floorStiffness = s->floor_stiffness;
  o.st.velocityDamping = s->velocity_damping;
  o.st.regularization = s->regularization;
  o.st.rotationEpsilon = s->rotation_epsilon;
  o.st.maxStep = s->max_step;
  o.st.residualTolerance = s->residual_tolerance;
  o.st.normalizedUpdateTolerance = s->normalized_update_tolerance;
  o.st.contactTangentialDamping = s->contact_tangential_damping;
  o.st.contactMargin = s->contact_margin;
  o.st.horizontalBodyCorrection = s->horizontal_body_correction != 0;
  o.st.ipcActivation = s->ipc_activation_distance;
  o.st.ipcStiffness = s->ipc_barrier_stiffness;
  // resolveStepSettings (jgs2-solver.ts:1999-2009): body correction is off
  // while objectives or mesh contacts act on the stable path.
  if (o.glob && (o.objectiveFlags != 0 || (o.NC > 0 && s->ipc_barrier_stiffness > 0)))
    o.st.horizontalBodyCorrection = false;
  // packUniforms (src/simulation/gpu/jgs2-solver.ts:604-730): the time vec4
  // is (dt, 1/dt, 1/dt^2, maxStep), formed in double and stored as f32.
  const double dt = s->timestep;
  const double inv = 1.0 / dt;
  o.dt = static_cast<T>(static_cast<float>(dt));
  o.invDt = sizeof(T) == 8 ? static_cast<T>(inv) : static_cast<T>(static_cast<float>(inv));
  o.invDt2 = sizeof(T) == 8 ? static_cast<T>(inv * inv) : static_cast<T>(static_cast<float>(inv * inv));
  o.stopEnabled = o.glob && stop;
}

template <class T>
void readVec(const std::vector<V3<T>>& src, float* out) {
  for (size_t v = 0; v < src.size(); ++v) {
    out[4 * v] = static_cast<float>(src[v].x);
    out[4 * v + 1] = static_cast<float>(src[v].y);
    out[4 * v + 2] = static_cast<float>(src[v].z);
    out[4 * v + 3] = 0.f;
  }
}
template <class T>
void readVec4(const std::vector<V4<T>>& src, float* out) {
  for (size_t v = 0; v < src.size(); ++v) {
    out[4 * v] = static_cast<float>(src[v].x);
    out[4 * v + 1] = static_cast<float>(src[v].y);
    out[4 * v + 2] = static_cast<float>(src[v].z);
    out[4 * v + 3] = static_cast<float>(src[v].w);
  }
}

template <class T>
int readImpl(Oracle<T>& o, int which, float* out) {
  switch (which) {
    case 0: readVec(o.posA, out); for (uint32_t v = 0; v < o.V; ++v) out[4 * v + 3] = 1.f; return 0;
    case 1: readVec(o.velocity, out); return 0;
    case 2: readVec(o.predicted, out); for (uint32_t v = 0; v < o.V; ++v) out[4 * v + 3] = 1.f; return 0;
    case 3: readVec4(o.finalUpdate, out); return 0;
    case 4:
      for (uint32_t v = 0; v < o.V; ++v)
        for (int c = 0; c < 3; ++c) {
          out[12 * v + 4 * c] = static_cast<float>(o.vertexRot[v].c[c].x);
          out[12 * v + 4 * c + 1] = static_cast<float>(o.vertexRot[v].c[c].y);
          out[12 * v + 4 * c + 2] = static_cast<float>(o.vertexRot[v].c[c].z);
          out[12 * v + 4 * c + 3] = 0.f;
        }
      return 0;
    case 5: readVec4(o.local, out); return 0;
    case 6: {
      std::vector<V4<T>> c(o.control, o.control + 4);
      readVec4(c, out);
      return 0;
    }
    case 7: readVec4(o.history, out); return 0;
    case 8: readVec4(o.conv, out); return 0;
    case 9: readVec4(o.vertexEnergy, out); return 0;
    default: return 1;
  }
}

// Scalar contact helpers at either precision: which = 0 the Lipschitz safe
// step cap (source distance, minimum distance, displacement bound, safety),
// 1 the lagged friction dissipation (slip, threshold, coefficient, normal
// force), 2 the PSD normal Hessian block of normal (args 0-2) and scale
// (arg 3), written to out[0..8] by rows.  Returns the scalar (0 for which 2).
template <class T> double ipcScalar(int which, const double* a, double* out) {
  if (which == 0) return ipcSafeStepCap<T>(T(a[0]), T(a[1]), T(a[2]), T(a[3]));
  if (which == 1) return ipcFrictionDissipation<T>(T(a[0]), T(a[1]), T(a[2]), T(a[3]));
  const M3<T> h = ipcPsdNormalHessian(v3<T>(T(a[0]), T(a[1]), T(a[2])), T(a[3]));
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[3 * r + c] = comp(h.c[c], r);
  return 0;
}

}  // namespace

extern "C" {

// Oracle C API used by tests (ctypes).  `precision` is 32 or 64.
void* jgs2_oracle_create(const jgs2_input* input, int precision) {
  if (!input) return nullptr;
  Handle* h = new Handle();
  h->dbl = precision == 64;
  if (h->dbl) initOracle(h->d, input);
  else initOracle(h->f, input);
  return h;
}

void jgs2_oracle_destroy(void* handle) { delete static_cast<Handle*>(handle); }

// The create-time IPC parameters (minimum distance, friction coefficient,
// friction velocity smoothing, step safety), which the reference writes into
// the contact buffer once at create (jgs2-solver.ts:1096-1105).
int jgs2_oracle_fix_contact(void* handle, const jgs2_settings* s) {
  Handle* h = static_cast<Handle*>(handle);
  auto body = [&](auto& o) {
    using T = std::remove_reference_t<decltype(o.dt)>;
    o.ipcMinDistance = static_cast<T>(s->ipc_minimum_distance);
    o.ipcFriction = static_cast<T>(s->ipc_friction_coefficient);
    o.ipcEpsilon = static_cast<T>(s->ipc_friction_velocity_epsilon);
    o.ipcSafety = static_cast<T>(s->ipc_step_safety);
    o.contactFixed = true;
  };
  if (h->dbl) body(h->d); else body(h->f);
  return 0;
}

void jgs2_oracle_set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
}

int jgs2_oracle_max_threads(void) { return omp_get_max_threads(); }

uint32_t jgs2_oracle_color_count(void* handle) {
  Handle* h = static_cast<Handle*>(handle);
  return h->dbl ? h->d.colorCount : h->f.colorCount;
}

int jgs2_oracle_colors(void* handle, uint32_t* out) {
  Handle* h = static_cast<Handle*>(handle);
  const auto& c = h->dbl ? h->d.colors : h->f.colors;
  std::memcpy(out, c.data(), c.size() * sizeof(uint32_t));
  return 0;
}

// Advance `frames` frames with exactly `iterations` iterations each, using
// already-resolved settings.  stop != 0 enables the convergence stop latch
// (production step()); callers pass odd-normalised iterations in that case.
int jgs2_oracle_step(void* handle, const jgs2_settings* settings, uint32_t frames, uint32_t iterations,
                     int stop) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h || !settings) return 1;
  for (uint32_t f = 0; f < frames; ++f) {
    if (h->dbl) { applySettings(h->d, settings, stop != 0); h->d.frame(iterations); }
    else { applySettings(h->f, settings, stop != 0); h->f.frame(iterations); }
  }
  return 0;
}

// which: 0 positions, 1 velocities, 2 predicted, 3 final updates,
// 4 vertex rotations (12/vertex), 5 local diagnostics (16/vertex),
// 6 control (16), 7 history (64 * 32), 8 convergence components (20/vertex),
// 9 assembled vertex energies (4/vertex).
int jgs2_oracle_read(void* handle, int which, float* out) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h || !out) return 1;
  return h->dbl ? readImpl(h->d, which, out) : readImpl(h->f, which, out);
}

// Local system of one vertex at the current canonical pose, as the first
// Jacobi iteration of a frame would see it after predict: out[0..2] gradient,
// out[3..11] Hessian columns, out[12] restricted energy delta along `d`,
// out[13] restricted minimum determinant along `d`.  Runs predict, so the
// inertial target is refreshed (use on a fresh oracle only).
int jgs2_oracle_local_system(void* handle, const jgs2_settings* settings, uint32_t vertex, const double* d,
                             double* out) {
  Handle* h = static_cast<Handle*>(handle);
  auto body = [&](auto& o, auto zero) {
    using T = decltype(zero);
    applySettings(o, settings, false);
    o.bind(&o.posA, &o.posA, -1);
    o.predict();
    if (o.glob) { o.candidateTetrahedron(); o.reduceCandidate(); }
    o.bind(&o.posB, &o.posA, -1);
    o.tetPolarRotation();
    o.vertexPolarRotation();
    // Re-run the gather part of solveVertex.
    const uint32_t v = vertex;
    const V3<T> position = (*o.src)[v];
    const T inertia = o.restMass[v].w * o.invDt2;
    V3<T> gradient = inertia * (position - o.predicted[v]);
    M3<T> hessian = inertia * identityM<T>();
    if (o.objectiveFlags != 0) gradient = gradient + o.objectiveGradient(v, position);
    if (o.targetEnabled()) hessian = hessian + o.targetRecord(v).w * identityM<T>();
    const uint32_t start = o.info[4 * v], count = o.info[4 * v + 1];
    for (uint32_t a = 0; a < count; ++a) {
      const uint32_t t = o.adjacency[start + a];
      const uint32_t slot = o.slotOf(o.tetIndices(t), v);
      if (slot >= 4) continue;
      V3<T> tg[4];
      o.tetGradient(t, tg);
      gradient = gradient + tg[slot];
      hessian = hessian + o.stableLocalHessian(t, slot);
    }
    o.clothLocal(v, *o.src, &gradient, &hessian);
    for (uint32_t s = 0; s < o.K; ++s) {
      const size_t rec = static_cast<size_t>(v) * o.K + s;
      const uint32_t t = o.cubTet[rec];
      const T w = o.cubW[rec];
      if (t == kEmptyTet || t >= o.Tn || !(w > T(0))) continue;
      const uint32_t* q = o.tetIndices(t);
      M3<T> basis[4];
      o.currentBasis(rec, v, q, basis);
      V3<T> tg[4];
      o.tetGradient(t, tg);
      V3<T> pg = v3<T>(0, 0, 0);
      for (int l = 0; l < 4; ++l) pg = pg + transpose(basis[l]) * (tg[l] + o.distributedInertiaGradient(q[l]));
      if (o.objectiveFlags != 0)
        for (int l = 0; l < 4; ++l) pg = pg + transpose(basis[l]) * o.distributedObjectiveGradient(q[l]);
      M3<T> ph = o.cubatureHessian(t, basis);
      for (int l = 0; l < 4; ++l) ph = ph + o.distributedInertiaWeight(q[l]) * (transpose(basis[l]) * basis[l]);
      if (o.targetEnabled())
        for (int l = 0; l < 4; ++l)
          ph = ph + o.distributedTargetStiffness(q[l]) * (transpose(basis[l]) * basis[l]);
      const uint32_t ss = o.slotOf(q, v);
      if (ss < 4) {
        pg = pg - (tg[ss] + o.distributedInertiaGradient(v));
        if (o.objectiveFlags != 0) pg = pg - o.distributedObjectiveGradient(v);
        ph = ph - (o.stableLocalHessian(t, ss) + o.distributedInertiaWeight(v) * identityM<T>());
        if (o.targetEnabled()) ph = ph - o.distributedTargetStiffness(v) * identityM<T>();
      }
      gradient = gradient + w * pg;
      hessian = hessian + w * ph;
    }
    out[0] = gradient.x; out[1] = gradient.y; out[2] = gradient.z;
    for (int c = 0; c < 3; ++c) { out[3 + 3 * c] = hessian.c[c].x; out[4 + 3 * c] = hessian.c[c].y; out[5 + 3 * c] = hessian.c[c].z; }
    const V3<T> dd = v3<T>(static_cast<T>(d[0]), static_cast<T>(d[1]), static_cast<T>(d[2]));
    out[12] = o.restrictedEnergyDelta(v, dd);
    out[13] = o.restrictedMinimumDeterminant(v, dd).minimum;
  };
  if (h->dbl) body(h->d, 0.0); else body(h->f, 0.0f);
  return 0;
}

// Single cloth elements, for the closed-form and finite-difference checks of
// the reference's cloth tests (src/simulation/cpu/cloth.test.ts).
// Membrane: positions 9, row-major inverse rest basis 4; out = energy, 9
// gradient entries.  Bending: positions 12; out = energy, 12 gradient
// entries (k L (theta - theta0) dtheta/dx), valid flag.
}  // extern "C"
namespace {
template <class T>
void clothMembraneElement(const double* x, const double* inverse, double area, double young, double poisson,
                          double thickness, double* out) {
  Oracle<T> o;
  o.C = 1;
  o.clothTri = {0, 1, 2};
  o.clothInv = {{static_cast<T>(inverse[0]), static_cast<T>(inverse[1]), static_cast<T>(inverse[2]),
                 static_cast<T>(inverse[3])}};
  o.clothArea = {static_cast<T>(area)};
  o.clothLambda = static_cast<T>(young * poisson / (1 - poisson * poisson));
  o.clothMu = static_cast<T>(young / (2 * (1 + poisson)));
  o.clothThickness = static_cast<T>(thickness);
  std::vector<V3<T>> p(3);
  for (int l = 0; l < 3; ++l) p[l] = v3<T>(x[3 * l], x[3 * l + 1], x[3 * l + 2]);
  const auto m = o.membraneAt(0, p, 0xffffffffu, v3<T>(0, 0, 0));
  out[0] = m.energy;
  for (int l = 0; l < 3; ++l) { out[1 + 3 * l] = m.g[l].x; out[2 + 3 * l] = m.g[l].y; out[3 + 3 * l] = m.g[l].z; }
}
template <class T>
void clothBendingElement(const double* x, double restAngle, double restLength, double stiffness, double* out) {
  Oracle<T> o;
  o.H = 1;
  o.hingeIdx = {0, 1, 2, 3};
  o.hingeAngle = {static_cast<T>(restAngle)};
  o.hingeLength = {static_cast<T>(restLength)};
  o.clothBending = static_cast<T>(stiffness);
  std::vector<V3<T>> p(4);
  for (int l = 0; l < 4; ++l) p[l] = v3<T>(x[3 * l], x[3 * l + 1], x[3 * l + 2]);
  const auto d = o.dihedralAt(0, p, 0xffffffffu, v3<T>(0, 0, 0));
  out[0] = o.bendingEnergyAt(0, p, 0xffffffffu, v3<T>(0, 0, 0));
  const T diff = d.valid ? Oracle<T>::wrappedAngleDifference(d.angle, o.hingeAngle[0]) : T(0);
  const T ws = o.clothBending * o.hingeLength[0];
  for (int l = 0; l < 4; ++l) {
    const V3<T> g = ws * diff * d.g[l];
    out[1 + 3 * l] = g.x; out[2 + 3 * l] = g.y; out[3 + 3 * l] = g.z;
  }
  out[13] = d.valid ? 1.0 : 0.0;
}
template <class T>
void snhDensity(const double* f, const double* h, double lambda, double mu, double* out) {
  M3<T> F, H;
  for (int col = 0; col < 3; ++col) {
    F.c[col] = v3(static_cast<T>(f[col]), static_cast<T>(f[3 + col]), static_cast<T>(f[6 + col]));
    H.c[col] = v3(static_cast<T>(h[col]), static_cast<T>(h[3 + col]), static_cast<T>(h[6 + col]));
  }
  const T l = static_cast<T>(lambda), m = static_cast<T>(mu);
  const M3<T> P = snhPiola(F, l, m);
  const M3<T> dP = snhTangent(F, H, l, m);
  out[0] = snhEnergy(F, l, m);
  for (int row = 0; row < 3; ++row)
    for (int col = 0; col < 3; ++col) {
      out[1 + 3 * row + col] = at(P, col, row);
      out[10 + 3 * row + col] = at(dP, col, row);
    }
  out[19] = det(F);
}

template <class T>
void localSolve(const double* hessian, const double* gradient, double inertia, double* out) {
  M3<T> H;
  for (int col = 0; col < 3; ++col)
    H.c[col] = v3(static_cast<T>(hessian[col]), static_cast<T>(hessian[3 + col]), static_cast<T>(hessian[6 + col]));
  const V3<T> g = v3(static_cast<T>(gradient[0]), static_cast<T>(gradient[1]), static_cast<T>(gradient[2]));
  const SolveResult<T> r = globalizationSolve(H, g, static_cast<T>(inertia));
  out[0] = r.status;
  out[1] = r.direction.x; out[2] = r.direction.y; out[3] = r.direction.z;
  out[4] = r.gdd; out[5] = r.scale; out[6] = r.minEig; out[7] = r.shift; out[8] = r.asym; out[9] = r.residual;
}

}  // namespace
extern "C" {

// IPC scalar kernels and contact features for the reference's contact tests
// (src/simulation/cpu/ipc-contact.test.ts).  barrier: out = B, B', B''.
// friction: out = f1 and the lagged dissipation for (mu, lambda) = (1, 1).
// contact: type 0 = point-triangle (p, t0, t1, t2), 1 = edge-edge; out =
// distance, normal xyz, weights xyzw, valid.
int jgs2_oracle_ipc_barrier(double d, double dHat, int precision, double* out) {
  if (precision == 64) {
    out[0] = ipcBarrier(d, dHat); out[1] = ipcBarrier1(d, dHat); out[2] = ipcBarrier2(d, dHat);
  } else {
    const float a = static_cast<float>(d), b = static_cast<float>(dHat);
    out[0] = ipcBarrier(a, b); out[1] = ipcBarrier1(a, b); out[2] = ipcBarrier2(a, b);
  }
  return 0;
}

int jgs2_oracle_ipc_friction(double slip, double eps, double* out) {
  out[0] = ipcFrictionF1(slip, eps);
  out[1] = ipcFrictionDissipation(slip, eps, 1.0, 1.0);
  return 0;
}

double jgs2_oracle_ipc_scalar(int which, const double* args, int precision, double* out) {
  return precision == 64 ? ipcScalar<double>(which, args, out) : ipcScalar<float>(which, args, out);
}

int jgs2_oracle_ipc_contact(uint32_t type, const double* x, double* out) {
  V3<double> p[4];
  for (int l = 0; l < 4; ++l) p[l] = v3(x[3 * l], x[3 * l + 1], x[3 * l + 2]);
  const Contact<double> k = type == 0 ? ipcPointTriangle(p[0], p[1], p[2], p[3]) : ipcEdgeEdge(p[0], p[1], p[2], p[3]);
  out[0] = k.distance;
  out[1] = k.normal.x; out[2] = k.normal.y; out[3] = k.normal.z;
  out[4] = k.weights.x; out[5] = k.weights.y; out[6] = k.weights.z; out[7] = k.weights.w;
  out[8] = k.valid ? 1.0 : 0.0;
  return 0;
}

// The same contact features in the f32 mirror (inputs rounded to float,
// computed in float): the plain-f32 error against the FP64 run.
int jgs2_oracle_ipc_contact_f32(uint32_t type, const double* x, double* out) {
  V3<float> p[4];
  for (int l = 0; l < 4; ++l)
    p[l] = v3(static_cast<float>(x[3 * l]), static_cast<float>(x[3 * l + 1]), static_cast<float>(x[3 * l + 2]));
  const Contact<float> k = type == 0 ? ipcPointTriangle(p[0], p[1], p[2], p[3]) : ipcEdgeEdge(p[0], p[1], p[2], p[3]);
  out[0] = k.distance;
  out[1] = k.normal.x; out[2] = k.normal.y; out[3] = k.normal.z;
  out[4] = k.weights.x; out[5] = k.weights.y; out[6] = k.weights.z; out[7] = k.weights.w;
  out[8] = k.valid ? 1.0 : 0.0;
  return 0;
}

// Minimum exact contact distance over the candidates at the current pose.
double jgs2_oracle_min_contact_distance(void* handle) {
  Handle* h = static_cast<Handle*>(handle);
  auto body = [&](auto& o) {
    double m = 3.0e38;
    for (uint32_t c = 0; c < o.NC; ++c) {
      const auto k = o.contactAt(c, o.posA, static_cast<decltype(o.dt)>(kF32Max));
      if (k.valid) m = std::min(m, static_cast<double>(k.distance));
    }
    return m;
  };
  return h->dbl ? body(h->d) : body(h->f);
}

int jgs2_oracle_cloth_membrane(const double* positions, const double* inverse, double area, double young,
                               double poisson, double thickness, int precision, double* out) {
  if (precision == 64) clothMembraneElement<double>(positions, inverse, area, young, poisson, thickness, out);
  else clothMembraneElement<float>(positions, inverse, area, young, poisson, thickness, out);
  return 0;
}

int jgs2_oracle_cloth_bending(const double* positions, double rest_angle, double rest_length, double stiffness,
                              int precision, double* out) {
  if (precision == 64) clothBendingElement<double>(positions, rest_angle, rest_length, stiffness, out);
  else clothBendingElement<float>(positions, rest_angle, rest_length, stiffness, out);
  return 0;
}

// The stable Neo-Hookean density of the step (snhEnergy, snhPiola,
// snhTangent; stable-neo-hookean-wgsl.ts:14-95) for the reference's density
// tests (src/simulation/cpu/stable-neo-hookean.test.ts:53-232).  f and h are
// 3x3 matrices stored by rows.  out[0] = energy density, out[1..9] = first
// Piola stress by rows, out[10..18] = the tangent action dP(f)[h] by rows,
// out[19] = det f.  precision 32 rounds the inputs to float and evaluates in
// float.
// The local globalization solve (globalizationSolve, jgs2-globalization-wgsl.ts:
// 166-492) for the reference's globalization tests
// (src/simulation/cpu/nonlinear-globalization.test.ts:38-158).  hessian is
// 3x3 by rows, gradient 3 values, inertia the scale floor.  out[0] = status
// code, out[1..3] = direction, out[4] = gradient . direction, out[5] = the
// normalising scale, out[6] = minimum eigenvalue and out[7] = diagonal shift
// of the normalised system, out[8] = maximum relative asymmetry, out[9] =
// relative linear residual.
int jgs2_oracle_local_solve(const double* hessian, const double* gradient, double inertia, int precision,
                            double* out) {
  if (precision == 64) localSolve<double>(hessian, gradient, inertia, out);
  else localSolve<float>(hessian, gradient, inertia, out);
  return 0;
}

// The step's convergence reduction (reduceConvergence) on caller data, for
// the reference's convergence cases
// (src/simulation/cpu/nonlinear-iteration.test.ts:181-400).  components: 20
// floats per vertex, the inertia, material, external-force, target and
// contact gradients as xyz_ each; updates: the accepted update length per
// vertex; control: the 16-float control record (geometry minima and validity
// bits, accept / revert flags, failures, history index, energies, sweep
// aggregates); scene_scale < 0 keeps the input's.  history_out receives the
// 32-float history record the reduction writes.
int jgs2_oracle_reduce_convergence(void* handle, const jgs2_settings* settings, const float* components,
                                   const float* updates, const float* control, double scene_scale,
                                   float* history_out) {
  Handle* h = static_cast<Handle*>(handle);
  auto body = [&](auto& o) {
    using T = std::remove_reference_t<decltype(o.dt)>;
    applySettings(o, settings, false);
    for (uint32_t v = 0; v < o.V; ++v) {
      for (int c = 0; c < 5; ++c) {
        const float* q = components + 20ull * v + 4 * c;
        o.conv[5ull * v + c] = {static_cast<T>(q[0]), static_cast<T>(q[1]), static_cast<T>(q[2]), T(0)};
      }
      o.finalUpdate[v] = {static_cast<T>(updates[v]), T(0), T(0), T(0)};
    }
    for (int i = 0; i < 4; ++i)
      o.control[i] = {static_cast<T>(control[4 * i]), static_cast<T>(control[4 * i + 1]),
                      static_cast<T>(control[4 * i + 2]), static_cast<T>(control[4 * i + 3])};
    if (scene_scale >= 0) o.sceneScale = static_cast<T>(scene_scale);
    const float hiRaw = control[7];
    o.reduceConvergence();
    const uint32_t hi = hiRaw >= 0 && hiRaw < float(kHistoryCapacity) ? static_cast<uint32_t>(hiRaw) : 0u;
    for (int k = 0; k < 8; ++k) {
      const V4<T> r = o.history[8ull * hi + k];
      history_out[4 * k] = static_cast<float>(r.x);
      history_out[4 * k + 1] = static_cast<float>(r.y);
      history_out[4 * k + 2] = static_cast<float>(r.z);
      history_out[4 * k + 3] = static_cast<float>(r.w);
    }
  };
  if (h->dbl) body(h->d); else body(h->f);
  return 0;
}

// The initial convergence scene scale of a position / vertexInfo pair.
double jgs2_oracle_initial_scene_scale(const float* positions, const uint32_t* vertex_info, uint32_t vertex_count) {
  return initialDynamicSceneScale(positions, vertex_info, vertex_count);
}

// The closed-form minimum eigenvalue of the symmetric part's upper triangle
// (minSymmetricEigenvalue); m is 3x3 by rows.
double jgs2_oracle_min_symmetric_eigenvalue(const double* m, int precision) {
  if (precision == 64) {
    M3<double> a;
    for (int col = 0; col < 3; ++col) a.c[col] = v3(m[col], m[3 + col], m[6 + col]);
    return minSymmetricEigenvalue(a);
  }
  M3<float> a;
  for (int col = 0; col < 3; ++col)
    a.c[col] = v3(static_cast<float>(m[col]), static_cast<float>(m[3 + col]), static_cast<float>(m[6 + col]));
  return minSymmetricEigenvalue(a);
}

int jgs2_oracle_snh_density(const double* f, const double* h, double lambda, double mu, int precision,
                            double* out) {
  if (precision == 64) snhDensity<double>(f, h, lambda, mu, out);
  else snhDensity<float>(f, h, lambda, mu, out);
  return 0;
}

// evaluateAssembledCandidateForTest (src/simulation/gpu/jgs2-solver.ts:2611-2726):
// posB = source, posA = candidate, predicted = source, local records and
// control cleared, then assembled energies, the determinant gate and the
// convergence reduction of one iteration.  Poses are 4 floats per vertex.
int jgs2_oracle_evaluate_candidate(void* handle, const jgs2_settings* settings, const float* source,
                                   const float* candidate) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h || !settings || !source || !candidate) return 1;
  auto body = [&](auto& o, auto zero) {
    using T = decltype(zero);
    applySettings(o, settings, false);
    for (uint32_t v = 0; v < o.V; ++v) {
      o.posB[v] = v3<T>(source[4 * v], source[4 * v + 1], source[4 * v + 2]);
      o.posA[v] = v3<T>(candidate[4 * v], candidate[4 * v + 1], candidate[4 * v + 2]);
      o.predicted[v] = o.posB[v];
    }
    for (auto& l : o.local) l = {0, 0, 0, 0};
    for (auto& c : o.control) c = {0, 0, 0, 0};
    o.bind(&o.posB, &o.posA, -1);
    o.assembledVertexEnergyAll();
    o.candidateTetrahedron();
    o.reduceCandidate();
    o.applyCandidate();
    o.convergenceGradient();
    o.reduceConvergence();
  };
  if (h->dbl) body(h->d, 0.0); else body(h->f, 0.0f);
  return 0;
}

// Replace the objective records (forces 3V, targets 3V + stiffness V); NULL
// arrays are left unchanged.  Recomputes the activity flags.
int jgs2_oracle_set_objectives(void* handle, const float* forces, const float* targets, const float* stiffness) {
  Handle* h = static_cast<Handle*>(handle);
  auto apply = [&](auto& o) {
    uint32_t nf = 0, nt = 0;
    for (uint32_t v = 0; v < o.V; ++v) {
      if (forces) { o.objectives[2 * v].x = forces[3 * v]; o.objectives[2 * v].y = forces[3 * v + 1]; o.objectives[2 * v].z = forces[3 * v + 2]; }
      if (targets) {
        o.objectives[2 * v + 1].x = targets[3 * v];
        o.objectives[2 * v + 1].y = targets[3 * v + 1];
        o.objectives[2 * v + 1].z = targets[3 * v + 2];
        o.objectives[2 * v + 1].w = stiffness[v];
      }
      const auto& f = o.objectives[2 * v];
      if (f.x != 0 || f.y != 0 || f.z != 0) nf++;
      if (o.objectives[2 * v + 1].w > 0) nt++;
    }
    o.objectiveFlags = (nf ? 1u : 0u) | (nt ? 2u : 0u);
  };
  if (h->dbl) apply(h->d); else apply(h->f);
  return 0;
}

}  // extern "C"
