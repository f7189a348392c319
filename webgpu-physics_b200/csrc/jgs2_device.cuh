// Device math for the JGS2 step on sm_100a: 3x3 algebra, the stable
// Neo-Hookean material, and the fail-closed local globalization solve.
//
// Formulas restate the reference's WGSL libraries
//   stable Neo-Hookean       src/simulation/gpu/stable-neo-hookean-wgsl.ts:14-95
//   globalization            src/simulation/gpu/jgs2-globalization-wgsl.ts:26-560
// with two algebraic rewrites that are exact in real arithmetic:
//   * the incident local Hessian block of vertex slot s is formed in closed
//     form, vol * (a |g|^2 I + c1 (F g)(F g)^T + lambda (cof F g)(cof F g)^T),
//     because the directional cofactor term D cof[e_d g^T] g vanishes
//     identically for a rank-one direction (det is affine in each column);
//   * projected (cubature) gradients and Hessians are written as Frobenius
//     products with the projected directions dF_r = sum_l B_l[:,r] g_l^T, so
//     the 12x12 element Hessian is never formed.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace jgs2 {

// ---- constants (jgs2-globalization-wgsl.ts:27-37; jgs2-shader.ts:64-118) ----
constexpr float kF32Max = 3.0e38f;
constexpr float kUnitRoundoff = 0.000000059604644775390625f;
constexpr float kPositionResolutionMultiplier = 8.0f;
constexpr float kRelativeEigenvalueFloor = 0.0000152587890625f;
constexpr float kMaxNormalizedShift = 0.001f;
constexpr float kArmijoC1 = 0.0001f;
constexpr float kBacktrackFactor = 0.5f;
constexpr uint32_t kMaxBacktracks = 12u;
constexpr uint32_t kTrialCount = 13u;
constexpr float kDeterminantFloor = 0.0001f;
constexpr float kTwoPiOverThree = 2.0943951023931953f;
constexpr uint32_t kEmptyTet = 0xffffffffu;
constexpr uint32_t kHistoryCapacity = 64u;

enum LocalStatus : uint32_t {
  kAccepted = 0, kPinned = 1, kZeroGradient = 2, kShiftLimit = 3, kNonDescent = 4,
  kLineSearchFailed = 5, kNonfinite = 6, kCholeskyFailed = 7,
};
enum ValidityBits : uint32_t {
  kSourceGeometryValid = 1u, kCandidateGeometryValid = 2u, kAcceptedMinimumValid = 4u,
  kLocalNumericsValid = 8u, kValidityMask = 15u, kStopLatchBit = 16u, kControlMask = 31u,
  kSourceEnergyValid = 16u, kCandidateEnergyValid = 32u,
};

struct M3 {  // three columns, like WGSL mat3x3f
  float3 c0, c1, c2;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

__device__ __forceinline__ M3 mzero() { return {f3(0, 0, 0), f3(0, 0, 0), f3(0, 0, 0)}; }
__device__ __forceinline__ M3 midentity() { return {f3(1, 0, 0), f3(0, 1, 0), f3(0, 0, 1)}; }
__device__ __forceinline__ M3 operator+(const M3& a, const M3& b) { return {a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2}; }
__device__ __forceinline__ M3 operator-(const M3& a, const M3& b) { return {a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2}; }
__device__ __forceinline__ M3 operator*(float s, const M3& a) { return {s * a.c0, s * a.c1, s * a.c2}; }
__device__ __forceinline__ float3 mv(const M3& m, float3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
// m^T v
__device__ __forceinline__ float3 mtv(const M3& m, float3 v) { return f3(dot3(m.c0, v), dot3(m.c1, v), dot3(m.c2, v)); }
__device__ __forceinline__ M3 mm(const M3& a, const M3& b) { return {mv(a, b.c0), mv(a, b.c1), mv(a, b.c2)}; }
__device__ __forceinline__ M3 mtrans(const M3& m) {
  return {f3(m.c0.x, m.c1.x, m.c2.x), f3(m.c0.y, m.c1.y, m.c2.y), f3(m.c0.z, m.c1.z, m.c2.z)};
}
// a b^T  (columns a * b_j)
__device__ __forceinline__ M3 outer(float3 a, float3 b) { return {a * b.x, a * b.y, a * b.z}; }
__device__ __forceinline__ float mdet(const M3& m) { return dot3(m.c0, cross3(m.c1, m.c2)); }
__device__ __forceinline__ float frob(const M3& a, const M3& b) {
  return dot3(a.c0, b.c0) + dot3(a.c1, b.c1) + dot3(a.c2, b.c2);
}
__device__ __forceinline__ M3 cofactor(const M3& f) {
  return {cross3(f.c1, f.c2), cross3(f.c2, f.c0), cross3(f.c0, f.c1)};
}
__device__ __forceinline__ M3 dcofactor(const M3& f, const M3& h) {
  return {cross3(h.c1, f.c2) + cross3(f.c1, h.c2), cross3(h.c2, f.c0) + cross3(f.c2, h.c0),
          cross3(h.c0, f.c1) + cross3(f.c0, h.c1)};
}

__device__ __forceinline__ bool finiteS(float v) { return v == v && fabsf(v) <= kF32Max; }
__device__ __forceinline__ bool finiteV(float3 v) { return finiteS(v.x) && finiteS(v.y) && finiteS(v.z); }
__device__ __forceinline__ bool finiteM(const M3& m) { return finiteV(m.c0) && finiteV(m.c1) && finiteV(m.c2); }

// Symmetric 3x3 stored as (xx, yy, zz, xy, xz, yz).
struct S3 {
  float xx, yy, zz, xy, xz, yz;
};
__device__ __forceinline__ S3 szero() { return {0, 0, 0, 0, 0, 0}; }
__device__ __forceinline__ void sadd(S3& a, const S3& b) {
  a.xx += b.xx; a.yy += b.yy; a.zz += b.zz; a.xy += b.xy; a.xz += b.xz; a.yz += b.yz;
}
__device__ __forceinline__ void saddScaled(S3& a, float s, const S3& b) {
  a.xx += s * b.xx; a.yy += s * b.yy; a.zz += s * b.zz; a.xy += s * b.xy; a.xz += s * b.xz; a.yz += s * b.yz;
}
__device__ __forceinline__ void saddOuter(S3& a, float s, float3 u) {
  a.xx += s * u.x * u.x; a.yy += s * u.y * u.y; a.zz += s * u.z * u.z;
  a.xy += s * u.x * u.y; a.xz += s * u.x * u.z; a.yz += s * u.y * u.z;
}
__device__ __forceinline__ void saddDiag(S3& a, float s) { a.xx += s; a.yy += s; a.zz += s; }
__device__ __forceinline__ float3 smv(const S3& a, float3 v) {
  return f3(a.xx * v.x + a.xy * v.y + a.xz * v.z, a.xy * v.x + a.yy * v.y + a.yz * v.z,
            a.xz * v.x + a.yz * v.y + a.zz * v.z);
}
// B^T B for a 3x3 B (columns).
// R S R^T of a symmetric S.
__device__ __forceinline__ S3 srotate(const M3& r, const S3& s) {
  const M3 rs = {mv(r, f3(s.xx, s.xy, s.xz)), mv(r, f3(s.xy, s.yy, s.yz)), mv(r, f3(s.xz, s.yz, s.zz))};
  // (R S R^T)_ij = row i of R S . row j of R
  const float3 a0 = f3(rs.c0.x, rs.c1.x, rs.c2.x), a1 = f3(rs.c0.y, rs.c1.y, rs.c2.y);
  const float3 a2 = f3(rs.c0.z, rs.c1.z, rs.c2.z);
  const float3 r0 = f3(r.c0.x, r.c1.x, r.c2.x), r1 = f3(r.c0.y, r.c1.y, r.c2.y), r2 = f3(r.c0.z, r.c1.z, r.c2.z);
  return {dot3(a0, r0), dot3(a1, r1), dot3(a2, r2), dot3(a0, r1), dot3(a0, r2), dot3(a1, r2)};
}
__device__ __forceinline__ S3 gramColumns(const M3& b) {
  return {dot3(b.c0, b.c0), dot3(b.c1, b.c1), dot3(b.c2, b.c2), dot3(b.c0, b.c1), dot3(b.c0, b.c2), dot3(b.c1, b.c2)};
}

// ---- compensated summation of the per-vertex gradient gathers --------------
// Knuth's TwoSum: t = fl(a + b) and the exact rounding error e with
// a + b = t + e, from six round-to-nearest operations.  The intrinsics keep
// the compiler from contracting or reassociating them.  The error is unique,
// so TwoSum(a, b) and TwoSum(b, a) give the same pair.
__device__ __forceinline__ float twoSum(float a, float b, float* e) {
  const float t = __fadd_rn(a, b);
  const float bp = __fsub_rn(t, a);
  *e = __fadd_rn(__fsub_rn(a, __fsub_rn(t, bp)), __fsub_rn(b, bp));
  return t;
}
// A float3 sum carried as value + compensation (Kahan-Babuska summation in
// Neumaier's form): each addend's rounding error is kept in `c`, and the
// result is rounded once at the end.  The error of a gather of n terms is
// then about one rounding of the result plus n u^2 of the terms, instead of
// n u of the terms for a plain f32 sum.
struct Comp3 {
  float3 s, c;
};
__device__ __forceinline__ Comp3 czero() { return {f3(0, 0, 0), f3(0, 0, 0)}; }
__device__ __forceinline__ void cadd(Comp3& a, float3 x) {
  float ex, ey, ez;
  a.s.x = twoSum(a.s.x, x.x, &ex);
  a.s.y = twoSum(a.s.y, x.y, &ey);
  a.s.z = twoSum(a.s.z, x.z, &ez);
  a.c.x = __fadd_rn(a.c.x, ex);
  a.c.y = __fadd_rn(a.c.y, ey);
  a.c.z = __fadd_rn(a.c.z, ez);
}
// Merge two compensated sums (symmetric in its arguments).
__device__ __forceinline__ void cmerge(Comp3& a, const Comp3& b) {
  float ex, ey, ez;
  a.s.x = twoSum(a.s.x, b.s.x, &ex);
  a.s.y = twoSum(a.s.y, b.s.y, &ey);
  a.s.z = twoSum(a.s.z, b.s.z, &ez);
  a.c.x = __fadd_rn(__fadd_rn(a.c.x, b.c.x), ex);
  a.c.y = __fadd_rn(__fadd_rn(a.c.y, b.c.y), ey);
  a.c.z = __fadd_rn(__fadd_rn(a.c.z, b.c.z), ez);
}
__device__ __forceinline__ float3 cvalue(const Comp3& a) {
  return f3(__fadd_rn(a.s.x, a.c.x), __fadd_rn(a.s.y, a.c.y), __fadd_rn(a.s.z, a.c.z));
}
// Gradient accumulation into a plain or a compensated sum.
__device__ __forceinline__ void gadd(float3& g, float3 x) { g = g + x; }
__device__ __forceinline__ void gadd(Comp3& g, float3 x) { cadd(g, x); }

// ---- stable Neo-Hookean (stable-neo-hookean-wgsl.ts:44-94) -------------------
__device__ __forceinline__ float snhEnergy(const M3& f, float lambda, float mu) {
  const float I1 = frob(f, f);
  const float dj = mdet(f) - 1.0f;
  return 0.5f * mu * (I1 - 3.0f) - 0.75f * mu * dj + 0.5f * lambda * dj * dj -
         0.5f * mu * logf((I1 + 1.0f) * 0.25f);
}

struct PiolaTerms {
  M3 cof;
  float I1, J, a, b, c1;  // P = a F + b cof;  c1 = 2 mu / (I1 + 1)^2
};
__device__ __forceinline__ PiolaTerms piolaTerms(const M3& f, float lambda, float mu) {
  PiolaTerms t;
  t.I1 = frob(f, f);
  const float den = t.I1 + 1.0f;
  t.cof = cofactor(f);
  t.J = dot3(f.c0, t.cof.c0);
  t.a = mu * (1.0f - 1.0f / den);
  t.b = lambda * (t.J - 1.0f) - 0.75f * mu;
  t.c1 = 2.0f * mu / (den * den);
  return t;
}
__device__ __forceinline__ M3 piola(const M3& f, const PiolaTerms& t) { return t.a * f + t.b * t.cof; }

// ---- cancellation-resistant energy delta (jgs2-globalization-wgsl.ts:494-559) --
__device__ __forceinline__ float logOnePlus(float v) {
  if (fabsf(v) <= 0.001f) {
    return v * (1.0f + v * (-0.5f + v * (0.3333333333333333f + v * (-0.25f + 0.2f * v))));
  }
  return logf(1.0f + v);
}
__device__ __forceinline__ float detDelta(const M3& i, const M3& d) {
  return dot3(d.c0, cross3(i.c1, i.c2)) + dot3(i.c0, cross3(d.c1, i.c2)) + dot3(i.c0, cross3(i.c1, d.c2)) +
         dot3(d.c0, cross3(d.c1, i.c2)) + dot3(d.c0, cross3(i.c1, d.c2)) + dot3(i.c0, cross3(d.c1, d.c2)) +
         dot3(d.c0, cross3(d.c1, d.c2));
}
// psi(F0 + D) - psi(F0); J0 and I0 = |F0|^2 of the initial pose are passed in.
__device__ __forceinline__ float snhEnergyDelta(const M3& f0, float I0, float J0, const M3& d, float lambda,
                                                float mu, float* Jtrial) {
  const M3 f1 = f0 + d;
  const float id = frob(d, f1 + f0);
  const float dj = detDelta(f0, d);
  const float J1 = mdet(f1);
  *Jtrial = J1;
  const float lr = logOnePlus(id / (I0 + 1.0f));
  return 0.5f * mu * id - 0.75f * mu * dj + 0.5f * lambda * dj * (J1 + J0 - 2.0f) - 0.5f * mu * lr;
}

#ifndef JGS2_LS_RANK1
#define JGS2_LS_RANK1 1
#endif
// snhEnergyDelta for a rank-one step D = d g^T (one vertex of a tet moving):
// <D, 2 F0 + D> = 2 d.(F0 g) + |d|^2 |g|^2 and det(F0 + D) - det(F0) =
// d.(cof(F0) g) exactly (the determinant is affine in a rank-one update), so
// the general trilinear expansion is not needed.  J1 is still det(F0 + D).
__device__ __forceinline__ float snhEnergyDeltaRankOne(const M3& f0, float I0, float J0, float3 d, float3 g,
                                                       float lambda, float mu, float* Jtrial) {
  const float id = 2.0f * dot3(d, mv(f0, g)) + dot3(d, d) * dot3(g, g);
  const float dj = dot3(d, mv(cofactor(f0), g));
  const float J1 = mdet(f0 + outer(d, g));
  *Jtrial = J1;
  const float lr = logOnePlus(id / (I0 + 1.0f));
  return 0.5f * mu * id - 0.75f * mu * dj + 0.5f * lambda * dj * (J1 + J0 - 2.0f) - 0.5f * mu * lr;
}

// ---- globalization solve (jgs2-globalization-wgsl.ts:166-492) -----------------
__device__ __forceinline__ float minSymmetricEigenvalue(const S3& m) {
  const float a00 = m.xx, a11 = m.yy, a22 = m.zz, a01 = m.xy, a02 = m.xz, a12 = m.yz;
  const float off = a01 * a01 + a02 * a02 + a12 * a12;
  if (off == 0.0f) return fminf(a00, fminf(a11, a22));
  const float mean = (a00 + a11 + a22) / 3.0f;
  const float d00 = a00 - mean, d11 = a11 - mean, d22 = a22 - mean;
  const float cs = d00 * d00 + d11 * d11 + d22 * d22 + 2.0f * off;
  const float ss = sqrtf(cs / 6.0f);
  if (!(ss > 0.0f)) return fminf(a00, fminf(a11, a22));
  const float n00 = d00 / ss, n11 = d11 / ss, n22 = d22 / ss, n01 = a01 / ss, n02 = a02 / ss, n12 = a12 / ss;
  const float det = n00 * (n11 * n22 - n12 * n12) - n01 * (n01 * n22 - n12 * n02) + n02 * (n01 * n12 - n11 * n02);
  const float hd = fminf(1.0f, fmaxf(-1.0f, 0.5f * det));
  const float angle = acosf(hd) / 3.0f;
  const float largest = mean + 2.0f * ss * cosf(angle);
  const float smallest = mean + 2.0f * ss * cosf(angle + kTwoPiOverThree);
  const float middle = 3.0f * mean - largest - smallest;
  return fminf(largest, fminf(middle, smallest));
}

__device__ __forceinline__ float scaledLength(float3 v) {
  const float mc = fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z)));
  if (!(mc > 0.0f)) return 0.0f;
  const float3 n = v * (1.0f / mc);
  return mc * sqrtf(dot3(n, n));
}

struct SolveResult {
  float3 direction;
  float gdd, scale, minEig, shift, residual;
  uint32_t status;
};

// Symmetric part of H is what the shader factors (it symmetrises first), so
// the accumulated Hessian is kept symmetric throughout.
__device__ inline SolveResult globalizationSolve(const S3& sym, float3 gradient, float inertia) {
  SolveResult out{f3(0, 0, 0), 0, 0, 0, 0, 0, kNonfinite};
  const bool hf = finiteS(sym.xx) && finiteS(sym.yy) && finiteS(sym.zz) && finiteS(sym.xy) && finiteS(sym.xz) &&
                  finiteS(sym.yz);
  if (!hf || !finiteS(inertia) || !(inertia > 0.0f)) return out;
  const float lad = fmaxf(fabsf(sym.xx), fmaxf(fabsf(sym.yy), fabsf(sym.zz)));
  // frobenius_over_sqrt_three
  float fo3 = 0.0f;
  {
    const float me = fmaxf(fmaxf(fmaxf(fabsf(sym.xx), fabsf(sym.yy)), fabsf(sym.zz)),
                           fmaxf(fmaxf(fabsf(sym.xy), fabsf(sym.xz)), fabsf(sym.yz)));
    if (me > 0.0f) {
      const float a00 = sym.xx / me, a11 = sym.yy / me, a22 = sym.zz / me;
      const float a01 = sym.xy / me, a02 = sym.xz / me, a12 = sym.yz / me;
      const float sq = a00 * a00 + a11 * a11 + a22 * a22 + 2.0f * (a01 * a01 + a02 * a02 + a12 * a12);
      fo3 = me * sqrtf(sq / 3.0f);
    }
  }
  const float scale = fmaxf(inertia, fmaxf(lad, fo3));
  if (!finiteS(scale) || !(scale > 0.0f)) return out;
  const S3 nh = {sym.xx / scale, sym.yy / scale, sym.zz / scale, sym.xy / scale, sym.xz / scale, sym.yz / scale};
  const float minEig = minSymmetricEigenvalue(nh);
  if (!finiteS(minEig)) return out;
  const float shift = fmaxf(0.0f, kRelativeEigenvalueFloor - minEig);
  out.scale = scale;
  out.minEig = minEig;
  out.shift = shift;
  if (shift > kMaxNormalizedShift) { out.status = kShiftLimit; return out; }
  if (!finiteV(gradient)) { out.status = kNonfinite; return out; }
  const float gs = fmaxf(fabsf(gradient.x), fmaxf(fabsf(gradient.y), fabsf(gradient.z)));
  if (!(gs > 0.0f)) { out.status = kZeroGradient; return out; }
  const float m00 = nh.xx + shift, m11 = nh.yy + shift, m22 = nh.zz + shift;
  const float m01 = nh.xy, m02 = nh.xz, m12 = nh.yz;
  const float3 rhs = f3(-gradient.x / scale, -gradient.y / scale, -gradient.z / scale);
  if (!finiteV(rhs)) { out.status = kNonfinite; return out; }
  if (!finiteS(m00) || !(m00 > 0.0f)) { out.status = kCholeskyFailed; return out; }
  const float l00 = sqrtf(m00);
  const float l10 = m01 / l00, l20 = m02 / l00;
  const float p1 = m11 - l10 * l10;
  if (!finiteS(p1) || !(p1 > 0.0f)) { out.status = kCholeskyFailed; return out; }
  const float l11 = sqrtf(p1);
  const float l21 = (m12 - l20 * l10) / l11;
  const float p2 = m22 - l20 * l20 - l21 * l21;
  if (!finiteS(p2) || !(p2 > 0.0f)) { out.status = kCholeskyFailed; return out; }
  const float l22 = sqrtf(p2);
  const float y0 = rhs.x / l00;
  const float y1 = (rhs.y - l10 * y0) / l11;
  const float y2 = (rhs.z - l20 * y0 - l21 * y1) / l22;
  const float x2 = y2 / l22;
  const float x1 = (y1 - l21 * x2) / l11;
  const float x0 = (y0 - l10 * x1 - l20 * x2) / l00;
  const float3 dir = f3(x0, x1, x2);
  if (!finiteV(dir)) { out.status = kCholeskyFailed; return out; }
  const float gdd = dot3(gradient, dir);
  if (!finiteS(gdd)) { out.status = kNonDescent; return out; }
  if (!(gdd < 0.0f)) { out.gdd = gdd; out.status = kNonDescent; return out; }
  const float3 res = f3(m00 * dir.x + m01 * dir.y + m02 * dir.z - rhs.x, m01 * dir.x + m11 * dir.y + m12 * dir.z - rhs.y,
                        m02 * dir.x + m12 * dir.y + m22 * dir.z - rhs.z);
  const float rr = scaledLength(res) / fmaxf(1.0f, scaledLength(rhs));
  if (!finiteS(rr)) { out.gdd = gdd; out.status = kCholeskyFailed; return out; }
  out.direction = dir;
  out.gdd = gdd;
  out.residual = rr;
  out.status = kAccepted;
  return out;
}

// ---- polar rotation (jgs2-shader.ts:924-978) ---------------------------------
__device__ __forceinline__ float3 safeNormalize(float3 v, float3 fallback, float eps) {
  const float sq = dot3(v, v);
  if (sq > eps * eps && sq < 1.0e30f) return v * rsqrtf(sq);
  return fallback;
}
__device__ __forceinline__ float3 perpendicularTo(float3 axis, float eps) {
  const float3 c = fabsf(axis.x) > 0.8f ? f3(0, 1, 0) : f3(1, 0, 0);
  return safeNormalize(cross3(axis, c), f3(0, 0, 1), eps);
}
__device__ __forceinline__ M3 orthonormalize(const M3& m, float eps) {
  const float3 c0 = safeNormalize(m.c0, f3(1, 0, 0), eps);
  const float3 c1c = m.c1 - c0 * dot3(c0, m.c1);
  float3 c1 = safeNormalize(c1c, perpendicularTo(c0, eps), eps);
  float3 c2 = safeNormalize(cross3(c0, c1), f3(0, 0, 1), eps);
  if (dot3(c2, m.c2) < 0.0f) { c1 = -c1; c2 = -c2; }
  c1 = safeNormalize(cross3(c2, c0), perpendicularTo(c0, eps), eps);
  return {c0, c1, c2};
}
__device__ __forceinline__ M3 polarRotation(M3 r, float eps) {
#pragma unroll 1
  for (int it = 0; it < 7; ++it) {
    const float d = mdet(r);
    const float mag = fabsf(d);
    if (!(mag > eps) || mag > 1.0e20f) break;
    const float recip = 1.0f / d;
    const M3 it2 = recip * cofactor(r);
    r = 0.5f * (r + it2);
  }
  return orthonormalize(r, eps);
}

}  // namespace jgs2
