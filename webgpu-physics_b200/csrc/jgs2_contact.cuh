// IPC contact on the device: closest features of vertex-triangle and
// edge-edge candidates, the log barrier B(d) = -(d - dHat)^2 log(d / dHat)
// with its PSD normal block, lagged friction with IPC's C1 smoothing, and
// the Lipschitz safe-step cap (src/simulation/gpu/ipc-contact-wgsl.ts:19-472
// and the contact helpers of src/simulation/gpu/jgs2-shader.ts:233-874).
//
// Candidate state (7 float4 per candidate): source contact (normal,
// distance; distance -1 when invalid) and its closest-feature weights, the
// same for the target pose, the lagged normal force (normal, magnitude) and
// its weights, and a scratch record.  Contact weights satisfy
// sum_i w_i x_i = point_a - point_b.
#pragma once

#include "jgs2_device.cuh"

namespace jgs2 {

constexpr float kIpcLengthSquaredFloor = 1.0e-20f;
constexpr float kIpcParallelRelativeEpsilon = 1.0e-6f;
constexpr uint32_t kIpcVertexTriangle = 0u, kIpcEdgeEdge = 1u;

enum ContactSlot : int {
  kContactSource = 0, kContactSourceWeights = 1, kContactTarget = 2, kContactTargetWeights = 3,
  kContactLagged = 4, kContactLaggedWeights = 5, kContactScratch = 6, kContactStateWords = 7,
};

struct ContactData {
  float distance;
  float3 normal;
  float4 weights;
  bool valid;
};

__device__ __forceinline__ bool finite4f(float4 v) { return finiteS(v.x) && finiteS(v.y) && finiteS(v.z) && finiteS(v.w); }

__device__ __forceinline__ float3 ipcSafeUnit(float3 v, float3 fallback) {
  const float l2 = dot3(v, v);
  if (finiteS(l2) && l2 > kIpcLengthSquaredFloor) return v * rsqrtf(l2);
  const float f2 = dot3(fallback, fallback);
  if (finiteS(f2) && f2 > kIpcLengthSquaredFloor) return fallback * rsqrtf(f2);
  return f3(1, 0, 0);
}

__device__ __forceinline__ float3 ipcOrthogonalUnit(float3 d) {
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  float3 axis = f3(1, 0, 0);
  if (ay <= ax && ay <= az) axis = f3(0, 1, 0);
  else if (az <= ax && az <= ay) axis = f3(0, 0, 1);
  return ipcSafeUnit(cross3(d, axis), f3(1, 0, 0));
}

__device__ __forceinline__ ContactData ipcInvalid() { return {0.0f, f3(1, 0, 0), make_float4(0, 0, 0, 0), false}; }

__device__ __forceinline__ ContactData ipcMake(float3 pa, float3 pb, float4 w, float3 fallback) {
  if (!finiteV(pa) || !finiteV(pb) || !finite4f(w)) return ipcInvalid();
  const float3 gap = pa - pb;
  const float sq = dot3(gap, gap);
  if (!finiteS(sq) || sq < 0.0f) return ipcInvalid();
  return {sqrtf(sq), ipcSafeUnit(gap, fallback), w, true};
}

__device__ __forceinline__ float clamp01f(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// ---- FP64 closest features of near-degenerate pairs -------------------------
// The f32 closest-feature arithmetic below loses its relative accuracy on two
// kinds of pair: near-degenerate geometry (a sliver triangle, near-parallel
// edges: the 2x2 barycentric system is ill-conditioned, sin^2 of the angle
// below kIpcWideAngle) and near-touching features (the squared distance below
// kIpcWideTouch of the squared feature extent, where the difference of two
// f32 closest points cancels).  Those pairs are recomputed in double from the
// same f32 coordinates, with the same branch structure, and the distance,
// normal and weights are rounded to f32 once.  All other pairs keep the f32
// result.
constexpr float kIpcWideAngle = 1.0e-3f;
constexpr float kIpcWideTouch = 9.5367431640625e-07f;  // 2^-20

struct WideContact {
  double distance;
  double3 normal;
  double4 weights;
  bool valid;
};
__device__ __forceinline__ double3 dd3(float3 v) { return make_double3(v.x, v.y, v.z); }
__device__ __forceinline__ double3 dadd(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 dsub(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 dscale(double s, double3 a) { return make_double3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double ddot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 dcross(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ bool dfinite(double v) { return v == v && fabs(v) <= 1.0e300; }
__device__ __forceinline__ bool dfinite3(double3 v) { return dfinite(v.x) && dfinite(v.y) && dfinite(v.z); }
__device__ __forceinline__ double dclamp01(double v) { return fmin(fmax(v, 0.0), 1.0); }
__device__ __forceinline__ double3 dSafeUnit(double3 v, double3 fallback) {
  const double l2 = ddot(v, v);
  if (dfinite(l2) && l2 > 1.0e-40) return dscale(1.0 / sqrt(l2), v);
  const double f2 = ddot(fallback, fallback);
  if (dfinite(f2) && f2 > 1.0e-40) return dscale(1.0 / sqrt(f2), fallback);
  return make_double3(1, 0, 0);
}
__device__ __forceinline__ double3 dOrthogonalUnit(double3 d) {
  const double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
  double3 axis = make_double3(1, 0, 0);
  if (ay <= ax && ay <= az) axis = make_double3(0, 1, 0);
  else if (az <= ax && az <= ay) axis = make_double3(0, 0, 1);
  return dSafeUnit(dcross(d, axis), make_double3(1, 0, 0));
}
__device__ __forceinline__ WideContact dMake(double3 pa, double3 pb, double4 w, double3 fallback) {
  const double3 gap = dsub(pa, pb);
  const double sq = ddot(gap, gap);
  if (!dfinite3(pa) || !dfinite3(pb) || !dfinite(sq)) return {0.0, make_double3(1, 0, 0), make_double4(0, 0, 0, 0), false};
  return {sqrt(sq), dSafeUnit(gap, fallback), w, true};
}
__device__ __forceinline__ void dClosestOnSegment(double3 q, double3 s, double3 e, double3* point, double* parameter,
                                                  double* squared) {
  const double3 edge = dsub(e, s);
  const double l2 = ddot(edge, edge);
  double t = 0.0;
  if (dfinite(l2) && l2 > 1.0e-20) t = dclamp01(ddot(dsub(q, s), edge) / l2);
  *point = dadd(s, dscale(t, edge));
  const double3 d = dsub(q, *point);
  *parameter = t;
  *squared = ddot(d, d);
}
// The FP64 run of jgs2_ipc_point_triangle_contact (ipc-contact-wgsl.ts:145-223).
__device__ __forceinline__ WideContact wideIpcPointTriangle(float3 pf, float3 t0f, float3 t1f, float3 t2f) {
  const double3 p = dd3(pf), t0 = dd3(t0f), t1 = dd3(t1f), t2 = dd3(t2f);
  const double3 e01 = dsub(t1, t0), e02 = dsub(t2, t0), e12 = dsub(t2, t1);
  const double s01 = ddot(e01, e01), s02 = ddot(e02, e02), s12 = ddot(e12, e12);
  const double largest = fmax(s01, fmax(s02, s12));
  const double3 an = dcross(e01, e02);
  const double a2 = ddot(an, an);
  const double threshold = fmax(1.0e-40, 1.0e-6 * largest * largest);
  double3 longest = e01;
  if (s02 > s01 && s02 >= s12) longest = e02;
  else if (s12 > s01 && s12 > s02) longest = e12;
  const double3 fallback = dSafeUnit(an, dOrthogonalUnit(longest));
  if (dfinite(a2) && a2 > threshold) {
    const double d01 = ddot(e01, e02);
    const double3 po = dsub(p, t0);
    const double d20 = ddot(po, e01), d21 = ddot(po, e02);
    const double den = s01 * s02 - d01 * d01;
    const double b1 = (s02 * d20 - d01 * d21) / den;
    const double b2 = (s01 * d21 - d01 * d20) / den;
    const double b0 = 1.0 - b1 - b2;
    if (b0 >= 0.0 && b1 >= 0.0 && b2 >= 0.0)
      return dMake(p, dadd(dadd(dscale(b0, t0), dscale(b1, t1)), dscale(b2, t2)), make_double4(1.0, -b0, -b1, -b2),
                   fallback);
  }
  double3 q01, q12, q20;
  double u01, u12, u20, sq01, sq12, sq20;
  dClosestOnSegment(p, t0, t1, &q01, &u01, &sq01);
  dClosestOnSegment(p, t1, t2, &q12, &u12, &sq12);
  dClosestOnSegment(p, t2, t0, &q20, &u20, &sq20);
  double3 best = q01, bary = make_double3(1.0 - u01, u01, 0.0);
  double bestSq = sq01;
  if (sq12 < bestSq) { best = q12; bestSq = sq12; bary = make_double3(0.0, 1.0 - u12, u12); }
  if (sq20 < bestSq) { best = q20; bary = make_double3(u20, 0.0, 1.0 - u20); }
  return dMake(p, best, make_double4(1.0, -bary.x, -bary.y, -bary.z), fallback);
}
// The FP64 run of jgs2_ipc_edge_edge_contact (ipc-contact-wgsl.ts:227-300).
__device__ __forceinline__ WideContact wideIpcEdgeEdge(float3 a0f, float3 a1f, float3 b0f, float3 b1f) {
  const double3 a0 = dd3(a0f), a1 = dd3(a1f), b0 = dd3(b0f), b1 = dd3(b1f);
  const double3 da = dsub(a1, a0), db = dsub(b1, b0), off = dsub(a0, b0);
  const double la = ddot(da, da), lb = ddot(db, db);
  const double degenerate = fmax(1.0e-20, 1.0e-6 * fmax(la, lb));
  const bool aDeg = !(la > degenerate), bDeg = !(lb > degenerate);
  double pa = 0.0, pb = 0.0;
  if (aDeg && !bDeg) {
    pb = dclamp01(ddot(db, off) / lb);
  } else if (!aDeg) {
    const double projA = ddot(da, off);
    if (bDeg) {
      pa = dclamp01(-projA / la);
    } else {
      const double coupling = ddot(da, db);
      const double projB = ddot(db, off);
      const double den = la * lb - coupling * coupling;
      if (den > 1.0e-6 * la * lb) pa = dclamp01((coupling * projB - projA * lb) / den);
      const double pbu = (coupling * pa + projB) / lb;
      if (pbu < 0.0) {
        pb = 0.0;
        pa = dclamp01(-projA / la);
      } else if (pbu > 1.0) {
        pb = 1.0;
        pa = dclamp01((coupling - projA) / la);
      } else {
        pb = pbu;
      }
    }
  }
  const double3 longest = lb > la ? db : da;
  const double3 fallback = dSafeUnit(dcross(da, db), dOrthogonalUnit(longest));
  return dMake(dadd(a0, dscale(pa, da)), dadd(b0, dscale(pb, db)), make_double4(1.0 - pa, pa, -(1.0 - pb), -pb),
               fallback);
}

struct SegmentPoint {
  float3 point;
  float parameter, squared;
};

__device__ __forceinline__ SegmentPoint ipcClosestOnSegment(float3 q, float3 s, float3 e) {
  const float3 edge = e - s;
  const float l2 = dot3(edge, edge);
  float t = 0.0f;
  if (finiteS(l2) && l2 > kIpcLengthSquaredFloor) t = clamp01f(dot3(q - s, edge) / l2);
  const float3 p = s + t * edge;
  const float3 d = q - p;
  return {p, t, dot3(d, d)};
}

__device__ __forceinline__ ContactData narrowContact(const WideContact& k) {
  if (!k.valid) return ipcInvalid();
  const float3 n = f3(float(k.normal.x), float(k.normal.y), float(k.normal.z));
  const float4 w = make_float4(float(k.weights.x), float(k.weights.y), float(k.weights.z), float(k.weights.w));
  const float d = float(k.distance);
  if (!finiteS(d) || !finiteV(n) || !finite4f(w)) return ipcInvalid();
  return {d, n, w, true};
}

// f32 point-triangle contact of jgs2_ipc_point_triangle_contact
// (ipc-contact-wgsl.ts:145-223); near-degenerate pairs (sliver triangle or
// near-touching point) take the FP64 run above (*wide set when they do).
__device__ __forceinline__ ContactData ipcPointTriangle(float3 p, float3 t0, float3 t1, float3 t2,
                                                        bool* wide = nullptr) {
  const float3 e01 = t1 - t0, e02 = t2 - t0, e12 = t2 - t1;
  const float s01 = dot3(e01, e01), s02 = dot3(e02, e02), s12 = dot3(e12, e12);
  const float largest = fmaxf(s01, fmaxf(s02, s12));
  const float3 an = cross3(e01, e02);
  const float a2 = dot3(an, an);
  const float threshold = fmaxf(kIpcLengthSquaredFloor * kIpcLengthSquaredFloor,
                                kIpcParallelRelativeEpsilon * largest * largest);
  float3 longest = e01;
  if (s02 > s01 && s02 >= s12) longest = e02;
  else if (s12 > s01 && s12 > s02) longest = e12;
  const float3 fallback = ipcSafeUnit(an, ipcOrthogonalUnit(longest));
  ContactData r;
  bool done = false;
  if (finiteS(a2) && a2 > threshold) {
    const float d01 = dot3(e01, e02);
    const float3 po = p - t0;
    const float d20 = dot3(po, e01), d21 = dot3(po, e02);
    const float den = s01 * s02 - d01 * d01;
    const float b1 = (s02 * d20 - d01 * d21) / den;
    const float b2 = (s01 * d21 - d01 * d20) / den;
    const float b0 = 1.0f - b1 - b2;
    if (b0 >= 0.0f && b1 >= 0.0f && b2 >= 0.0f) {
      r = ipcMake(p, b0 * t0 + b1 * t1 + b2 * t2, make_float4(1.0f, -b0, -b1, -b2), fallback);
      done = true;
    }
  }
  if (!done) {
    const SegmentPoint c01 = ipcClosestOnSegment(p, t0, t1);
    const SegmentPoint c12 = ipcClosestOnSegment(p, t1, t2);
    const SegmentPoint c20 = ipcClosestOnSegment(p, t2, t0);
    SegmentPoint best = c01;
    float3 bary = f3(1.0f - c01.parameter, c01.parameter, 0.0f);
    if (c12.squared < best.squared) { best = c12; bary = f3(0.0f, 1.0f - c12.parameter, c12.parameter); }
    if (c20.squared < best.squared) { best = c20; bary = f3(c20.parameter, 0.0f, 1.0f - c20.parameter); }
    r = ipcMake(p, best.point, make_float4(1.0f, -bary.x, -bary.y, -bary.z), fallback);
  }
  // Sliver triangle (a2 = s01 s02 sin^2) or near-touching point: FP64.
  const bool sliver = !(a2 > kIpcWideAngle * s01 * s02);
  const bool touching = r.valid && r.distance * r.distance < kIpcWideTouch * largest;
  const bool useWide = finiteS(largest) && (sliver || touching);
  if (wide) *wide = useWide;
  return useWide ? narrowContact(wideIpcPointTriangle(p, t0, t1, t2)) : r;
}

// f32 edge-edge contact of jgs2_ipc_edge_edge_contact
// (ipc-contact-wgsl.ts:227-300); near-degenerate pairs (near-parallel edges
// or near-touching edges) take the FP64 run above (*wide set when they do).
__device__ __forceinline__ ContactData ipcEdgeEdge(float3 a0, float3 a1, float3 b0, float3 b1, bool* wide = nullptr) {
  const float3 da = a1 - a0, db = b1 - b0, off = a0 - b0;
  const float la = dot3(da, da), lb = dot3(db, db);
  const float degenerate = fmaxf(kIpcLengthSquaredFloor, kIpcParallelRelativeEpsilon * fmaxf(la, lb));
  const bool aDeg = !(la > degenerate), bDeg = !(lb > degenerate);
  const float crossDen = la * lb - dot3(da, db) * dot3(da, db);
  float pa = 0.0f, pb = 0.0f;
  if (aDeg && !bDeg) {
    pb = clamp01f(dot3(db, off) / lb);
  } else if (!aDeg) {
    const float projA = dot3(da, off);
    if (bDeg) {
      pa = clamp01f(-projA / la);
    } else {
      const float coupling = dot3(da, db);
      const float projB = dot3(db, off);
      const float den = la * lb - coupling * coupling;
      if (den > kIpcParallelRelativeEpsilon * la * lb) pa = clamp01f((coupling * projB - projA * lb) / den);
      const float pbu = (coupling * pa + projB) / lb;
      if (pbu < 0.0f) {
        pb = 0.0f;
        pa = clamp01f(-projA / la);
      } else if (pbu > 1.0f) {
        pb = 1.0f;
        pa = clamp01f((coupling - projA) / la);
      } else {
        pb = pbu;
      }
    }
  }
  const float3 longest = lb > la ? db : da;
  const float3 fallback = ipcSafeUnit(cross3(da, db), ipcOrthogonalUnit(longest));
  const ContactData r = ipcMake(a0 + pa * da, b0 + pb * db, make_float4(1.0f - pa, pa, -(1.0f - pb), -pb), fallback);
  // Near-parallel edges (crossDen = la lb sin^2) or near-touching edges: FP64.
  const bool parallel = !(crossDen > kIpcWideAngle * la * lb);
  const bool touching = r.valid && r.distance * r.distance < kIpcWideTouch * fmaxf(la, lb);
  const bool useWide = finiteS(la) && finiteS(lb) && (parallel || touching);
  if (wide) *wide = useWide;
  return useWide ? narrowContact(wideIpcEdgeEdge(a0, a1, b0, b1)) : r;
}

__device__ __forceinline__ bool ipcBarrierActive(float d, float dHat) {
  return finiteS(d) && finiteS(dHat) && d > 0.0f && d < dHat;
}
__device__ __forceinline__ float ipcBarrier(float d, float dHat) {
  if (!ipcBarrierActive(d, dHat)) return 0.0f;
  const float o = d - dHat;
  return -(o * o) * (logf(d) - logf(dHat));
}
__device__ __forceinline__ float ipcBarrier1(float d, float dHat) {
  if (!ipcBarrierActive(d, dHat)) return 0.0f;
  const float o = d - dHat;
  return -2.0f * o * (logf(d) - logf(dHat)) - o * o / d;
}
__device__ __forceinline__ float ipcBarrier2(float d, float dHat) {
  if (!ipcBarrierActive(d, dHat)) return 0.0f;
  const float o = d - dHat;
  return -2.0f * (logf(d) - logf(dHat)) - 4.0f * o / d + o * o / (d * d);
}
__device__ __forceinline__ float ipcNormalGradientScalar(float w, float kappa, float b1) {
  if (!finiteS(w) || !finiteS(kappa) || !finiteS(b1) || kappa < 0.0f) return 0.0f;
  return w * kappa * b1;
}
__device__ __forceinline__ float ipcPsdScalar(float w, float kappa, float b2) {
  if (!finiteS(w) || !finiteS(kappa) || !finiteS(b2) || kappa <= 0.0f || w == 0.0f || b2 <= 0.0f) return 0.0f;
  const float s = kappa * w * w * b2;
  return finiteS(s) ? s : kF32Max;
}
// ipcSafeStepCap (ipc-contact-wgsl.ts:402-422): the Lipschitz bound
// safety (src - dMin) / L, formed in FP64 (the gap src - dMin of two f32
// values is exact there, however close they are) and rounded once.
__device__ __forceinline__ float ipcSafeStepCap(float src, float dMin, float L, float safety) {
  if (!finiteS(src) || !finiteS(dMin) || !finiteS(L) || !finiteS(safety) || dMin < 0.0f || src <= dMin || L < 0.0f)
    return 0.0f;
  if (L == 0.0f) return 1.0f;
  const double cap = double(clamp01f(safety)) * (double(src) - double(dMin)) / double(L);
  return clamp01f(float(fmin(fmax(cap, 0.0), 1.0)));
}
__device__ __forceinline__ float ipcFrictionF1(float s, float eps) {
  const float n = fmaxf(s, 0.0f);
  if (!(eps > 0.0f) || n >= eps) return n > 0.0f ? 1.0f : 0.0f;
  const float u = n / eps;
  return u * (2.0f - u);
}
__device__ __forceinline__ float ipcFrictionDissipation(float slip, float eps, float mu, float lambda) {
  if (!finiteS(slip) || !finiteS(eps) || !finiteS(mu) || !finiteS(lambda)) return 0.0f;
  const float n = fmaxf(slip, 0.0f);
  const float scale = fmaxf(mu, 0.0f) * fmaxf(lambda, 0.0f);
  if (!(eps > 0.0f)) return scale * n;
  if (n < eps) {
    const float u = n / eps;
    return scale * eps * u * u * (1.0f - u / 3.0f);
  }
  return scale * (n - eps / 3.0f);
}

__device__ __forceinline__ float3 fmin3(float3 a, float3 b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ float3 fmax3(float3 a, float3 b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

// ipcContactFromPositions (jgs2-shader.ts:520-592): a separated contact at
// the AABB distance lower bound when that bound reaches the threshold.
__device__ __forceinline__ ContactData ipcContactFromPositions(uint32_t type, float3 p0, float3 p1, float3 p2,
                                                               float3 p3, float threshold) {
  float3 gap;
  if (type == kIpcVertexTriangle) {
    const float3 lo = fmin3(p1, fmin3(p2, p3)), hi = fmax3(p1, fmax3(p2, p3));
    gap = fmax3(fmax3(lo - p0, p0 - hi), f3(0, 0, 0));
  } else {
    gap = fmax3(fmax3(fmin3(p2, p3) - fmax3(p0, p1), fmin3(p0, p1) - fmax3(p2, p3)), f3(0, 0, 0));
  }
  const float lb = sqrtf(dot3(gap, gap));
  if (finiteS(lb) && lb >= threshold) return {lb, f3(1, 0, 0), make_float4(0, 0, 0, 0), true};
  if (type == kIpcVertexTriangle) return ipcPointTriangle(p0, p1, p2, p3);
  return ipcEdgeEdge(p0, p1, p2, p3);
}

// ipcCachedContact (jgs2-shader.ts:408-437).
__device__ __forceinline__ ContactData ipcCached(float4 nd, float4 w) {
  const bool valid = nd.w >= 0.0f && finite4f(nd) && finite4f(w);
  return {valid ? nd.w : 0.0f, valid ? f3(nd.x, nd.y, nd.z) : f3(1, 0, 0), valid ? w : make_float4(0, 0, 0, 0),
          valid};
}

// ipcStoreCachedContact (jgs2-shader.ts:378-406).
__device__ __forceinline__ void ipcStoreCached(float4* state, int slot, const ContactData& k) {
  const bool valid = k.valid && finiteS(k.distance) && k.distance >= 0.0f && finiteV(k.normal) && finite4f(k.weights);
  state[slot] = valid ? make_float4(k.normal.x, k.normal.y, k.normal.z, k.distance) : make_float4(0, 0, 0, -1.0f);
  state[slot + 1] = valid ? k.weights : make_float4(0, 0, 0, 0);
}

__device__ __forceinline__ float ipcWeightFor(uint4 q, float4 w, uint32_t v) {
  float r = 0.0f;
  if (q.x == v) r += w.x;
  if (q.y == v) r += w.y;
  if (q.z == v) r += w.z;
  if (q.w == v) r += w.w;
  return r;
}

}  // namespace jgs2
