// Triangle cloth on the device: St. Venant-Kirchhoff membrane triangles in
// plane stress and quadratic dihedral bending hinges
// (src/simulation/gpu/jgs2-shader.ts:1225-1844, restating
// src/simulation/cpu/cloth.ts:107-391).
//
// Layout: a triangle is two float4, (i0, i1, i2 as uint bits, rest area) and
// the row-major inverse rest basis; a hinge is two float4, (i0..i3 as uint
// bits) and (rest angle, rest edge length, 0, 0).  Indices are global
// (scene offsets applied).  Each vertex owns a range of `incidence` entries
// element * 4 + local slot, triangles first, then hinges.
//
// One algebraic rewrite, exact in real arithmetic: the membrane's diagonal
// Hessian block (clothMembraneLocalHessian, :1610-1660, built column by
// column and symmetrised) is formed in closed form,
//   A t [ (g^T S g) I + (mu + lambda) u u^T + mu |g|^2 (f0 f0^T + f1 f1^T) ],
// with g the vertex's 2D shape gradient, S the second Piola stress, f0 / f1
// the columns of the 3x2 deformation gradient and u = F g; it is symmetric
// as formed.  The dihedral differential is evaluated for the three
// coordinates of one vertex slot only, with the per-coordinate formula of
// the reference.
#pragma once

#include "jgs2_device.cuh"

namespace jgs2 {

struct ClothMaterial {
  float lambda;     // plane-stress lambda E nu / (1 - nu^2)
  float mu;         // E / (2 (1 + nu))
  float thickness;
  float bending;    // bending stiffness k
};

struct ClothTri {
  uint32_t i0, i1, i2;
  float area;
  float4 inv;  // row-major inverse rest basis (x y / z w)
};

__device__ __forceinline__ ClothTri loadClothTri(const float4* __restrict__ tris, uint32_t c) {
  const float4 a = __ldg(&tris[2ull * c]);
  const float4 inv = __ldg(&tris[2ull * c + 1]);
  return {__float_as_uint(a.x), __float_as_uint(a.y), __float_as_uint(a.z), a.w, inv};
}

// clothTriangleShapeGradient (jgs2-shader.ts:1536-1547).
__device__ __forceinline__ float2 clothShapeGradient(const float4& inv, uint32_t slot) {
  if (slot == 1u) return make_float2(inv.x, inv.y);
  if (slot == 2u) return make_float2(inv.z, inv.w);
  return make_float2(-inv.x - inv.z, -inv.y - inv.w);
}

struct Membrane {
  float energy;
  float3 f0, f1;     // deformation gradient columns
  float s0, s1, s2;  // second Piola stress (00, 01, 11)
};

// clothMembraneEvaluationAt (jgs2-shader.ts:1549-1608): Green strain of the
// 3x2 deformation gradient, S = 2 mu E + lambda tr(E) I, energy
// A t (mu |E|^2 + lambda / 2 tr(E)^2).
__device__ __forceinline__ Membrane clothMembrane(const ClothTri& t, float3 x0, float3 x1, float3 x2,
                                                  const ClothMaterial& m) {
  const float3 e01 = x1 - x0, e02 = x2 - x0;
  Membrane r;
  r.f0 = e01 * t.inv.x + e02 * t.inv.z;
  r.f1 = e01 * t.inv.y + e02 * t.inv.w;
  const float e00 = 0.5f * (dot3(r.f0, r.f0) - 1.0f);
  const float e01s = 0.5f * dot3(r.f0, r.f1);
  const float e11 = 0.5f * (dot3(r.f1, r.f1) - 1.0f);
  const float tr = e00 + e11;
  r.s0 = 2.0f * m.mu * e00 + m.lambda * tr;
  r.s1 = 2.0f * m.mu * e01s;
  r.s2 = 2.0f * m.mu * e11 + m.lambda * tr;
  const float density = m.mu * (e00 * e00 + 2.0f * e01s * e01s + e11 * e11) + 0.5f * m.lambda * tr * tr;
  r.energy = (t.area * m.thickness) * density;
  return r;
}

// Energy only (the line search and the gate).
__device__ __forceinline__ float clothMembraneEnergy(const ClothTri& t, float3 x0, float3 x1, float3 x2,
                                                     const ClothMaterial& m) {
  return clothMembrane(t, x0, x1, x2, m).energy;
}

// Gradient of the membrane energy at the vertex in `slot`.
__device__ __forceinline__ float3 clothMembraneGradient(const ClothTri& t, const Membrane& e, uint32_t slot,
                                                        const ClothMaterial& m) {
  const float2 g = clothShapeGradient(t.inv, slot);
  const float3 p0 = e.f0 * e.s0 + e.f1 * e.s1;
  const float3 p1 = e.f0 * e.s1 + e.f1 * e.s2;
  return (t.area * m.thickness) * (p0 * g.x + p1 * g.y);
}

// Exact diagonal Hessian block of the membrane at the vertex in `slot`.
__device__ __forceinline__ void clothMembraneHessian(S3& h, const ClothTri& t, const Membrane& e, uint32_t slot,
                                                     const ClothMaterial& m) {
  const float2 g = clothShapeGradient(t.inv, slot);
  const float aw = t.area * m.thickness;
  const float gsg = g.x * g.x * e.s0 + 2.0f * g.x * g.y * e.s1 + g.y * g.y * e.s2;
  const float gg = g.x * g.x + g.y * g.y;
  const float3 u = e.f0 * g.x + e.f1 * g.y;
  S3 blk = szero();
  saddDiag(blk, gsg);
  saddOuter(blk, m.mu + m.lambda, u);
  saddOuter(blk, m.mu * gg, e.f0);
  saddOuter(blk, m.mu * gg, e.f1);
  saddScaled(h, aw, blk);
}

// Signed relative area stretch |n| / 2A of a triangle (jgs2-shader.ts:2067-2116).
__device__ __forceinline__ float3 clothRawNormal(float3 x0, float3 x1, float3 x2) {
  return cross3(x1 - x0, x2 - x0);
}

__device__ __forceinline__ float length3(float3 v) { return sqrtf(dot3(v, v)); }

struct DihedralFrame {
  float3 edge, to2, rev, to3;
  float3 t, n0, n1, nc;
  float edgeLength, nl0, nl1;
  float sine, cosine, den;
  bool valid;
};

// Geometry of clothDihedralEvaluationAt (jgs2-shader.ts:1702-1760) for the
// oriented hinge (0, 1, 2) / (1, 0, 3).
__device__ __forceinline__ DihedralFrame clothDihedralFrame(float3 p0, float3 p1, float3 p2, float3 p3) {
  DihedralFrame f;
  f.edge = p1 - p0;
  f.edgeLength = length3(f.edge);
  f.to2 = p2 - p0;
  f.rev = -f.edge;
  f.to3 = p3 - p1;
  const float3 n0r = cross3(f.edge, f.to2), n1r = cross3(f.rev, f.to3);
  f.nl0 = length3(n0r);
  f.nl1 = length3(n1r);
  const float es0 = fmaxf(f.edgeLength, fmaxf(length3(f.to2), length3(f.to2 - f.edge)));
  const float es1 = fmaxf(f.edgeLength, fmaxf(length3(f.to3), length3(f.to3 - f.rev)));
  f.valid = finiteS(f.edgeLength) && f.edgeLength > 0.0f && finiteS(f.nl0) && finiteS(f.nl1) &&
            f.nl0 > 1.0e-12f * es0 * es0 && f.nl1 > 1.0e-12f * es1 * es1;
  if (!f.valid) return f;
  f.t = f.edge * (1.0f / f.edgeLength);
  f.n0 = n0r * (1.0f / f.nl0);
  f.n1 = n1r * (1.0f / f.nl1);
  f.nc = cross3(f.n0, f.n1);
  f.sine = dot3(f.t, f.nc);
  f.cosine = dot3(f.n0, f.n1);
  f.den = f.sine * f.sine + f.cosine * f.cosine;
  f.valid = finiteS(f.den) && f.den > 0.0f;
  return f;
}

__device__ __forceinline__ float3 clothNormalizedDifferential(float3 unit, float len, float3 d) {
  return (d - unit * dot3(unit, d)) * (1.0f / len);
}

// d theta / d x_slot: the reference's per-coordinate differential
// (jgs2-shader.ts:1761-1798) for the three coordinates of one slot.
__device__ __forceinline__ float3 clothDihedralGradient(const DihedralFrame& f, uint32_t slot) {
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float3 e = f3(k == 0 ? 1.f : 0.f, k == 1 ? 1.f : 0.f, k == 2 ? 1.f : 0.f);
    const float3 z = f3(0, 0, 0);
    const float3 dEdge = slot == 1u ? e : (slot == 0u ? -e : z);
    const float3 dTo2 = slot == 2u ? e : (slot == 0u ? -e : z);
    const float3 dTo3 = slot == 3u ? e : (slot == 1u ? -e : z);
    const float3 dt = clothNormalizedDifferential(f.t, f.edgeLength, dEdge);
    const float3 dn0r = cross3(dEdge, f.to2) + cross3(f.edge, dTo2);
    const float3 dn1r = cross3(-dEdge, f.to3) + cross3(f.rev, dTo3);
    const float3 dn0 = clothNormalizedDifferential(f.n0, f.nl0, dn0r);
    const float3 dn1 = clothNormalizedDifferential(f.n1, f.nl1, dn1r);
    const float dcos = dot3(dn0, f.n1) + dot3(f.n0, dn1);
    const float dsin = dot3(dt, f.nc) + dot3(f.t, cross3(dn0, f.n1) + cross3(f.n0, dn1));
    r[k] = (f.cosine * dsin - f.sine * dcos) / f.den;
  }
  return f3(r[0], r[1], r[2]);
}

// clothWrappedAngleDifference (jgs2-shader.ts:1815-1818).
__device__ __forceinline__ float clothWrappedAngle(float angle, float reference) {
  const float d = angle - reference;
  return atan2f(sinf(d), cosf(d));
}

// clothBendingEnergyAt (jgs2-shader.ts:1820-1836): k L0 / 2 wrap(theta - theta0)^2,
// kF32Max for a degenerate hinge.
__device__ __forceinline__ float clothBendingEnergy(float3 p0, float3 p1, float3 p2, float3 p3, float4 rest,
                                                    float bending) {
  const DihedralFrame f = clothDihedralFrame(p0, p1, p2, p3);
  if (!f.valid) return kF32Max;
  const float angle = atan2f(f.sine, f.cosine);
  if (!finiteS(angle)) return kF32Max;
  const float diff = clothWrappedAngle(angle, rest.x);
  const float ws = bending * rest.y;
  return 0.5f * ws * diff * diff;
}

__device__ __forceinline__ uint4 hingeIndices(const float4* __restrict__ hinges, uint32_t h) {
  const float4 a = __ldg(&hinges[2ull * h]);
  return make_uint4(__float_as_uint(a.x), __float_as_uint(a.y), __float_as_uint(a.z), __float_as_uint(a.w));
}

// Membrane and bending gradient of vertex v at pose x and, with `hess`, the
// membrane diagonal blocks plus the Gauss-Newton bending blocks
// k L0 (dtheta/dx)(dtheta/dx)^T: the cloth loops of jgs2Solve
// (jgs2-shader.ts:3113-3186).  Entries [first, first + count) step `stride`
// of the vertex's incidence range (lane-split gathers pass their lane).
// A position read of the cloth gathers; kCoherent reads with a weak load that
// fences order (see the solve kernel's coherent loads).
template <bool kCoherent>
__device__ __forceinline__ float4 clothPos(const float4* x, uint32_t i) {
  if constexpr (kCoherent) return __ldca(x + i);
  else return x[i];
}

template <bool kHessian, bool kCoherent = false, class G>
__device__ __forceinline__ void clothLocalSystem(const float4* __restrict__ tris, const float4* __restrict__ hinges,
                                                 const uint32_t* __restrict__ incidence, const uint4& range,
                                                 const float4* __restrict__ x, const ClothMaterial& m,
                                                 uint32_t first, uint32_t stride, G& grad, S3& hess) {
  for (uint32_t a = first; a < range.y; a += stride) {
    const uint32_t entry = __ldg(&incidence[range.x + a]);
    const uint32_t slot = entry & 3u;
    const ClothTri t = loadClothTri(tris, entry >> 2);
    const Membrane e = clothMembrane(t, xyz(clothPos<kCoherent>(x, t.i0)), xyz(clothPos<kCoherent>(x, t.i1)), xyz(clothPos<kCoherent>(x, t.i2)), m);
    gadd(grad, clothMembraneGradient(t, e, slot, m));
    if (kHessian) clothMembraneHessian(hess, t, e, slot, m);
  }
  for (uint32_t a = first; a < range.w; a += stride) {
    const uint32_t entry = __ldg(&incidence[range.z + a]);
    const uint32_t slot = entry & 3u;
    const uint32_t h = entry >> 2;
    const uint4 q = hingeIndices(hinges, h);
    const DihedralFrame f = clothDihedralFrame(xyz(clothPos<kCoherent>(x, q.x)), xyz(clothPos<kCoherent>(x, q.y)), xyz(clothPos<kCoherent>(x, q.z)),
                                                    xyz(clothPos<kCoherent>(x, q.w)));
    const float angle = f.valid ? atan2f(f.sine, f.cosine) : 0.0f;
    const float3 ag = f.valid ? clothDihedralGradient(f, slot) : f3(0, 0, 0);
    if (!f.valid || !finiteS(angle) || !finiteV(ag)) {
      gadd(grad, f3(kF32Max, kF32Max, kF32Max));
      continue;
    }
    const float4 rest = __ldg(&hinges[2ull * h + 1]);
    const float ws = m.bending * rest.y;
    gadd(grad, (ws * clothWrappedAngle(angle, rest.x)) * ag);
    if (kHessian) saddOuter(hess, ws, ag);
  }
}

}  // namespace jgs2
