// JGS2 step kernels for sm_100a.
//
// One frame of the stable Neo-Hookean Jacobi schedule runs as
//   prologue            predict + iteration-0 vertex frames + source preflight
//   per iteration:
//     solve             warp-cooperative per-vertex JGS2 local solve
//     gate              assembled determinant / energy reduction + accept
//     convergence       whole-pose revert, five-component residual, history,
//                       and the next iteration's vertex frames
//   epilogue            canonical copy, optional body correction, finalize
// which covers the reference's predict, tetPolarRotation, vertexPolarRotation,
// jgs2Solve, assembledVertexEnergy, candidateTetrahedron, reduceCandidate,
// applyCandidate, convergenceGradient, reduceConvergence, copyPosition,
// bodyHorizontalCorrection and finalize entry points
// (src/simulation/gpu/jgs2-shader.ts:2660-4589).  The graph-coloured schedule
// adds a copy and, per colour, a frame pass over the vertices that colour
// reads plus an in-place solve over the colour's vertices.
//
// Grid-wide reductions finish in the last block to arrive (a ticket counter);
// sums are combined in block order so results are deterministic.  No kernel
// waits on another block.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "jgs2_cloth.cuh"
#include "jgs2_contact.cuh"
#include "jgs2_device.cuh"
#include "jgs2_kernels.cuh"

namespace jgs2 {
namespace {

constexpr int kBlock = 128;

// Checked build: device index checks in the gathers.  A failing check records
// its site once (the host reports it at the next synchronisation as
// JGS2_DEVICE_ERROR) and the gather skips the element, so the kernel never
// reads out of bounds.  Compiled out otherwise.
#ifndef JGS2_BOUNDS_CHECKS
#define JGS2_BOUNDS_CHECKS 0
#endif
enum BoundsSite : uint32_t {
  kSiteRecordTet = 1, kSiteRecordVertex = 2, kSiteIncidentTet = 3, kSiteTetVertex = 4, kSiteContactVertex = 5,
  kSiteListVertex = 6,
};
#if JGS2_BOUNDS_CHECKS
__device__ uint32_t gBoundsViolation;
#endif
__device__ __forceinline__ bool inBounds(uint64_t index, uint64_t limit, uint32_t site) {
#if JGS2_BOUNDS_CHECKS
  if (index < limit) return true;
  atomicCAS(&gBoundsViolation, 0u, site);
  return false;
#else
  (void)index; (void)limit; (void)site;
  return true;
#endif
}
__device__ __forceinline__ bool tetVerticesInBounds(const uint4& q, uint32_t V) {
  return inBounds(q.x, V, kSiteTetVertex) && inBounds(q.y, V, kSiteTetVertex) && inBounds(q.z, V, kSiteTetVertex) &&
         inBounds(q.w, V, kSiteTetVertex);
}
#ifndef JGS2_SOLVE_LANES
#define JGS2_SOLVE_LANES 4
#endif
// Lanes per vertex in the solve kernel.  A warp holds 32 / kGroup lane groups;
// a width that does not divide 32 leaves the warp's last lanes idle.
constexpr int kGroup = JGS2_SOLVE_LANES;
#ifndef JGS2_FRAME_QUAT
#define JGS2_FRAME_QUAT 0
#endif
// Incident-tet gathers request the next tet's record before the current
// one's arithmetic (convergence, frames, the line search).
#ifndef JGS2_CONV_LOOKAHEAD
#define JGS2_CONV_LOOKAHEAD 1
#endif
constexpr int kRecFloats = 56;  // cached cubature record state

struct TetRec {
  float3 g1, g2, g3;
  float vol, lambda, mu;
  uint4 idx;
};

__device__ __forceinline__ TetRec loadTet(const float4* __restrict__ tets, uint32_t t) {
  const float4 a = __ldg(&tets[4ull * t]);
  const float4 b = __ldg(&tets[4ull * t + 1]);
  const float4 c = __ldg(&tets[4ull * t + 2]);
  const uint4 q = __ldg(reinterpret_cast<const uint4*>(tets) + 4ull * t + 3);
  TetRec r;
  r.g1 = f3(a.x, a.y, a.z);
  r.g2 = f3(b.x, b.y, b.z);
  r.g3 = f3(c.x, c.y, c.z);
  r.vol = a.w;
  r.lambda = b.w;
  r.mu = c.w;
  r.idx = q;
  return r;
}

// An incident-tet entry (tet * 4 + slot) and its record; false when a
// checked build finds the tet or one of its vertices out of range.
__device__ __forceinline__ bool incidentTetChecked(const float4* __restrict__ tets, uint32_t entry, uint32_t T,
                                                   uint32_t V, TetRec* r) {
  if (!inBounds(entry >> 2, T, kSiteIncidentTet)) return false;
  *r = loadTet(tets, entry >> 2);
  return tetVerticesInBounds(r->idx, V);
}

__device__ __forceinline__ float3 shapeGradient(const TetRec& r, uint32_t slot) {
  if (slot == 1) return r.g1;
  if (slot == 2) return r.g2;
  if (slot == 3) return r.g3;
  return -(r.g1 + r.g2 + r.g3);
}

__device__ __forceinline__ uint32_t idxAt(const uint4& q, uint32_t l) {
  return l == 0 ? q.x : (l == 1 ? q.y : (l == 2 ? q.z : q.w));
}

__device__ __forceinline__ M3 deformation(const TetRec& r, float3 x0, float3 x1, float3 x2, float3 x3) {
  return outer(x1 - x0, r.g1) + outer(x2 - x0, r.g2) + outer(x3 - x0, r.g3);
}

__device__ __forceinline__ M3 deformationAt(const TetRec& r, const float4* __restrict__ x) {
  return deformation(r, xyz(x[r.idx.x]), xyz(x[r.idx.y]), xyz(x[r.idx.z]), xyz(x[r.idx.w]));
}

__device__ __forceinline__ M3 loadRot(const float4* __restrict__ rot, uint32_t v) {
  const float4 a = rot[3ull * v], b = rot[3ull * v + 1], c = rot[3ull * v + 2];
  return {f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z)};
}

// Reads of arrays that other blocks of the same launch may write (positions
// and vertex frames inside the persistent coloured sweep): kCoherent loads are
// ordinary weak loads (ld.global.ca), which the grid barrier's release and
// acquire fences order after the other blocks' writes; they never take the
// non-coherent read-only path (ld.global.nc), which a const __restrict__
// pointer may select and which no fence orders.  Other launches read these
// arrays as read-only data.
template <bool kCoherent>
__device__ __forceinline__ float4 ldPos(const float4* p, size_t i) {
  if constexpr (kCoherent) return __ldca(p + i);
  else return p[i];
}
__device__ __forceinline__ M3 quaternionFrame(float4 q);
template <bool kCoherent>
__device__ __forceinline__ M3 loadRotT(const float4* rot, uint32_t v) {
#if JGS2_FRAME_QUAT
  return quaternionFrame(kCoherent ? __ldca(rot + 3ull * v) : rot[3ull * v]);
#endif
  if constexpr (kCoherent) {
    const float4 a = __ldca(rot + 3ull * v), b = __ldca(rot + 3ull * v + 1), c = __ldca(rot + 3ull * v + 2);
    return {f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z)};
  } else {
    return loadRot(rot, v);
  }
}
template <bool kCoherent>
__device__ __forceinline__ M3 deformationAtT(const TetRec& r, const float4* x) {
  if constexpr (kCoherent)
    return deformation(r, xyz(__ldca(x + r.idx.x)), xyz(__ldca(x + r.idx.y)), xyz(__ldca(x + r.idx.z)),
                       xyz(__ldca(x + r.idx.w)));
  else
    return deformationAt(r, x);
}

__device__ __forceinline__ void storeRot(float4* __restrict__ rot, uint32_t v, const M3& m) {
  rot[3ull * v] = make_float4(m.c0.x, m.c0.y, m.c0.z, 0.f);
  rot[3ull * v + 1] = make_float4(m.c1.x, m.c1.y, m.c1.z, 0.f);
  rot[3ull * v + 2] = make_float4(m.c2.x, m.c2.y, m.c2.z, 0.f);
}

// Vertex frames.  With JGS2_FRAME_QUAT a frame is stored as a unit
// quaternion in the first float4 of its three (one vector load per read
// instead of three); the matrix is rebuilt from it on every read.
__device__ __forceinline__ float4 frameQuaternion(const M3& m) {
  // Shepperd's method on the largest of the trace and the diagonal.
  const float m00 = m.c0.x, m11 = m.c1.y, m22 = m.c2.z;
  const float m21 = m.c1.z, m12 = m.c2.y, m02 = m.c2.x, m20 = m.c0.z, m10 = m.c0.y, m01 = m.c1.x;
  const float tr = m00 + m11 + m22;
  float4 q;
  if (tr > 0.0f) {
    const float t = sqrtf(tr + 1.0f) * 2.0f;
    q = make_float4((m21 - m12) / t, (m02 - m20) / t, (m10 - m01) / t, 0.25f * t);
  } else if (m00 > m11 && m00 > m22) {
    const float t = sqrtf(1.0f + m00 - m11 - m22) * 2.0f;
    q = make_float4(0.25f * t, (m01 + m10) / t, (m02 + m20) / t, (m21 - m12) / t);
  } else if (m11 > m22) {
    const float t = sqrtf(1.0f + m11 - m00 - m22) * 2.0f;
    q = make_float4((m01 + m10) / t, 0.25f * t, (m12 + m21) / t, (m02 - m20) / t);
  } else {
    const float t = sqrtf(1.0f + m22 - m00 - m11) * 2.0f;
    q = make_float4((m02 + m20) / t, (m12 + m21) / t, 0.25f * t, (m10 - m01) / t);
  }
  const float n = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  return make_float4(q.x * n, q.y * n, q.z * n, q.w * n);
}
__device__ __forceinline__ M3 quaternionFrame(float4 q) {
  const float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
  const float xx = q.x * x2, yy = q.y * y2, zz = q.z * z2;
  const float xy = q.x * y2, xz = q.x * z2, yz = q.y * z2;
  const float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
  return {f3(1.0f - (yy + zz), xy + wz, xz - wy), f3(xy - wz, 1.0f - (xx + zz), yz + wx),
          f3(xz + wy, yz - wx, 1.0f - (xx + yy))};
}
__device__ __forceinline__ void storeFrame(float4* __restrict__ rot, uint32_t v, const M3& m) {
#if JGS2_FRAME_QUAT
  rot[3ull * v] = frameQuaternion(m);
#else
  storeRot(rot, v, m);
#endif
}
__device__ __forceinline__ M3 loadFrame(const float4* __restrict__ rot, uint32_t v) {
#if JGS2_FRAME_QUAT
  return quaternionFrame(rot[3ull * v]);
#else
  return loadRot(rot, v);
#endif
}

// Row-major stored Ubar block l -> columns (cubatureBlock, jgs2-shader.ts:1204-1212).
// The record's 36 basis floats are 9 float4: floats [9l, 9l + 9) lie
// in the three float4 starting at (9l) / 4, so three vector loads replace nine
// scalar ones.  l must be a compile-time constant after unrolling.
__device__ __forceinline__ M3 loadBlockVec(const float4* __restrict__ rec, int l) {
  const int k0 = (9 * l) >> 2;
  const int off = 9 * l - 4 * k0;
  const float4 a = __ldg(rec + k0), b = __ldg(rec + k0 + 1), c = __ldg(rec + k0 + 2);
  const float f[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
  return {f3(f[off + 0], f[off + 3], f[off + 6]), f3(f[off + 1], f[off + 4], f[off + 7]),
          f3(f[off + 2], f[off + 5], f[off + 8])};
}

__device__ __forceinline__ uint32_t controlBits(float packed) {
  if (!finiteS(packed) || packed < 0.0f || packed > float(kControlMask) || packed != floorf(packed)) return 0u;
  return static_cast<uint32_t>(packed);
}

__device__ __forceinline__ bool latched(const DevParams& p, const FrameState* fs) {
  if (!p.stopEnabled) return false;
  return (controlBits(fs->control[0].w) & kStopLatchBit) != 0u;
}

__device__ __forceinline__ bool finiteNonnegInt(float v, float maximum) {
  return finiteS(v) && v >= 0.0f && v <= maximum && v == floorf(v);
}

__device__ __forceinline__ bool isPinned(const uint4& info) { return info.z != 0u; }

__device__ __forceinline__ ClothMaterial clothMaterial(const DevParams& p) {
  return {p.clothLambda, p.clothMu, p.clothThickness, p.clothBending};
}

__device__ __forceinline__ float distributedInertiaWeight(const float4& rm, const uint4& info, float invDt2) {
  if (isPinned(info)) return 0.0f;
  return rm.w * invDt2 / float(info.y > 1u ? info.y : 1u);
}

// vertexObjectiveGradient (jgs2-shader.ts:1926-1938).
__device__ __forceinline__ float3 objectiveGradient(const DevParams& p, const Buffers& b, uint32_t v, float3 pos) {
  float3 r = f3(0, 0, 0);
  if (p.objectiveFlags & 1u) r = r - xyz(b.forces[v]);
  if (p.objectiveFlags & 2u) {
    const float4 t = b.targets[v];
    if (t.w > 0.0f) r = r + t.w * (pos - xyz(t));
  }
  return r;
}

__device__ __forceinline__ float targetStiffness(const DevParams& p, const Buffers& b, uint32_t v) {
  return (p.objectiveFlags & 2u) ? b.targets[v].w : 0.0f;
}

// vertexObjectiveEnergyDelta (jgs2-shader.ts:1903-1924).
__device__ __forceinline__ float objectiveDelta(const DevParams& p, const Buffers& b, uint32_t v, float3 base,
                                                float3 d) {
  float r = 0.0f;
  if (p.objectiveFlags & 1u) r -= dot3(xyz(b.forces[v]), d);
  if (p.objectiveFlags & 2u) {
    const float4 t = b.targets[v];
    if (t.w > 0.0f) r += t.w * (dot3(base - xyz(t), d) + 0.5f * dot3(d, d));
  }
  return r;
}

__device__ __forceinline__ float floorDelta(const DevParams& p, float baseY, float dY) {
  if (!(p.floorStiffness > 0.0f)) return 0.0f;
  const float i = fminf(0.0f, baseY - p.floorHeight);
  const float f = fminf(0.0f, baseY + dY - p.floorHeight);
  return 0.5f * p.floorStiffness * (f - i) * (f + i);
}

// vertexImplicitEnergyAt without cloth/IPC terms (jgs2-shader.ts:2557-2645).
__device__ __forceinline__ float implicitEnergy(const DevParams& p, const Buffers& b, uint32_t v, float3 x,
                                                const uint4& info) {
  if (isPinned(info)) return 0.0f;
  const float4 rm = b.restMass[v];
  const float3 r = x - xyz(b.predicted[v]);
  float e = 0.5f * (rm.w * p.invDt2) * dot3(r, r);
  if (p.objectiveFlags != 0u) {
    if (p.objectiveFlags & 1u) e -= dot3(xyz(b.forces[v]), x);
    if (p.objectiveFlags & 2u) {
      const float4 t = b.targets[v];
      if (t.w > 0.0f) {
        const float3 q = x - xyz(t);
        e += 0.5f * t.w * dot3(q, q);
      }
    }
  }
  if (p.floorStiffness > 0.0f) {
    const float pen = fminf(0.0f, x.y - p.floorHeight);
    e += 0.5f * p.floorStiffness * pen * pen;
  }
  return e;
}

// Reductions over a lane group of W lanes inside one warp.  A power-of-two
// width folds with an xor butterfly; another width gathers the group's values
// in lane order on every lane, so all lanes hold the same, order-fixed result.
template <int W>
__device__ __forceinline__ uint32_t groupBase() {
  return ((threadIdx.x & 31u) / W) * W;
}
template <int W>
__device__ __forceinline__ float groupSum(float v, unsigned mask) {
  if constexpr ((W & (W - 1)) == 0) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, W);
    return v;
  } else {
    const uint32_t base = groupBase<W>();
    float s = __shfl_sync(mask, v, base);
#pragma unroll
    for (int j = 1; j < W; ++j) s += __shfl_sync(mask, v, base + j);
    return s;
  }
}
// Merge of the lanes' compensated sums over a lane group (xor butterfly;
// every lane ends with the same pair because the merge is symmetric).
template <int W>
__device__ __forceinline__ Comp3 shflComp(const Comp3& a, unsigned mask, uint32_t src) {
  Comp3 t;
  t.s.x = __shfl_sync(mask, a.s.x, src);
  t.s.y = __shfl_sync(mask, a.s.y, src);
  t.s.z = __shfl_sync(mask, a.s.z, src);
  t.c.x = __shfl_sync(mask, a.c.x, src);
  t.c.y = __shfl_sync(mask, a.c.y, src);
  t.c.z = __shfl_sync(mask, a.c.z, src);
  return t;
}
template <int W>
__device__ __forceinline__ void groupMerge(Comp3& a, unsigned mask) {
  if constexpr ((W & (W - 1)) == 0) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) {
      Comp3 t;
      t.s.x = __shfl_xor_sync(mask, a.s.x, o, W);
      t.s.y = __shfl_xor_sync(mask, a.s.y, o, W);
      t.s.z = __shfl_xor_sync(mask, a.s.z, o, W);
      t.c.x = __shfl_xor_sync(mask, a.c.x, o, W);
      t.c.y = __shfl_xor_sync(mask, a.c.y, o, W);
      t.c.z = __shfl_xor_sync(mask, a.c.z, o, W);
      cmerge(a, t);
    }
  } else {
    const uint32_t base = groupBase<W>();
    Comp3 r = shflComp<W>(a, mask, base);
#pragma unroll
    for (int j = 1; j < W; ++j) cmerge(r, shflComp<W>(a, mask, base + j));
    a = r;
  }
}
template <int W>
__device__ __forceinline__ float groupMin(float v, unsigned mask) {
  if constexpr ((W & (W - 1)) == 0) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(mask, v, o, W));
    return v;
  } else {
    const uint32_t base = groupBase<W>();
    float m = __shfl_sync(mask, v, base);
#pragma unroll
    for (int j = 1; j < W; ++j) m = fminf(m, __shfl_sync(mask, v, base + j));
    return m;
  }
}

// Deterministic block sum of doubles (fixed tree order).
template <int N>
__device__ __forceinline__ void blockSumDoubles(double (&vals)[N], double* scratch /* N * kBlock */) {
#pragma unroll
  for (int i = 0; i < N; ++i) scratch[i * kBlock + threadIdx.x] = vals[i];
  __syncthreads();
  for (int stride = kBlock / 2; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) {
#pragma unroll
      for (int i = 0; i < N; ++i)
        scratch[i * kBlock + threadIdx.x] += scratch[i * kBlock + threadIdx.x + stride];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < N; ++i) vals[i] = scratch[i * kBlock];
}

// Exact incident block of the local Hessian for shape gradient g
// (jgs2-shader.ts:3097-3111): vol (a |g|^2 I + c1 u u^T + lambda w w^T) with
// u = F g and w = cof(F) g, the stable Neo-Hookean tangent applied to the
// rank-one direction e_i g^T.
__device__ __forceinline__ void addIncidentBlock(S3& hess, const TetRec& r, const M3& F, const PiolaTerms& pt,
                                                 float3 g) {
  const float3 u1 = mv(F, g), w1 = mv(pt.cof, g);
  S3 blk = szero();
  saddDiag(blk, pt.a * dot3(g, g));
  saddOuter(blk, pt.c1, u1);
  saddOuter(blk, r.lambda, w1);
  saddScaled(hess, r.vol, blk);
}

__device__ __forceinline__ void storeIncident(float4* __restrict__ inc, uint32_t v, float3 g, const S3& h) {
  inc[3ull * v] = make_float4(g.x, g.y, g.z, h.xx);
  inc[3ull * v + 1] = make_float4(h.yy, h.zz, h.xy, h.xz);
  inc[3ull * v + 2] = make_float4(h.yz, 0.0f, 0.0f, 0.0f);
}

// Vertex frame and incident system of a free vertex at pose x in one pass
// over its incident tets: the frame is the polar of the volume-weighted
// average F (vertexPolarRotation, jgs2-shader.ts:2959-2989), the system the
// incident material gradient sum vol P(F) g and Hessian blocks, plus the
// cloth membrane and bending terms of the vertex's incident elements.
__device__ __forceinline__ void frameAndIncident(const Buffers& b, const DevParams& p, const float4* __restrict__ x,
                                                 uint32_t v, const uint4& info, float eps) {
  M3 avg = mzero();
  float total = 0.0f;
  Comp3 grad = czero();  // compensated gradient gather
  S3 hess = szero();
#if JGS2_CONV_LOOKAHEAD
  uint32_t nextEntry = info.y ? __ldg(&b.adjacency[info.x]) : 0u;
  TetRec nextRec;
  bool nextOk = false;
  if (info.y) nextOk = incidentTetChecked(b.tets, nextEntry, b.tetTotal, b.vertexTotal, &nextRec);
#endif
  for (uint32_t a = 0; a < info.y; ++a) {
#if JGS2_CONV_LOOKAHEAD
    const uint32_t entry = nextEntry;
    const TetRec r = nextRec;
    const bool tetOk = nextOk;
    if (a + 1 < info.y) {
      nextEntry = __ldg(&b.adjacency[info.x + a + 1]);
      nextOk = incidentTetChecked(b.tets, nextEntry, b.tetTotal, b.vertexTotal, &nextRec);
    }
#else
    const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
    TetRec r;
    const bool tetOk = incidentTetChecked(b.tets, entry, b.tetTotal, b.vertexTotal, &r);
#endif
    if (!tetOk) continue;
    const M3 F = deformationAt(r, x);
    const PiolaTerms pt = piolaTerms(F, r.lambda, r.mu);
    const float3 g = shapeGradient(r, entry & 3u);
    cadd(grad, r.vol * mv(piola(F, pt), g));
    addIncidentBlock(hess, r, F, pt, g);
    avg = avg + r.vol * F;
    total += r.vol;
  }
  if (p.cloth)
    clothLocalSystem<true>(b.clothTris, b.clothHinges, b.clothIncidence, b.clothRange[v], x, clothMaterial(p), 0u, 1u,
                           grad, hess);
  const M3 favg = total > 0.0f ? (1.0f / total) * avg : midentity();
  storeFrame(b.vertexRot, v, info.y == 0u ? midentity() : polarRotation(favg, eps));
  storeIncident(b.incident, v, cvalue(grad), hess);
}

// Vertex frame: polar of the volume-weighted average F over incident tets
// (vertexPolarRotation, jgs2-shader.ts:2959-2989).
template <bool kCoherent = false>
__device__ __forceinline__ M3 vertexFrame(const Buffers& b, const float4* __restrict__ x, uint32_t v, float eps) {
  const uint4 info = b.vinfo[v];
  if (info.y == 0u) return midentity();
  M3 avg = mzero();
  float total = 0.0f;
  for (uint32_t a = 0; a < info.y; ++a) {
    const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
    TetRec r;
    if (!incidentTetChecked(b.tets, entry, b.tetTotal, b.vertexTotal, &r)) continue;
    avg = avg + r.vol * deformationAtT<kCoherent>(r, x);
    total += r.vol;
  }
  avg = total > 0.0f ? (1.0f / total) * avg : midentity();
  return polarRotation(avg, eps);
}

// Vertex frames for a list of vertices (or all) from pose x.
__global__ void __launch_bounds__(kBlock) vertexPolarKernel(Buffers b, const DevParams* __restrict__ pp,
                                                            const float4* __restrict__ x,
                                                            const uint32_t* __restrict__ list, uint32_t count) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= count) return;
  const uint32_t v = list ? list[i] : i;
  const uint32_t scene = b.vertexScene[v];
  const DevParams& p = pp[scene];
  if (!p.active || latched(p, &b.frames[scene])) return;
  storeFrame(b.vertexRot, v, vertexFrame(b, x, v, p.rotationEpsilon));
}

// ---------------------------------------------------------------------------
// Co-rotated linear path (the reference's legacy co-rotated branches of
// jgs2Solve and tetPolarRotation, jgs2-shader.ts:2931-2957, 2991-3263,
// 2479-2512).  No globalization: each vertex takes a regularised Newton step
// clamped to maxStep, and no gate or convergence pass follows.

// Tet frames: polar of each co-rotated tet's deformation gradient.
__global__ void __launch_bounds__(kBlock) tetPolarKernel(Buffers b, const DevParams* __restrict__ pp,
                                                         const float4* __restrict__ x, uint32_t T) {
  const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= T) return;
  const DevParams& p = pp[b.tetScene[t]];
  if (!p.active) return;
  const TetRec r = loadTet(b.tets, t);
  storeRot(b.tetRot, t, polarRotation(deformationAt(r, x), p.rotationEpsilon));
}

// Block (rv, cv) of a tet's 12 x 12 row-major rest stiffness, as columns.
__device__ __forceinline__ M3 stiffnessBlock(const float* __restrict__ k, uint32_t rv, uint32_t cv) {
  const float* r0 = k + (3 * rv) * 12 + 3 * cv;
  const float* r1 = r0 + 12;
  const float* r2 = r1 + 12;
  return {f3(r0[0], r1[0], r2[0]), f3(r0[1], r1[1], r2[1]), f3(r0[2], r1[2], r2[2])};
}

// Element gradient of a co-rotated tet at pose x (tetGradient):
// R K (R^T (x_l - centroid) - (X_l - rest centroid)) per vertex slot.
__device__ __forceinline__ void corotatedGradient(const Buffers& b, const float4* __restrict__ x, uint32_t t,
                                                  const uint4& q, const M3& R, float3 out[4]) {
  float3 cur[4], rest[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const uint32_t v = idxAt(q, l);
    cur[l] = xyz(x[v]);
    rest[l] = xyz(b.restMass[v]);
  }
  const float3 cc = 0.25f * (cur[0] + cur[1] + cur[2] + cur[3]);
  const float3 rc = 0.25f * (rest[0] + rest[1] + rest[2] + rest[3]);
  const M3 Rt = mtrans(R);
  float3 disp[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) disp[l] = mv(Rt, cur[l] - cc) - (rest[l] - rc);
  const float* k = b.stiffness + 144ull * t;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    float3 lg = f3(0, 0, 0);
#pragma unroll
    for (int c = 0; c < 4; ++c) lg = lg + mv(stiffnessBlock(k, r, c), disp[c]);
    out[r] = mv(R, lg);
  }
}

// Reduced Hessian of a co-rotated record (cubatureHessian):
// column c = sum_l B_l^T R K_l. R^T B_.[:, c].
__device__ __forceinline__ M3 corotatedRecordHessian(const Buffers& b, uint32_t t, const M3& R, const M3 basis[4]) {
  const M3 Rt = mtrans(R);
  const float* k = b.stiffness + 144ull * t;
  M3 out;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float3 ld[4], wp[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) ld[l] = mv(Rt, c == 0 ? basis[l].c0 : (c == 1 ? basis[l].c1 : basis[l].c2));
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      float3 lp = f3(0, 0, 0);
#pragma unroll
      for (int cv = 0; cv < 4; ++cv) lp = lp + mv(stiffnessBlock(k, r, cv), ld[cv]);
      wp[r] = mv(R, lp);
    }
    float3 col;
    col.x = dot3(basis[0].c0, wp[0]) + dot3(basis[1].c0, wp[1]) + dot3(basis[2].c0, wp[2]) + dot3(basis[3].c0, wp[3]);
    col.y = dot3(basis[0].c1, wp[0]) + dot3(basis[1].c1, wp[1]) + dot3(basis[2].c1, wp[2]) + dot3(basis[3].c1, wp[3]);
    col.z = dot3(basis[0].c2, wp[0]) + dot3(basis[1].c2, wp[1]) + dot3(basis[2].c2, wp[2]) + dot3(basis[3].c2, wp[3]);
    if (c == 0) out.c0 = col;
    else if (c == 1) out.c1 = col;
    else out.c2 = col;
  }
  return out;
}

// Distributed objective gradient / target stiffness of a record vertex.
__device__ __forceinline__ float3 distributedObjective(const DevParams& p, const Buffers& b, uint32_t q, float3 x,
                                                     const uint4& qi) {
  if (isPinned(qi)) return f3(0, 0, 0);
  return objectiveGradient(p, b, q, x) * (1.0f / float(qi.y > 1u ? qi.y : 1u));
}

// One thread per vertex: the exact co-rotated gather, the cubature
// complement and the regularised solve (regularizedSolve, :2479-2512).
__global__ void __launch_bounds__(kBlock) corotatedSolveKernel(Buffers b, const DevParams* __restrict__ pp,
                                                               const float4* __restrict__ src, float4* tgt,
                                                               const uint32_t* __restrict__ list, uint32_t count,
                                                               uint32_t K) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= count) return;
  const uint32_t v = list ? list[i] : i;
  const DevParams& p = pp[b.vertexScene[v]];
  if (!p.active) return;
  const uint4 info = b.vinfo[v];
  const float4 rm = b.restMass[v];
  if (isPinned(info)) {
    tgt[v] = make_float4(rm.x, rm.y, rm.z, 1.0f);
    b.finalUpdate[v] = 0.0f;
    return;
  }
  const float3 position = xyz(src[v]);
  const float4 pv = b.predicted[v];
  const float inertia = rm.w * p.invDt2;
  const bool objActive = p.objectiveFlags != 0u;
  Comp3 gsum = czero();  // compensated gradient gather
  cadd(gsum, inertia * (position - xyz(pv)));
  M3 hess = inertia * midentity();
  if (objActive) cadd(gsum, objectiveGradient(p, b, v, position));
  if (p.objectiveFlags & 2u) hess = hess + targetStiffness(p, b, v) * midentity();
  for (uint32_t a = 0; a < info.y; ++a) {
    const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
    const uint32_t t = entry >> 2, slot = entry & 3u;
    const TetRec r = loadTet(b.tets, t);
    const M3 R = loadRot(b.tetRot, t);
    float3 tg[4];
    corotatedGradient(b, src, t, r.idx, R, tg);
    cadd(gsum, tg[slot]);
    hess = hess + mm(mm(R, stiffnessBlock(b.stiffness + 144ull * t, slot, slot)), mtrans(R));
  }
  if (p.floorStiffness > 0.0f && position.y < p.floorHeight) {
    cadd(gsum, f3(0.0f, p.floorStiffness * (position.y - p.floorHeight), 0.0f));
    hess.c1.y += p.floorStiffness;
  }
  const M3 RsT = mtrans(loadFrame(b.vertexRot, v));
  const float dWs = pv.w;
  for (uint32_t s = 0; s < K; ++s) {
    const size_t rec = static_cast<size_t>(v) * K + s;
    const uint4 head = __ldg(&b.cubHead[2 * rec]);
    const float w = __uint_as_float(head.y);
    if (head.x == kEmptyTet || !(w > 0.0f)) continue;
    const uint32_t t = head.x;
    const uint4 q = __ldg(&b.cubHead[2 * rec + 1]);
    const float4* U = b.cubBasis + 9ull * rec;
    M3 basis[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) basis[l] = mm(mm(loadFrame(b.vertexRot, idxAt(q, l)), loadBlockVec(U, l)), RsT);
    const M3 R = loadRot(b.tetRot, t);
    float3 tg[4];
    corotatedGradient(b, src, t, q, R, tg);
    float3 pg = f3(0, 0, 0);
    M3 ih = mzero();
    uint32_t ss = 4;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const uint32_t qv = idxAt(q, l);
      if (qv == v) ss = l;
      const float4 pq = b.predicted[qv];
      const float3 xq = xyz(src[qv]);
      pg = pg + mtv(basis[l], tg[l] + pq.w * (xq - xyz(pq)));
      ih = ih + pq.w * mm(mtrans(basis[l]), basis[l]);
    }
    if (objActive) {
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const uint32_t qv = idxAt(q, l);
        pg = pg + mtv(basis[l], distributedObjective(p, b, qv, xyz(src[qv]), b.vinfo[qv]));
      }
    }
    M3 ph = corotatedRecordHessian(b, t, R, basis) + ih;
    if (p.objectiveFlags & 2u) {
      M3 oh = mzero();
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const uint32_t qv = idxAt(q, l);
        const uint4 qi = b.vinfo[qv];
        const float kt = isPinned(qi) ? 0.0f : targetStiffness(p, b, qv) / float(qi.y > 1u ? qi.y : 1u);
        oh = oh + kt * mm(mtrans(basis[l]), basis[l]);
      }
      ph = ph + oh;
    }
    if (ss < 4) {
      pg = pg - (tg[ss] + dWs * (position - xyz(pv)));
      if (objActive) pg = pg - distributedObjective(p, b, v, position, info);
      ph = ph - (mm(mm(R, stiffnessBlock(b.stiffness + 144ull * t, ss, ss)), mtrans(R)) + dWs * midentity());
      if (p.objectiveFlags & 2u)
        ph = ph - (targetStiffness(p, b, v) / float(info.y > 1u ? info.y : 1u)) * midentity();
    }
    cadd(gsum, w * pg);
    hess = hess + w * ph;
  }
  // Regularised Cholesky solve with the shift max(regularization * scale, 1e-9).
  const float ds = fmaxf(1.0f, fmaxf(fabsf(hess.c0.x), fmaxf(fabsf(hess.c1.y), fabsf(hess.c2.z))));
  const float shift = fmaxf(p.regularization * ds, 1.0e-9f);
  const float a00 = hess.c0.x + shift, a11 = hess.c1.y + shift, a22 = hess.c2.z + shift;
  const float a01 = 0.5f * (hess.c0.y + hess.c1.x);
  const float a02 = 0.5f * (hess.c0.z + hess.c2.x);
  const float a12 = 0.5f * (hess.c1.z + hess.c2.y);
  const float3 rhs = -cvalue(gsum);
  const float l00 = sqrtf(fmaxf(a00, shift));
  const float l10 = a01 / l00, l20 = a02 / l00;
  const float l11 = sqrtf(fmaxf(a11 - l10 * l10, shift));
  const float l21 = (a12 - l20 * l10) / l11;
  const float l22 = sqrtf(fmaxf(a22 - l20 * l20 - l21 * l21, shift));
  const float y0 = rhs.x / l00, y1 = (rhs.y - l10 * y0) / l11, y2 = (rhs.z - l20 * y0 - l21 * y1) / l22;
  const float x2 = y2 / l22, x1 = (y1 - l21 * x2) / l11, x0 = (y0 - l10 * x1 - l20 * x2) / l00;
  float3 delta = f3(x0, x1, x2);
  const float sq = dot3(delta, delta);
  if (!(sq >= 0.0f && sq < 1.0e30f)) delta = f3(0, 0, 0);
  const float dls = dot3(delta, delta);
  if (p.maxStep > 0.0f && dls > p.maxStep * p.maxStep) delta = delta * (p.maxStep * (1.0f / sqrtf(dls)));
  const float3 np = position + delta;
  tgt[v] = make_float4(np.x, np.y, np.z, 1.0f);
  b.finalUpdate[v] = sqrtf(dot3(delta, delta));
}

__global__ void __launch_bounds__(kBlock) copyKernel(Buffers b, const DevParams* __restrict__ pp,
                                                     const float4* __restrict__ src, float4* __restrict__ dst,
                                                     uint32_t V) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < V && pp[b.vertexScene[i]].active) {
    const float4 s = src[i];
    dst[i] = make_float4(s.x, s.y, s.z, 1.0f);
  }
}

// ---------------------------------------------------------------------------
// IPC contact (jgs2-shader.ts:233-874, 2694-2917).

// Candidates listed this iteration: the broad phase's count with a contact
// surface, else the static total.  Candidate kernels stride over it.
__device__ __forceinline__ uint32_t contactListed(const Buffers& b) {
  return b.contactDynamic ? __ldcg(b.bpStatus) : b.contactCount;
}

__device__ __forceinline__ uint4 contactIndices(const Buffers& b, uint32_t c, uint32_t* type) {
  uint4 q = __ldg(&b.contactIdx[c]);
  *type = q.w >> 31;
  q.w &= 0x7fffffffu;
#if JGS2_BOUNDS_CHECKS
  // An out-of-range candidate vertex is recorded and read as vertex 0.
  if (!inBounds(q.x, b.vertexTotal, kSiteContactVertex)) q.x = 0;
  if (!inBounds(q.y, b.vertexTotal, kSiteContactVertex)) q.y = 0;
  if (!inBounds(q.z, b.vertexTotal, kSiteContactVertex)) q.z = 0;
  if (!inBounds(q.w, b.vertexTotal, kSiteContactVertex)) q.w = 0;
#endif
  return q;
}

__device__ __forceinline__ float3 posOverride(const float4* __restrict__ x, uint32_t q, uint32_t ov, float3 op) {
  return q == ov ? op : xyz(x[q]);
}

// ipcContactAtThreshold / ipcContactAtOverride (:594-668).
__device__ __forceinline__ ContactData contactAt(const Buffers& b, uint32_t c, const float4* __restrict__ x,
                                                 float threshold, uint32_t ov = 0xffffffffu,
                                                 float3 op = make_float3(0.f, 0.f, 0.f)) {
  uint32_t type;
  const uint4 q = contactIndices(b, c, &type);
  return ipcContactFromPositions(type, posOverride(x, q.x, ov, op), posOverride(x, q.y, ov, op),
                                 posOverride(x, q.z, ov, op), posOverride(x, q.w, ov, op), threshold);
}

// ipcContactRoundingReach (:505-509).
__device__ __forceinline__ float contactRoundingReach(const DevParams& p) {
  return fmaxf(fmaxf(p.sceneScale, p.ipcActivation), 1.0e-12f) * kUnitRoundoff * kPositionResolutionMultiplier;
}

// ipcCandidatePinnedMotionExceedsBound (:476-503).
__device__ __forceinline__ bool contactPinnedMotion(const Buffers& b, uint4 q, const float4* __restrict__ src,
                                                    float bound) {
  const uint32_t vs[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    if (!isPinned(b.vinfo[vs[l]])) continue;
    const float3 d = xyz(b.restMass[vs[l]]) - xyz(src[vs[l]]);
    const float len = length3(d);
    if (!finiteV(d) || !finiteS(len) || len > bound) return true;
  }
  return false;
}

// includeCandidate of buildActiveContactRows (:2742-2782): a candidate stays
// active unless its source cache is valid, beyond the reach a bounded step can
// cross, frictionless and free of unbounded pinned motion.  The decision
// depends on the candidate only, so every incident vertex agrees.
__device__ __forceinline__ bool contactIncluded(const Buffers& b, const DevParams& p, uint32_t c,
                                                const float4* __restrict__ src) {
  const float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
  const ContactData k = ipcCached(st[kContactSource], st[kContactSourceWeights]);
  const bool friction = p.ipcFriction > 0.0f && st[kContactLagged].w > 0.0f;
  const bool bounded = p.maxStep > 0.0f;
  const float reach = p.ipcActivation + 2.0f * (fmaxf(p.maxStep, 0.0f) + contactRoundingReach(p));
  uint32_t type;
  const uint4 q = contactIndices(b, c, &type);
  const bool pinnedMotion = contactPinnedMotion(b, q, src, fmaxf(p.maxStep, 0.0f));
  return !k.valid || !bounded || k.distance <= reach || friction || pinnedMotion;
}

// Displacement since the frame start weighted by the lagged weights
// (ipcWeightedDisplacement, :686-708).
__device__ __forceinline__ float3 contactRelative(const Buffers& b, uint4 q, float4 w, const float4* __restrict__ x,
                                                  uint32_t ov, float3 op) {
  float3 r = w.x * (posOverride(x, q.x, ov, op) - xyz(b.old[q.x]));
  r = r + w.y * (posOverride(x, q.y, ov, op) - xyz(b.old[q.y]));
  r = r + w.z * (posOverride(x, q.z, ov, op) - xyz(b.old[q.z]));
  r = r + w.w * (posOverride(x, q.w, ov, op) - xyz(b.old[q.w]));
  return r;
}

// ipcCandidateEnergyFromContact (:710-741).
__device__ __forceinline__ float contactEnergy(const Buffers& b, const DevParams& p, uint32_t c, const ContactData& k,
                                               const float4* __restrict__ x, uint32_t ov, float3 op) {
  if (!k.valid || !(k.distance > p.ipcMinDistance)) return kF32Max;
  float e = p.ipcStiffness * ipcBarrier(k.distance, p.ipcActivation);
  const float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
  const float4 lag = st[kContactLagged];
  if (p.ipcFriction > 0.0f && lag.w > 0.0f) {
    const float3 n = ipcSafeUnit(xyz(lag), k.normal);
    uint32_t type;
    const uint4 q = contactIndices(b, c, &type);
    const float3 rel = contactRelative(b, q, st[kContactLaggedWeights], x, ov, op);
    const float3 tang = rel - n * dot3(n, rel);
    e += p.dt * ipcFrictionDissipation(length3(tang) * p.invDt, p.ipcEpsilon, p.ipcFriction, lag.w);
  }
  return e;
}

// ipcLocalContribution (:788-869) over the vertex's active candidates
// [first, count) step `stride`: barrier gradient and PSD normal block, lagged
// friction gradient and tangential block.  `fresh` evaluates the contact at x
// (the coloured schedule), otherwise the cache at `slot` is used.
template <bool kHessian, class G>
__device__ __forceinline__ void contactLocal(const Buffers& b, const DevParams& p, uint32_t v,
                                             const float4* __restrict__ x, bool fresh, int slot, uint32_t first,
                                             uint32_t stride, G& grad, S3& hess) {
  const uint2 range = b.contactRange[v];
  const uint32_t n = b.activeCount[v];
  for (uint32_t a = first; a < n; a += stride) {
    const uint32_t c = b.activeIds[range.x + a];
    const float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
    const ContactData k = fresh ? contactAt(b, c, x, p.ipcActivation) : ipcCached(st[slot], st[slot + 1]);
    if (!k.valid) continue;
    const bool barrier = ipcBarrierActive(k.distance, p.ipcActivation);
    const float4 lag = st[kContactLagged];
    const bool friction = p.ipcFriction > 0.0f && lag.w > 0.0f;
    if (!barrier && !friction) continue;
    uint32_t type;
    const uint4 q = contactIndices(b, c, &type);
    if (ipcWeightFor(q, make_float4(1.f, 1.f, 1.f, 1.f), v) == 0.0f) continue;
    const float w = ipcWeightFor(q, k.weights, v);
    if (w != 0.0f && barrier) {
      gadd(grad, ipcNormalGradientScalar(w, p.ipcStiffness, ipcBarrier1(k.distance, p.ipcActivation)) * k.normal);
      if (kHessian) {
        const float s = ipcPsdScalar(w, p.ipcStiffness, ipcBarrier2(k.distance, p.ipcActivation));
        saddOuter(hess, fmaxf(s, 0.0f), ipcSafeUnit(k.normal, f3(1, 0, 0)));
      }
    }
    const float4 lagW = st[kContactLaggedWeights];
    const float lw = ipcWeightFor(q, lagW, v);
    if (friction && lw != 0.0f) {
      const float3 nrm = ipcSafeUnit(xyz(lag), k.normal);
      const float3 rel = contactRelative(b, q, lagW, x, 0xffffffffu, f3(0, 0, 0));
      const float3 tang = rel - nrm * dot3(nrm, rel);
      const float slip = length3(tang);
      const float scale = p.ipcFriction * lag.w;
      const float3 dir = slip > 1.0e-12f ? tang * (1.0f / slip) : f3(0, 0, 0);
      const float f1 = ipcFrictionF1(slip * p.invDt, p.ipcEpsilon);
      gadd(grad, (lw * scale * f1) * dir);
      if (kHessian) {
        float curvature = 2.0f * scale / fmaxf(p.ipcEpsilon * p.dt, 1.0e-12f);
        if (slip > 1.0e-12f) curvature = scale * f1 / slip;
        const float c2 = lw * lw * fmaxf(curvature, 0.0f);
        saddDiag(hess, c2);
        saddOuter(hess, -c2, ipcSafeUnit(nrm, f3(1, 0, 0)));
      }
    }
  }
}

// JGS2_CONTACT_MIN_BLOCKS: blocks per SM the register budgets of the
// per-candidate contact kernels (lag, safe step, validation, broad-phase
// initialisation) must allow (0: the compiler's choice).
#ifndef JGS2_CONTACT_MIN_BLOCKS
#define JGS2_CONTACT_MIN_BLOCKS 0
#endif
#if JGS2_CONTACT_MIN_BLOCKS > 0
#define JGS2_CONTACT_BOUNDS __launch_bounds__(kBlock, JGS2_CONTACT_MIN_BLOCKS)
#else
#define JGS2_CONTACT_BOUNDS __launch_bounds__(kBlock)
#endif

// lagContact (:2712-2740): source cache and lagged normal force at the
// accepted pose, once per frame.
__global__ void JGS2_CONTACT_BOUNDS contactLagKernel(Buffers b, const DevParams* __restrict__ pp) {
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  if (c >= b.contactCount) return;
  const uint32_t scene = b.contactScene[c];
  const DevParams& p = pp[scene];
  if (!p.active || !p.ipc) return;
  const ContactData k = contactAt(b, c, b.pos[0], p.ipcActivation + contactRoundingReach(p));
  float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
  ipcStoreCached(st, kContactSource, k);
  float4 force = make_float4(0, 0, 0, 0), w = make_float4(0, 0, 0, 0);
  if (k.valid && k.distance > p.ipcMinDistance) {
    const float f = fmaxf(0.0f, -p.ipcStiffness * ipcBarrier1(k.distance, p.ipcActivation));
    if (finiteS(f)) {
      force = make_float4(k.normal.x, k.normal.y, k.normal.z, f);
      w = k.weights;
    }
  }
  st[kContactLagged] = force;
  st[kContactLaggedWeights] = w;
  st[kContactScratch] = make_float4(1, 0, 0, 0);
  if (c == b.scenes[scene].kOff) b.frames[scene].contactAlpha = 1.0f;
}

// buildActiveContactRows (:2742-2782) in two passes: the candidate's
// inclusion (a property of the candidate alone), with the reset of the
// iteration's safe-step reductions...
__global__ void __launch_bounds__(kBlock) contactFlagKernel(Buffers b, const DevParams* __restrict__ pp,
                                                            const float4* __restrict__ src) {
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  if (c >= b.contactCount) return;
  const uint32_t scene = b.contactScene[c];
  const DevParams& p = pp[scene];
  if (!p.active || !p.ipc) return;
  if (c == b.scenes[scene].kOff) {
    FrameState* fs = &b.frames[scene];
    fs->stepAlphaBits = __float_as_uint(1.0f);
    fs->stepValid = 1u;
    fs->checkAlphaBits = __float_as_uint(1.0f);
    fs->checkValid = 1u;
  }
  b.contactFlag[c] = contactIncluded(b, p, c, src) ? 1u : 0u;
}

// ...then, one warp per vertex, the ordered compaction of its included
// incident candidates into its active row.
__global__ void __launch_bounds__(kBlock) contactRowsKernel(Buffers b, const DevParams* __restrict__ pp,
                                                            uint32_t V) {
  const uint32_t v = blockIdx.x * (kBlock / 32) + threadIdx.x / 32;
  const uint32_t lane = threadIdx.x & 31u;
  if (v >= V) return;  // uniform across the warp
  const DevParams& p = pp[b.vertexScene[v]];
  if (!p.active || !p.ipc) return;
  const uint2 r = b.contactRange[v];
  uint32_t n = 0;
  for (uint32_t k0 = 0; k0 < r.y; k0 += 32) {
    const uint32_t k = k0 + lane;
    const uint32_t c = k < r.y ? b.contactIds[r.x + k] : 0u;
    const bool keep = k < r.y && b.contactFlag[c] != 0u;
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    if (keep) b.activeIds[r.x + n + __popc(ballot & ((1u << lane) - 1u))] = c;
    n += __popc(ballot);
  }
  if (lane == 0) b.activeCount[v] = n;
}

// The IPC part of convergenceGradient's contact component (:4086-4088) at
// the accepted pose, one warp per vertex, from the contacts the promotion
// pass makes the next source cache.
__global__ void __launch_bounds__(kBlock) contactGradientKernel(Buffers b, const DevParams* __restrict__ pp,
                                                                const float4* __restrict__ src,
                                                                const float4* __restrict__ tgt, uint32_t V) {
  const uint32_t v = blockIdx.x * (kBlock / 32) + threadIdx.x / 32;
  const uint32_t lane = threadIdx.x & 31u;
  if (v >= V) return;  // uniform across the warp
  const uint32_t scene = b.vertexScene[v];
  const DevParams& p = pp[scene];
  const FrameState* fs = &b.frames[scene];
  if (!p.active || !p.ipc || latched(p, fs)) return;
  if (isPinned(b.vinfo[v])) return;
  const bool accepted = fs->control[1].x == 1.0f;
  const float alpha = fs->contactAlpha;
  const int slot = (accepted && finiteS(alpha) && alpha > 0.0f) ? kContactTarget : kContactSource;
  float3 g = f3(0, 0, 0);
  S3 unused = szero();
  contactLocal<false>(b, p, v, accepted ? tgt : src, false, slot, lane, 32u, g, unused);
  g.x = groupSum<32>(g.x, 0xffffffffu);
  g.y = groupSum<32>(g.y, 0xffffffffu);
  g.z = groupSum<32>(g.z, 0xffffffffu);
  if (lane == 0) b.contactGrad[v] = make_float4(g.x, g.y, g.z, 0.0f);
}

__device__ __forceinline__ uint32_t alphaBits(float a) { return a > 0.0f ? __float_as_uint(a) : 0u; }

// candidateContactStep of one candidate.
__device__ __forceinline__ void contactStepOne(const Buffers& b, const DevParams* __restrict__ pp,
                                               const float4* __restrict__ src, const float4* __restrict__ tgt,
                                               uint32_t c) {
  const uint32_t scene = b.contactScene[c];
  const DevParams& p = pp[scene];
  if (!p.active || !p.ipc) return;
  FrameState* fs = &b.frames[scene];
  float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
  if (latched(p, fs)) {
    st[kContactScratch] = make_float4(1, 0, 0, 1);
    return;  // alpha one, valid: the reduction's identity
  }
  uint32_t type;
  const uint4 q = contactIndices(b, c, &type);
  const float3 d0 = xyz(tgt[q.x]) - xyz(src[q.x]), d1 = xyz(tgt[q.y]) - xyz(src[q.y]);
  const float3 d2 = xyz(tgt[q.z]) - xyz(src[q.z]), d3 = xyz(tgt[q.w]) - xyz(src[q.w]);
  float L = 0.0f;
  if (type == kIpcVertexTriangle) L = length3(d0) + fmaxf(length3(d1), fmaxf(length3(d2), length3(d3)));
  else L = fmaxf(length3(d0), length3(d1)) + fmaxf(length3(d2), length3(d3));
  ContactData source = ipcCached(st[kContactSource], st[kContactSourceWeights]);
  bool fullStepSafe = source.valid && finiteS(L) && source.distance - L > p.ipcMinDistance;
  if (!fullStepSafe) {
    source = contactAt(b, c, src, kF32Max);
    fullStepSafe = source.valid && finiteS(L) && source.distance - L > p.ipcMinDistance;
  }
  const bool trialValid = finiteV(d0) && finiteV(d1) && finiteV(d2) && finiteV(d3);
  const bool valid = source.valid && trialValid && source.distance > p.ipcMinDistance && finiteS(L);
  float alpha = 0.0f;
  if (valid) alpha = fullStepSafe ? 1.0f : ipcSafeStepCap(source.distance, p.ipcMinDistance, L, p.ipcSafety);
  st[kContactScratch] = make_float4(alpha, source.valid ? source.distance : 0.0f,
                                    trialValid ? source.distance : 0.0f, valid ? 1.0f : 0.0f);
  if (valid && finiteS(alpha)) {
    if (alpha < 1.0f) atomicMin(&fs->stepAlphaBits, alphaBits(alpha));
  } else {
    atomicMin(&fs->stepAlphaBits, 0u);
    atomicAnd(&fs->stepValid, 0u);
  }
}

// candidateContactStep (:2784-2847) with the min / all-valid reduction of
// reduceContactStep folded in as order-free atomics.
__global__ void JGS2_CONTACT_BOUNDS contactStepKernel(Buffers b, const DevParams* __restrict__ pp,
                                                            const float4* __restrict__ src,
                                                            const float4* __restrict__ tgt) {
  const uint32_t n = contactListed(b);
  for (uint32_t c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock)
    contactStepOne(b, pp, src, tgt, c);
}

// applyContactStep (:2909-2917): candidate = source + alpha (candidate -
// source) with the safe-step alpha, or after validation with 1 (kept) or 0
// (restored); the validated alpha becomes the iteration's contact alpha.
__global__ void __launch_bounds__(kBlock) contactApplyKernel(Buffers b, const DevParams* __restrict__ pp,
                                                             const float4* __restrict__ src, float4* tgt,
                                                             uint32_t V, int validated) {
  const uint32_t v = blockIdx.x * kBlock + threadIdx.x;
  if (v >= V) return;
  const uint32_t scene = b.vertexScene[v];
  const DevParams& p = pp[scene];
  if (!p.active || !p.ipc) return;
  FrameState* fs = &b.frames[scene];
  const uint32_t bits = validated ? fs->checkAlphaBits : fs->stepAlphaBits;
  const uint32_t ok = validated ? fs->checkValid : fs->stepValid;
  const float alpha = ok ? clamp01f(__uint_as_float(bits)) : 0.0f;
  if (validated && v == b.scenes[scene].vOff) fs->contactAlpha = alpha;
  if (latched(p, fs)) return;
  const float3 s = xyz(src[v]);
  const float3 t = s + alpha * (xyz(tgt[v]) - s);
  tgt[v] = make_float4(t.x, t.y, t.z, 1.0f);
}

// validateContactStep (:2849-2868): exact contacts of the scaled candidate
// (the target cache) and the all-valid reduction.
__global__ void JGS2_CONTACT_BOUNDS contactValidateKernel(Buffers b, const DevParams* __restrict__ pp,
                                                                const float4* __restrict__ tgt) {
  const uint32_t n = contactListed(b);
  for (uint32_t c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock) {
    const uint32_t scene = b.contactScene[c];
    const DevParams& p = pp[scene];
    if (!p.active || !p.ipc) continue;
    FrameState* fs = &b.frames[scene];
    const ContactData k = contactAt(b, c, tgt, p.ipcActivation + contactRoundingReach(p));
    float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
    ipcStoreCached(st, kContactTarget, k);
    const bool valid = k.valid && finiteS(k.distance) && k.distance > p.ipcMinDistance;
    const float d = valid ? k.distance : 0.0f;
    st[kContactScratch] = make_float4(1.0f, d, d, valid ? 1.0f : 0.0f);
    if (!valid) {
      atomicMin(&fs->checkAlphaBits, 0u);
      atomicAnd(&fs->checkValid, 0u);
    }
  }
}

// Closest features of caller-given pairs (a diagnostic, not part of the
// step): the device routine every contact pass uses, f32 with the FP64 run
// for near-degenerate pairs; 9 floats per pair out (distance, normal,
// weights, valid) and whether the FP64 run was taken.
__global__ void __launch_bounds__(kBlock) contactFeatureKernel(const float* __restrict__ points,
                                                               const uint32_t* __restrict__ types, uint32_t n,
                                                               float* __restrict__ out, uint32_t* __restrict__ wide) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const float* x = points + 12ull * i;
  const float3 p0 = f3(x[0], x[1], x[2]), p1 = f3(x[3], x[4], x[5]);
  const float3 p2 = f3(x[6], x[7], x[8]), p3 = f3(x[9], x[10], x[11]);
  bool w = false;
  const ContactData k = types[i] == kIpcVertexTriangle ? ipcPointTriangle(p0, p1, p2, p3, &w)
                                                       : ipcEdgeEdge(p0, p1, p2, p3, &w);
  float* o = out + 9ull * i;
  o[0] = k.distance;
  o[1] = k.normal.x; o[2] = k.normal.y; o[3] = k.normal.z;
  o[4] = k.weights.x; o[5] = k.weights.y; o[6] = k.weights.z; o[7] = k.weights.w;
  o[8] = k.valid ? 1.0f : 0.0f;
  wide[i] = w ? 1u : 0u;
}

// promoteAcceptedContactCache (:2694-2710).
__global__ void __launch_bounds__(kBlock) contactPromoteKernel(Buffers b, const DevParams* __restrict__ pp) {
  const uint32_t n = contactListed(b);
  for (uint32_t c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock) {
    const uint32_t scene = b.contactScene[c];
    const DevParams& p = pp[scene];
    if (!p.active || !p.ipc) continue;
    const FrameState* fs = &b.frames[scene];
    const float alpha = fs->contactAlpha;
    if (fs->control[1].x == 1.0f && finiteS(alpha) && alpha > 0.0f) {
      float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
      st[kContactSource] = st[kContactTarget];
      st[kContactSourceWeights] = st[kContactTargetWeights];
    }
  }
}

// ---------------------------------------------------------------------------
// IPC broad phase over the static candidate superset (contact surfaces).
//
// The superset (buildStaticIpcContactCandidates, ipc-contact.ts:591-665) is
// never listed.  Every iteration one warp per row (a vertex against its
// scene's surface triangles, or a surface edge against the later edges)
// walks the row's columns in canonical order, 32-primitive chunk boxes
// first, and lists the pairs whose boxes, each widened by the largest motion
// its vertices can make this iteration, are not separated by more than the
// activation distance plus the rounding reach; pairs of the previous list
// that carry lagged friction stay listed for the frame.  A pair left out is
// farther than that from every pose the iteration can produce, so the
// reference's passes give it no active row, a full safe step, a valid check
// and no energy: it does not act.  A listed pair's state is carried from the
// previous list (the promoted source cache, the lagged friction) or formed
// from the source pose as lagContact does.  The per-vertex active rows come
// from a stable radix sort of the active candidates' vertex entries, so each
// row keeps ascending candidate order, as the static rows do.

constexpr uint32_t kBpChunk = 32;
constexpr uint32_t kBpClosedMax = 64;  // closed one-ring vertices a row keeps in shared memory
constexpr float kBpInf = __builtin_huge_valf();

struct BpBox {
  float3 lo, hi;
  float m;  // largest motion of the primitive's vertices this iteration
};

// A vertex's largest displacement in one iteration: maxStep for a free
// vertex (the line search caps each local step at maxStep, :3322-3445) and
// the snap to rest for a pinned one, widened by a relative 2^-12 and 16 ulps
// of the coordinates for the rounding of the committed positions.
__device__ __forceinline__ float bpMotion(const Buffers& b, const DevParams& p, uint32_t v, float3 x) {
  float m = fmaxf(p.maxStep, 0.0f);
  if (isPinned(b.vinfo[v])) m = fmaxf(m, length3(xyz(b.restMass[v]) - x));
  const float ax = fmaxf(fabsf(x.x), fmaxf(fabsf(x.y), fabsf(x.z)));
  const float r = m * (1.0f + 0x1p-12f) + ax * 0x1p-19f;
  return finiteS(r) ? r : kBpInf;
}

__device__ __forceinline__ BpBox bpEmpty() { return {f3(kBpInf, kBpInf, kBpInf), f3(-kBpInf, -kBpInf, -kBpInf), 0.0f}; }
__device__ __forceinline__ BpBox bpEverything() {
  return {f3(-kBpInf, -kBpInf, -kBpInf), f3(kBpInf, kBpInf, kBpInf), kBpInf};
}

// Bounds and largest motion of a primitive at x; non-finite data widens it
// to everything (such a pair is always listed, as the static path keeps it).
template <int N>
__device__ __forceinline__ BpBox bpPrimitive(const Buffers& b, const DevParams& p, const float4* __restrict__ x,
                                             const uint32_t (&vs)[N]) {
  BpBox q = bpEmpty();
  bool ok = true;
#pragma unroll
  for (int l = 0; l < N; ++l) {
    const float3 y = xyz(x[vs[l]]);
    ok = ok && finiteV(y);
    q.lo = fmin3(q.lo, y);
    q.hi = fmax3(q.hi, y);
    q.m = fmaxf(q.m, bpMotion(b, p, vs[l], y));
  }
  return (ok && finiteS(q.m)) ? q : bpEverything();
}

__device__ __forceinline__ void bpStore(float4* boxes, uint32_t i, const BpBox& q) {
  boxes[2ull * i] = make_float4(q.lo.x, q.lo.y, q.lo.z, q.m);
  boxes[2ull * i + 1] = make_float4(q.hi.x, q.hi.y, q.hi.z, 0.0f);
}
__device__ __forceinline__ BpBox bpLoad(const float4* __restrict__ boxes, uint32_t i) {
  const float4 a = boxes[2ull * i], c = boxes[2ull * i + 1];
  return {f3(a.x, a.y, a.z), f3(c.x, c.y, c.z), a.w};
}

// Separated by more than `reach` once both boxes are widened by their
// motions: the per-axis gaps less the motions, as a Euclidean length.  Each
// step is monotone in the boxes, so a chunk box that contains a primitive's
// box (and its motion) separates no more than the primitive's does.
__device__ __forceinline__ bool bpSeparated(const BpBox& a, const BpBox& c, float reach) {
  const float m = a.m + c.m;
  const float3 g = fmax3(fmax3(c.lo - a.hi, a.lo - c.hi), f3(0, 0, 0));
  const float3 h = fmax3(g - f3(m, m, m), f3(0, 0, 0));
  return dot3(h, h) > reach * reach;
}

// The activation distance and twice the rounding reach
// (ipcActiveContactReach less its step terms, which the motions carry),
// widened by 2^-10.
__device__ __forceinline__ float bpReach(const DevParams& p) {
  return (p.ipcActivation + 2.0f * contactRoundingReach(p)) * (1.0f + 0x1p-10f);
}

// closed(a, v) of the enumeration: a == v or v in a's surface one-ring.
__device__ __forceinline__ bool bpClosed(const Buffers& b, uint32_t a, uint32_t v) {
  if (a == v) return true;
  const uint2 r = b.bpRing[a];
  for (uint32_t i = 0; i < r.y; ++i)
    if (b.bpRingIds[r.x + i] == v) return true;
  return false;
}

// The superset leaves out a vertex and a triangle of its closed one-ring,
// and two edges with an endpoint of one in the other's closed one-rings.
__device__ __forceinline__ bool bpPairClosed(const Buffers& b, bool edgeRow, const uint32_t (&rv)[2], uint32_t col) {
  if (!edgeRow) {
    const uint4 t = b.bpTris[col];
    return bpClosed(b, rv[0], t.x) || bpClosed(b, rv[0], t.y) || bpClosed(b, rv[0], t.z);
  }
  const uint2 e = b.bpEdges[col];
  return bpClosed(b, rv[0], e.x) || bpClosed(b, rv[0], e.y) || bpClosed(b, rv[1], e.x) || bpClosed(b, rv[1], e.y);
}

// Primitive and chunk boxes at the iteration's source pose (a warp's 32
// primitives form one chunk), and the reset of every vertex's active row.
__global__ void __launch_bounds__(kBlock) bpBoxesKernel(Buffers b, const DevParams* __restrict__ pp,
                                                        const float4* __restrict__ src, uint32_t triBlocks,
                                                        uint32_t edgeBlocks, uint32_t V) {
  const uint32_t blk = blockIdx.x;
  if (blk < triBlocks + edgeBlocks) {
    const bool edges = blk >= triBlocks;
    const uint32_t i = (edges ? blk - triBlocks : blk) * kBlock + threadIdx.x;
    const uint32_t n = edges ? b.bpEdgeTotal : b.bpTriTotal;
    BpBox q = bpEmpty();
    if (i < n) {
      if (edges) {
        const uint2 e = b.bpEdges[i];
        const uint32_t vs[2] = {e.x, e.y};
        q = bpPrimitive(b, pp[b.vertexScene[e.x]], src, vs);
        bpStore(b.bpEdgeBox, i, q);
      } else {
        const uint4 t = b.bpTris[i];
        const uint32_t vs[3] = {t.x, t.y, t.z};
        q = bpPrimitive(b, pp[t.w], src, vs);
        bpStore(b.bpTriBox, i, q);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      q.lo.x = fminf(q.lo.x, __shfl_xor_sync(0xffffffffu, q.lo.x, o));
      q.lo.y = fminf(q.lo.y, __shfl_xor_sync(0xffffffffu, q.lo.y, o));
      q.lo.z = fminf(q.lo.z, __shfl_xor_sync(0xffffffffu, q.lo.z, o));
      q.hi.x = fmaxf(q.hi.x, __shfl_xor_sync(0xffffffffu, q.hi.x, o));
      q.hi.y = fmaxf(q.hi.y, __shfl_xor_sync(0xffffffffu, q.hi.y, o));
      q.hi.z = fmaxf(q.hi.z, __shfl_xor_sync(0xffffffffu, q.hi.z, o));
      q.m = fmaxf(q.m, __shfl_xor_sync(0xffffffffu, q.m, o));
    }
    if ((threadIdx.x & 31u) == 0u && i < n) bpStore(edges ? b.bpEdgeChunk : b.bpTriChunk, i / kBpChunk, q);
    return;
  }
  const uint32_t v = (blk - triBlocks - edgeBlocks) * kBlock + threadIdx.x;
  if (v >= V) return;
  b.activeCount[v] = 0u;
  // ipcCandidatePinnedMotionExceedsBound per vertex (contactPinnedMotion).
  uint32_t move = 0u;
  if (isPinned(b.vinfo[v])) {
    const DevParams& p = pp[b.vertexScene[v]];
    const float3 d = xyz(b.restMass[v]) - xyz(src[v]);
    const float len = length3(d);
    move = (!finiteV(d) || !finiteS(len) || len > fmaxf(p.maxStep, 0.0f)) ? 1u : 0u;
  }
  b.bpPinnedMove[v] = move;
}

// Superchunk boxes: one warp per 32 chunks (the union of their boxes).
__global__ void __launch_bounds__(kBlock) bpSuperKernel(Buffers b, uint32_t triSupers, uint32_t edgeSupers) {
  const uint32_t w = blockIdx.x * (kBlock / 32) + threadIdx.x / 32, lane = threadIdx.x & 31u;
  if (w >= triSupers + edgeSupers) return;  // uniform across the warp
  const bool edges = w >= triSupers;
  const uint32_t sc = edges ? w - triSupers : w;
  const uint32_t chunks = ((edges ? b.bpEdgeTotal : b.bpTriTotal) + kBpChunk - 1) / kBpChunk;
  const uint32_t chunk = sc * kBpChunk + lane;
  BpBox q = chunk < chunks ? bpLoad(edges ? b.bpEdgeChunk : b.bpTriChunk, chunk) : bpEmpty();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    q.lo.x = fminf(q.lo.x, __shfl_xor_sync(0xffffffffu, q.lo.x, o));
    q.lo.y = fminf(q.lo.y, __shfl_xor_sync(0xffffffffu, q.lo.y, o));
    q.lo.z = fminf(q.lo.z, __shfl_xor_sync(0xffffffffu, q.lo.z, o));
    q.hi.x = fmaxf(q.hi.x, __shfl_xor_sync(0xffffffffu, q.hi.x, o));
    q.hi.y = fmaxf(q.hi.y, __shfl_xor_sync(0xffffffffu, q.hi.y, o));
    q.hi.z = fmaxf(q.hi.z, __shfl_xor_sync(0xffffffffu, q.hi.z, o));
    q.m = fmaxf(q.m, __shfl_xor_sync(0xffffffffu, q.m, o));
  }
  if (lane == 0) bpStore(edges ? b.bpEdgeSuper : b.bpTriSuper, sc, q);
}

// A listed pair's state: carried from the previous list (its entry
// `bpPrev`), else the source contact and, at the frame's first iteration, its
// lagged force as lagContact (:2712-2740) forms them; its activity
// (contactIncluded) and its four sort entries (vertex, candidate), whose key
// is the sentinel when the pair is inactive.  One thread per candidate.
__global__ void JGS2_CONTACT_BOUNDS bpInitKernel(Buffers b, const DevParams* __restrict__ pp,
                                                       const float4* __restrict__ src, int first) {
  const uint32_t n = __ldcg(b.bpStatus);
  for (uint32_t c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock) {
    const DevParams& p = pp[b.contactScene[c]];
    uint32_t type;
    const uint4 q = contactIndices(b, c, &type);
    float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
    float4 lagF = make_float4(0, 0, 0, 0), lagW = make_float4(0, 0, 0, 0);
    const uint32_t prev = first ? 0xffffffffu : b.bpPrev[c];
    float4 s0, s1;
    if (prev != 0xffffffffu) {
      const float4* ps = b.bpPrevState + kContactStateWords * static_cast<size_t>(prev);
      s0 = ps[kContactSource];
      s1 = ps[kContactSourceWeights];
      lagF = ps[kContactLagged];
      lagW = ps[kContactLaggedWeights];
      st[kContactSource] = s0;
      st[kContactSourceWeights] = s1;
    } else {
      const ContactData k = ipcContactFromPositions(type, xyz(src[q.x]), xyz(src[q.y]), xyz(src[q.z]), xyz(src[q.w]),
                                                    p.ipcActivation + contactRoundingReach(p));
      ipcStoreCached(st, kContactSource, k);
      s0 = st[kContactSource];
      s1 = st[kContactSourceWeights];
      if (first && k.valid && k.distance > p.ipcMinDistance) {
        const float f = fmaxf(0.0f, -p.ipcStiffness * ipcBarrier1(k.distance, p.ipcActivation));
        if (finiteS(f)) {
          lagF = make_float4(k.normal.x, k.normal.y, k.normal.z, f);
          lagW = k.weights;
        }
      }
    }
    st[kContactLagged] = lagF;
    st[kContactLaggedWeights] = lagW;
    st[kContactScratch] = make_float4(1, 0, 0, 0);
    // contactIncluded on the state just written.
    const ContactData k = ipcCached(s0, s1);
    const bool friction = p.ipcFriction > 0.0f && lagF.w > 0.0f;
    const bool bounded = p.maxStep > 0.0f;
    const float reach = p.ipcActivation + 2.0f * (fmaxf(p.maxStep, 0.0f) + contactRoundingReach(p));
    const bool pinnedMove =
        (b.bpPinnedMove[q.x] | b.bpPinnedMove[q.y] | b.bpPinnedMove[q.z] | b.bpPinnedMove[q.w]) != 0u;
    const bool active = !k.valid || !bounded || k.distance <= reach || friction || pinnedMove;
    b.contactFlag[c] = active ? 1u : 0u;
    const uint32_t key = b.bpSentinel;
    reinterpret_cast<uint4*>(b.bpKeys[0])[c] =
        active ? make_uint4(q.x, q.y, q.z, q.w) : make_uint4(key, key, key, key);
    reinterpret_cast<uint4*>(b.bpVals[0])[c] = make_uint4(c, c, c, c);
  }
}

// One warp per row: the row's pairs in column order, counted (kWrite false,
// into bpRowOff[row]) or placed at the row's offset with their previous
// entry (kWrite true).  The columns are walked 32 superchunks (of 32 chunks
// of 32 primitives) at a time, then 32 chunks, then 32 primitives, each
// level only inside the boxes the row's box does not clear.
template <bool kWrite>
__global__ void __launch_bounds__(kBlock) bpRowsKernel(Buffers b, const DevParams* __restrict__ pp,
                                                       const float4* __restrict__ src, int first) {
  __shared__ uint32_t carried[kBlock / 32][32];
  __shared__ uint32_t closedSet[kBlock / 32][kBpClosedMax];
  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x & 31u;
  const uint32_t r = blockIdx.x * (kBlock / 32) + warp;
  if (r >= b.bpRowTotal) return;                   // uniform across the warp
  if (kWrite && __ldcg(&b.bpStatus[3])) return;   // over capacity: nothing listed this iteration
  const uint4 row = b.bpRows[r];
  const uint32_t scene = row.y & 0x7fffffffu;
  const bool edgeRow = (row.y >> 31) != 0u;
  const DevParams& p = pp[scene];
  uint32_t count = 0;
  if (p.active && p.ipc && row.z < row.w) {
    const float reach = bpReach(p);
    uint32_t rv[2];
    BpBox P;
    if (edgeRow) {
      const uint2 e = b.bpEdges[row.x];
      rv[0] = e.x;
      rv[1] = e.y;
      P = bpLoad(b.bpEdgeBox, row.x);
    } else {
      rv[0] = rv[1] = row.x;
      const uint32_t vs[1] = {row.x};
      P = bpPrimitive(b, p, src, vs);
    }
    // The row's closed one-ring set: a pair whose other vertices meet it is
    // not in the superset (more than kBpClosedMax vertices: the ring lists).
    uint32_t nClosed = 0;
    {
      const uint2 r0 = b.bpRing[rv[0]];
      const uint2 r1 = edgeRow ? b.bpRing[rv[1]] : make_uint2(0u, 0u);
      nClosed = (edgeRow ? 2u : 1u) + r0.y + r1.y;
      if (nClosed <= kBpClosedMax) {
        for (uint32_t i = lane; i < nClosed; i += 32) {
          uint32_t v;
          if (i == 0) v = rv[0];
          else if (i <= r0.y) v = b.bpRingIds[r0.x + i - 1];
          else if (i == r0.y + 1) v = rv[1];
          else v = b.bpRingIds[r1.x + i - r0.y - 2];
          closedSet[warp][i] = v;
        }
      }
      __syncwarp();
    }
    auto closed = [&](uint32_t col) {
      if (nClosed > kBpClosedMax) return bpPairClosed(b, edgeRow, rv, col);
      uint32_t q0, q1, q2;
      if (edgeRow) {
        const uint2 e = b.bpEdges[col];
        q0 = e.x;
        q1 = q2 = e.y;
      } else {
        const uint4 t = b.bpTris[col];
        q0 = t.x;
        q1 = t.y;
        q2 = t.z;
      }
      for (uint32_t i = 0; i < nClosed; ++i) {
        const uint32_t v = closedSet[warp][i];
        if (v == q0 || v == q1 || v == q2) return true;
      }
      return false;
    };
    const uint32_t base = kWrite ? b.bpRowOff[r] : 0u;
    uint32_t pc = 0, pe = 0;  // this row's entries of the previous list
    if (!first) {
      pc = b.bpPrevRowOff[r];
      pe = b.bpPrevRowOff[r + 1];
    }
    uint32_t qc = pc;  // carry cursor: first previous entry at or past the current chunk
    const uint32_t chunkLo = row.z / kBpChunk, chunkHi = (row.w - 1) / kBpChunk;
    const float4* superBoxes = edgeRow ? b.bpEdgeSuper : b.bpTriSuper;
    const float4* chunkBoxes = edgeRow ? b.bpEdgeChunk : b.bpTriChunk;
    const float4* primBoxes = edgeRow ? b.bpEdgeBox : b.bpTriBox;
    // Rows whose previous entries carry no lagged friction skip whole
    // superchunks whose box the row's box clears.
    bool friction = false;
    if (!first && p.ipcFriction > 0.0f)
      for (uint32_t i0 = pc; i0 < pe && !friction; i0 += 32) {
        const uint32_t i = i0 + lane;
        friction = __any_sync(0xffffffffu,
                              i < pe && b.bpPrevState[kContactStateWords * static_cast<size_t>(i) + kContactLagged].w >
                                            0.0f);
      }
    const uint32_t superLo = chunkLo / kBpChunk, superHi = chunkHi / kBpChunk;
    for (uint32_t s0 = superLo; s0 <= superHi; s0 += 32) {
      const uint32_t sc = s0 + lane;
      unsigned superTodo = __ballot_sync(0xffffffffu, sc <= superHi && (friction || !bpSeparated(
                                                                                     P, bpLoad(superBoxes, sc), reach)));
      while (superTodo) {
        const uint32_t c0 = (s0 + __ffs(superTodo) - 1) * kBpChunk;  // the superchunk's first chunk
        superTodo &= superTodo - 1;
        const uint32_t windowEnd = (c0 + 32) * kBpChunk;
        carried[warp][lane] = 0u;
        __syncwarp();
        // Previous pairs of this window that carry lagged friction and that
        // the box test leaves out stay listed.
        while (friction && pc < pe) {
          const uint32_t i = pc + lane;
          const uint32_t col = i < pe ? b.bpPrevCols[i] : 0xffffffffu;
          const bool in = i < pe && col < windowEnd;
          if (in && b.bpPrevState[kContactStateWords * static_cast<size_t>(i) + kContactLagged].w > 0.0f &&
              bpSeparated(P, bpLoad(primBoxes, col), reach))
            atomicOr(&carried[warp][col / kBpChunk - c0], 1u << (col % kBpChunk));
          const unsigned inMask = __ballot_sync(0xffffffffu, in);
          pc += __popc(inMask);
          if (inMask != 0xffffffffu) break;
        }
        __syncwarp();
        const uint32_t chunk = c0 + lane;
        const bool look = chunk >= chunkLo && chunk <= chunkHi &&
                          (carried[warp][lane] != 0u || !bpSeparated(P, bpLoad(chunkBoxes, chunk), reach));
        unsigned todo = __ballot_sync(0xffffffffu, look);
        while (todo) {
          const uint32_t j = __ffs(todo) - 1;
          todo &= todo - 1;
          const uint32_t col = (c0 + j) * kBpChunk + lane;
          bool hit = false;
          if (col >= row.z && col < row.w) {
            hit = ((carried[warp][j] >> lane) & 1u) != 0u;
            if (!hit && !bpSeparated(P, bpLoad(primBoxes, col), reach)) hit = !closed(col);
          }
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (kWrite && m) {
            // The previous list's entries of this chunk (sorted, at most 32):
            // a bit per column, so a listed pair finds its entry by rank.
            uint32_t prev = 0xffffffffu;
            if (!first) {
              const uint32_t chunkStart = (c0 + j) * kBpChunk;
              while (qc < pe) {
                const uint32_t i = qc + lane;
                const unsigned below = __ballot_sync(0xffffffffu, i < pe && b.bpPrevCols[i] < chunkStart);
                qc += __popc(below);
                if (below != 0xffffffffu) break;
              }
              const uint32_t i = qc + lane;
              const uint32_t pcol = i < pe ? b.bpPrevCols[i] : 0xffffffffu;
              const uint32_t off = pcol - chunkStart;
              const unsigned have = __reduce_or_sync(0xffffffffu, off < kBpChunk ? (1u << off) : 0u);
              if ((have >> lane) & 1u) prev = qc + __popc(have & ((1u << lane) - 1u));
            }
            if (hit) {
              const uint32_t pos = base + count + __popc(m & ((1u << lane) - 1u));
              uint4 q;
              if (edgeRow) {
                const uint2 e = b.bpEdges[col];
                q = make_uint4(rv[0], rv[1], e.x, e.y | 0x80000000u);
              } else {
                const uint4 t = b.bpTris[col];
                q = make_uint4(rv[0], t.x, t.y, t.z);
              }
              b.contactIdx[pos] = q;
              b.contactScene[pos] = scene;
              b.bpCols[pos] = col;
              b.bpPrev[pos] = prev;
            }
          }
          count += __popc(m);
        }
        __syncwarp();  // carried[] is rewritten by the next window
      }
    }
  }
  if (!kWrite && lane == 0) b.bpRowOff[r] = count;
}

constexpr int kScanThreads = 1024;

// Exclusive scan of data[0, n) in place by one block of kScanThreads threads
// (a contiguous run per thread); returns the total.  With the total above
// `limit` every entry becomes zero.
__device__ uint64_t blockScan(uint32_t* data, uint32_t n, uint64_t limit) {
  __shared__ uint64_t part[kScanThreads];
  const uint32_t per = (n + kScanThreads - 1) / kScanThreads;
  const uint32_t lo = min(n, threadIdx.x * per), hi = min(n, lo + per);
  uint64_t s = 0;
  for (uint32_t i = lo; i < hi; ++i) s += data[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (uint32_t o = 1; o < kScanThreads; o <<= 1) {
    const uint64_t add = threadIdx.x >= o ? part[threadIdx.x - o] : 0ull;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  const uint64_t total = part[kScanThreads - 1];
  const bool over = total > limit;
  uint64_t run = part[threadIdx.x] - s;
  for (uint32_t i = lo; i < hi; ++i) {
    const uint32_t c = data[i];
    data[i] = over ? 0u : static_cast<uint32_t>(run);
    run += c;
  }
  __syncthreads();
  return total;
}

// Row offsets, the list's size (zero, with the overflow flags set, when it
// exceeds the capacity), each scene's span of the list, and the resets the
// static path makes in its flag and lag passes: the safe-step reductions
// every iteration, the contact alpha at the frame's first.
__global__ void __launch_bounds__(kScanThreads) bpScanKernel(Buffers b, const DevParams* __restrict__ pp,
                                                             int first) {
  const uint32_t R = b.bpRowTotal;
  const uint64_t total = blockScan(b.bpRowOff, R, b.contactCount);
  const bool over = total > b.contactCount;
  if (threadIdx.x == 0) {
    b.bpRowOff[R] = over ? 0u : static_cast<uint32_t>(total);
    b.bpStatus[0] = over ? 0u : static_cast<uint32_t>(total);
    b.bpStatus[3] = over ? 1u : 0u;
    if (over) {
      b.bpStatus[1] = 1u;
      b.bpStatus[2] = max(b.bpStatus[2], static_cast<uint32_t>(total > 0xffffffffull ? 0xffffffffull : total));
    }
  }
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < b.sceneCount; s += blockDim.x) {
    const SceneRange sr = b.scenes[s];
    uint2 span = make_uint2(0u, 0u);
    if (sr.rowCount) {
      const uint32_t a = b.bpRowOff[sr.rowOff], e = b.bpRowOff[sr.rowOff + sr.rowCount];
      span = make_uint2(a, e - a);
    }
    b.bpSpan[s] = span;
    const DevParams& p = pp[s];
    if (!p.active || !p.ipc) continue;
    FrameState* fs = &b.frames[s];
    fs->stepAlphaBits = __float_as_uint(1.0f);
    fs->stepValid = 1u;
    fs->checkAlphaBits = __float_as_uint(1.0f);
    fs->checkValid = 1u;
    if (first) fs->contactAlpha = 1.0f;
  }
}

// Stable LSD radix sort of the (vertex, candidate) entries, 8 bits a pass:
// per 4096-entry tile a digit histogram, one scan of the histograms in
// digit-major order, then a scatter in which each warp ranks its entries in
// input order (match_any peers) so equal digits keep their order.
constexpr uint32_t kSortThreads = 256, kSortItems = 16, kSortTile = kSortThreads * kSortItems;

__device__ __forceinline__ uint32_t sortTiles(const uint32_t* status) {
  return (4u * __ldcg(status) + kSortTile - 1) / kSortTile;
}

__global__ void __launch_bounds__(kSortThreads) bpSortHistKernel(const uint32_t* __restrict__ keys,
                                                                 const uint32_t* status, uint32_t shift,
                                                                 uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  const uint32_t M = 4u * __ldcg(status), tiles = sortTiles(status);
  if (blockIdx.x >= tiles) return;
  h[threadIdx.x] = 0u;
  __syncthreads();
#pragma unroll
  for (uint32_t j = 0; j < kSortItems; ++j) {
    const uint32_t i = blockIdx.x * kSortTile + j * kSortThreads + threadIdx.x;
    if (i < M) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// One block per digit: the exclusive scan of the digit's tile counts and the
// digit's total (after the 256 x tiles histogram).
__global__ void __launch_bounds__(kScanThreads) bpSortScanKernel(const uint32_t* status, uint32_t* hist) {
  const uint32_t tiles = sortTiles(status);
  const uint64_t total = blockScan(hist + static_cast<size_t>(blockIdx.x) * tiles, tiles, ~0ull);
  if (threadIdx.x == 0) hist[256u * tiles + blockIdx.x] = static_cast<uint32_t>(total);
}

__global__ void __launch_bounds__(kSortThreads) bpSortScatterKernel(const uint32_t* __restrict__ kin,
                                                                    const uint32_t* __restrict__ vin,
                                                                    uint32_t* __restrict__ kout,
                                                                    uint32_t* __restrict__ vout,
                                                                    const uint32_t* status, uint32_t shift,
                                                                    const uint32_t* __restrict__ hist) {
  __shared__ uint32_t wh[kSortThreads / 32][256];
  __shared__ uint32_t digitBase[256];
  const uint32_t M = 4u * __ldcg(status), tiles = sortTiles(status);
  const uint32_t tile = blockIdx.x;
  if (tile >= tiles) return;
  const uint32_t w = threadIdx.x / 32, lane = threadIdx.x & 31u;
  for (uint32_t d = threadIdx.x; d < 256u * (kSortThreads / 32); d += kSortThreads) (&wh[0][0])[d] = 0u;
  // Exclusive prefix of the digit totals (one digit per thread).
  digitBase[threadIdx.x] = hist[256u * tiles + threadIdx.x];
  __syncthreads();
  for (uint32_t o = 1; o < 256u; o <<= 1) {
    const uint32_t add = threadIdx.x >= o ? digitBase[threadIdx.x - o] : 0u;
    __syncthreads();
    digitBase[threadIdx.x] += add;
    __syncthreads();
  }
  const uint32_t mine = digitBase[threadIdx.x] - hist[256u * tiles + threadIdx.x];
  __syncthreads();
  digitBase[threadIdx.x] = mine;
  __syncthreads();
  const uint32_t base = tile * kSortTile + w * (kSortItems * 32);
  uint32_t dig[kSortItems], pos[kSortItems];
#pragma unroll
  for (uint32_t j = 0; j < kSortItems; ++j) {
    const uint32_t i = base + j * 32 + lane;
    const bool valid = i < M;
    const uint32_t d = valid ? (kin[i] >> shift) & 255u : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    const uint32_t before = valid ? wh[w][d] : 0u;
    __syncwarp();
    if (valid && rank == 0) wh[w][d] = before + __popc(peers);
    __syncwarp();
    dig[j] = d;
    pos[j] = before + rank;
  }
  __syncthreads();
  {
    const uint32_t d = threadIdx.x;  // one digit per thread
    uint32_t run = 0;
#pragma unroll
    for (uint32_t ww = 0; ww < kSortThreads / 32; ++ww) {
      const uint32_t t = wh[ww][d];
      wh[ww][d] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (uint32_t j = 0; j < kSortItems; ++j) {
    if (dig[j] < 256u) {
      const uint32_t i = base + j * 32 + lane;
      const uint32_t o = digitBase[dig[j]] + hist[dig[j] * tiles + tile] + wh[w][dig[j]] + pos[j];
      kout[o] = kin[i];
      vout[o] = vin[i];
    }
  }
}

// Each vertex's run of the sorted keys is its active row.
__global__ void __launch_bounds__(kBlock) bpSegmentsKernel(Buffers b, const uint32_t* __restrict__ keys) {
  const uint32_t M = 4u * __ldcg(b.bpStatus);
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < M; i += gridDim.x * kBlock) {
    const uint32_t k = keys[i];
    if (k >= b.bpSentinel || (i > 0 && keys[i - 1] == k)) continue;
    uint32_t lo = i + 1, hi = M;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (keys[mid] <= k) lo = mid + 1;
      else hi = mid;
    }
    b.contactRange[k] = make_uint2(i, 0u);
    b.activeCount[k] = lo - i;
  }
}

// ---------------------------------------------------------------------------
// The per-vertex JGS2 local solve, stable Neo-Hookean path
// (jgs2Solve, jgs2-shader.ts:2991-3473).  W lanes cooperate on one vertex:
// item u < K is cubature record u, item u >= K is incident tet u - K; lane j
// takes items j, j + W, ...  Cubature record state is cached in shared memory
// for the line search; incident deformation gradients are recomputed per
// trial from L1-resident data.
struct CubState {
  M3 F;
  float I0, J0;
  M3 dF0, dF1, dF2;
  float3 gQ;
  S3 HQ;
  float w, vol, lambda, mu;
  uint32_t slot;
  float3 gs;
};
static_assert(sizeof(CubState) <= kRecFloats * 4, "cubature cache record too small");

#ifndef JGS2_SOLVE_STAGE
#define JGS2_SOLVE_STAGE 1
#endif
// Shared-memory slot of one cubature record of a solve block.  The block
// first stages every record's header, basis blocks and tetrahedron record
// into its slot with asynchronous copies (all independent, so the whole
// block's input is in flight at once instead of one dependent chain per
// record and lane); the lane that owns the record then reads its inputs from
// the slot and overwrites the slot with the record's cached state for the
// line search.
struct RecSlot {
  uint4 head[2];   // (tet, weight bits, 0, 0), the tet's vertex indices
  float4 basis[9]; // 36 floats: four row-major 3x3 blocks
  float4 tet[4];   // [g1 vol] [g2 lambda] [g3 mu] [indices]
};
static_assert(sizeof(CubState) <= sizeof(RecSlot), "record state must fit its staging slot");
// Records per vertex up to this many bytes of cached state are cached in
// shared memory (K <= 68 with staging); wider ones are recomputed per trial.
#ifndef JGS2_SOLVE_CACHE_BYTES
#define JGS2_SOLVE_CACHE_BYTES 16384
#endif
constexpr size_t kSolveCacheBytesPerVertex = JGS2_SOLVE_CACHE_BYTES;
#if JGS2_SOLVE_STAGE
constexpr size_t kSolveSlotBytes = sizeof(RecSlot);
#else
constexpr size_t kSolveSlotBytes = sizeof(CubState);
#endif

__device__ __forceinline__ void cpAsync16(void* smem, const void* gmem) {
  const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpAsyncWaitAll() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ TetRec tetFromSlot(const float4* q) {
  const float4 a = q[0], b = q[1], c = q[2];
  const float4 d = q[3];
  TetRec r;
  r.g1 = f3(a.x, a.y, a.z);
  r.g2 = f3(b.x, b.y, b.z);
  r.g3 = f3(c.x, c.y, c.z);
  r.vol = a.w;
  r.lambda = b.w;
  r.mu = c.w;
  r.idx = make_uint4(__float_as_uint(d.x), __float_as_uint(d.y), __float_as_uint(d.z), __float_as_uint(d.w));
  return r;
}
// loadBlockVec from a shared-memory copy of the record's basis.
__device__ __forceinline__ M3 loadBlockVecShared(const float4* rec, int l) {
  const int k0 = (9 * l) >> 2;
  const int off = 9 * l - 4 * k0;
  const float4 a = rec[k0], b = rec[k0 + 1], c = rec[k0 + 2];
  const float f[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
  return {f3(f[off + 0], f[off + 3], f[off + 6]), f3(f[off + 1], f[off + 4], f[off + 7]),
          f3(f[off + 2], f[off + 5], f[off + 8])};
}

#ifndef JGS2_SOLVE_MIN_BLOCKS
#define JGS2_SOLVE_MIN_BLOCKS 4
#endif

// kExt: some scene of the engine has cloth or contact candidates (their
// gathers and line search terms are compiled out otherwise).
// State of cubature record `rec` of vertex v (jgs2-shader.ts:3197-3263), all
// in the source vertex's frame: the record tet's deformation gradient F and
// its invariants, the projected directions dF_c = sum_l B'_l[:,c] g_l^T with
// B'_l = R_l Ubar_l, the inertia / objective quadratic (gQ, HQ), the weight,
// the tet's material and, when v is one of the tet's vertices, its slot and
// shape gradient.  Read from the block's staged slot or from global memory;
// st.w = 0 for an empty record.  `r` receives the record's tet.
template <bool kCoherent, bool kStaged>
__device__ __forceinline__ void recordState(const Buffers& b, const DevParams& p, uint32_t v, size_t rec,
                                            const RecSlot* staged, const float4* __restrict__ src, bool objActive,
                                            CubState& st, TetRec& r) {
  uint4 head, idx;
  if constexpr (kStaged) {
    head = staged->head[0];
    idx = staged->head[1];
  } else {
    head = __ldg(&b.cubHead[2 * rec]);
    idx = __ldg(&b.cubHead[2 * rec + 1]);
  }
  const uint32_t t = head.x;
  const float w = __uint_as_float(head.y);
  st.w = 0.0f;
  // Headers hold global tet ids; out-of-range records were emptied at create.
  if (!(t != kEmptyTet && w > 0.0f)) return;
  if (!inBounds(t, b.tetTotal, kSiteRecordTet) || !inBounds(idx.x, b.vertexTotal, kSiteRecordVertex) ||
      !inBounds(idx.y, b.vertexTotal, kSiteRecordVertex) || !inBounds(idx.z, b.vertexTotal, kSiteRecordVertex) ||
      !inBounds(idx.w, b.vertexTotal, kSiteRecordVertex))
    return;
  const float4* U;
  if constexpr (kStaged) {
    r = tetFromSlot(staged->tet);
    U = staged->basis;
  } else {
    r = loadTet(b.tets, t);
    U = b.cubBasis + 9ull * rec;
  }
  M3 F = mzero(), dF0 = mzero(), dF1 = mzero(), dF2 = mzero();
  float3 gQ = f3(0, 0, 0);
  S3 HQ = szero();
  uint32_t slot = 4;
  const float3 x0 = xyz(ldPos<kCoherent>(src, idx.x));
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const uint32_t q = idxAt(idx, l);
    if (q == v) slot = l;
    const float3 gl = shapeGradient(r, l);
    M3 B;
    if constexpr (kStaged) B = mm(loadRotT<kCoherent>(b.vertexRot, q), loadBlockVecShared(U, l));
    else B = mm(loadRotT<kCoherent>(b.vertexRot, q), loadBlockVec(U, l));
    const float3 xl = l == 0 ? x0 : xyz(ldPos<kCoherent>(src, q));
    if (l > 0) F = F + outer(xl - x0, gl);
    dF0 = dF0 + outer(B.c0, gl);
    dF1 = dF1 + outer(B.c1, gl);
    dF2 = dF2 + outer(B.c2, gl);
    // predicted w = distributed inertia weight (0 when pinned).
    const float4 pq = b.predicted[q];
    const float dW = pq.w;
    float3 lin = dW * (xl - xyz(pq));
    float quad = dW;
    const uint4 qi = objActive ? b.vinfo[q] : make_uint4(0u, 0u, 1u, 0u);
    if (objActive && !isPinned(qi)) {
      const float nq = float(qi.y > 1u ? qi.y : 1u);
      lin = lin + objectiveGradient(p, b, q, xl) * (1.0f / nq);
      quad += targetStiffness(p, b, q) / nq;
    }
    gQ = gQ + mtv(B, lin);
    saddScaled(HQ, quad, gramColumns(B));
  }
  st.F = F;
  st.I0 = frob(F, F);
  st.J0 = mdet(F);
  st.dF0 = dF0; st.dF1 = dF1; st.dF2 = dF2;
  st.gQ = gQ;
  st.HQ = HQ;
  st.w = w;
  st.vol = r.vol; st.lambda = r.lambda; st.mu = r.mu;
  st.slot = slot;
  st.gs = slot < 4 ? shapeGradient(r, slot) : f3(0, 0, 0);
}

// One block's chunk `chunk` of the vertex list: vertices
// [chunk * groupsPerBlock, (chunk + 1) * groupsPerBlock) of `list` (or of all
// vertices).  Every thread of the block calls it with the same chunk.
template <int W, bool kExt, bool kCoherent = false, bool kCache = true>
__device__ __forceinline__ void solveChunk(const Buffers& b, const DevParams* __restrict__ pp,
                                           const float4* __restrict__ src, float4* tgt,
                                           const uint32_t* __restrict__ list, uint32_t count, uint32_t K,
                                           int cachedIncident, uint32_t groupsPerBlock, uint32_t chunk) {
  extern __shared__ float4 cache4[];
  unsigned char* slotBase = reinterpret_cast<unsigned char*>(cache4);
  __shared__ uint32_t sFail, sMaxBack, sSkip, sEvals, sMaxShift, sValid, sScene;
  // Lane groups never straddle a warp: warp w holds groups w * (32 / W) ...;
  // lanes past the warp's last whole group, or past groupsPerBlock, are idle.
  constexpr uint32_t kGroupsPerWarp = 32 / W;
  const uint32_t lane = (threadIdx.x & 31u) % W;
  const uint32_t groupInWarp = (threadIdx.x & 31u) / W;
  const uint32_t group = (threadIdx.x >> 5) * kGroupsPerWarp + groupInWarp;
  const bool groupLane = groupInWarp < kGroupsPerWarp && group < groupsPerBlock;
  const unsigned mask = W == 32 ? 0xffffffffu : (((1u << W) - 1u) << (groupInWarp * W));
  if (threadIdx.x == 0) {
    sFail = 0; sMaxBack = 0; sSkip = 0; sEvals = 0; sMaxShift = 0; sValid = 1;
    const uint32_t first = chunk * groupsPerBlock;
    sScene = b.vertexScene[list ? list[first] : first];
  }
  __syncthreads();
#if JGS2_SOLVE_STAGE
  if constexpr (kCache) {
    // Stage the block's records: headers and basis blocks, then (once the
    // headers have landed) the tetrahedron records they name.
    RecSlot* slots = reinterpret_cast<RecSlot*>(slotBase);
    const uint32_t nrec = groupsPerBlock * K;
    // Sixteen-byte chunks in address order: a record's two header chunks and
    // nine basis chunks are consecutive, so a warp's copies are coalesced.
    for (uint32_t c = threadIdx.x; c < nrec * 11u; c += blockDim.x) {
      const uint32_t r = c / 11u, part = c - r * 11u;
      const uint32_t g = r / K, it = chunk * groupsPerBlock + g;
      if (it >= count) continue;
      const uint32_t sv = list ? list[it] : it;
      if (!inBounds(sv, b.vertexTotal, kSiteListVertex)) continue;
      const size_t rec = static_cast<size_t>(sv) * K + (r - g * K);
      if (part < 2u) cpAsync16(&slots[r].head[part], &b.cubHead[2 * rec + part]);
      else cpAsync16(&slots[r].basis[part - 2u], &b.cubBasis[9 * rec + (part - 2u)]);
    }
    cpAsyncWaitAll();
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < nrec * 4u; c += blockDim.x) {
      const uint32_t r = c >> 2, part = c & 3u;
      if (chunk * groupsPerBlock + r / K >= count) continue;
      const uint4 head = slots[r].head[0];
      if (head.x != kEmptyTet && __uint_as_float(head.y) > 0.0f && inBounds(head.x, b.tetTotal, kSiteRecordTet))
        cpAsync16(&slots[r].tet[part], &b.tets[4ull * head.x + part]);
    }
    cpAsyncWaitAll();
    __syncthreads();
  }
#endif
  // One vertex per lane group; its scene selects the settings and records.
  const uint32_t item = chunk * groupsPerBlock + group;
  const uint32_t listed = (groupLane && item < count) ? (list ? list[item] : item) : 0u;
  const bool haveVertex = groupLane && item < count && inBounds(listed, b.vertexTotal, kSiteListVertex);
  const uint32_t v = haveVertex ? listed : 0u;
  const uint32_t scene = haveVertex ? b.vertexScene[v] : sScene;
  // Per-vertex outputs owned by lane 0.
  uint32_t status = kNonfinite, backtracks = 0, evals = 0;
  float shiftN = 0.0f;
  bool localValid = true, haveRecord = false;
  if (haveVertex && pp[scene].active) {
    const DevParams p = pp[scene];
    FrameState* fs = &b.frames[scene];
    const bool isLatched = latched(p, fs);
    const uint4 info = b.vinfo[v];
    const float4 rm = b.restMass[v];
    if (isLatched) {
      if (lane == 0) tgt[v] = ldPos<kCoherent>(src, v);
    } else if (isPinned(info)) {
      if (lane == 0) {
        tgt[v] = make_float4(rm.x, rm.y, rm.z, 1.0f);
        b.finalUpdate[v] = 0.0f;
        float4* L = &b.local[4ull * v];
        L[0] = L[1] = L[2] = make_float4(0, 0, 0, 0);
        L[3] = make_float4(0, 0, 0, float(kPinned));
        status = kPinned;
        haveRecord = true;
      }
    } else {
      const float4 c0 = fs->control[0];
      const uint32_t vb = controlBits(c0.w) & kValidityMask;
      const bool amv = (vb & kAcceptedMinimumValid) != 0u && finiteS(c0.z);
      if (!(amv && c0.z > kDeterminantFloor)) {
        // Preflight rejection before any material evaluation (jgs2-shader.ts:3042-3081).
        if (lane == 0) {
          tgt[v] = ldPos<kCoherent>(src, v);
          b.finalUpdate[v] = 0.0f;
          float4* L = &b.local[4ull * v];
          L[0] = L[1] = L[2] = make_float4(0, 0, 0, 0);
          status = amv ? kLineSearchFailed : kNonfinite;
          L[3] = make_float4(amv ? c0.z : 0.f, 0, 0, float(status));
          localValid = status != kNonfinite;
          haveRecord = true;
        }
      } else {
        const float3 position = xyz(ldPos<kCoherent>(src, v));
        const float3 predV = xyz(b.predicted[v]);
        const float inertia = rm.w * p.invDt2;
        const float dWs = distributedInertiaWeight(rm, info, p.invDt2);
        const float nS = float(info.y > 1u ? info.y : 1u);
        const bool objActive = p.objectiveFlags != 0u;
        const float3 objS = objActive ? objectiveGradient(p, b, v, position) : f3(0, 0, 0);
        const float ktS = targetStiffness(p, b, v);
        Comp3 gsum = czero();  // compensated gradient gather
        S3 hess = szero();
        // Record terms are formed in the source vertex's frame: with
        // B_l = R_l Ubar_l R_s^T = B'_l R_s^T, a record's projected gradient
        // and Hessian are R_s g' and R_s H' R_s^T of the same expressions over
        // B'_l = R_l Ubar_l, so R_s is applied once per record instead of once
        // per basis block.  The exact source block subtracted for a record at
        // the vertex's own slot is formed in the world frame.
        const M3 Rs = loadRotT<kCoherent>(b.vertexRot, v);
        unsigned char* mySlots = slotBase + static_cast<size_t>(group) * K * kSolveSlotBytes;
        // Cubature records first, then (unless cached) the incident tets, in
        // separate loops so the two kinds of item never share a divergent pass.
        for (uint32_t u = lane; u < K; u += W) {
          // ---- cubature record (jgs2-shader.ts:3197-3263) ----
          CubState st;
          TetRec r;
          const size_t rec = static_cast<size_t>(v) * K + u;
          if constexpr (kCache && JGS2_SOLVE_STAGE)
            recordState<kCoherent, true>(b, p, v, rec, reinterpret_cast<const RecSlot*>(mySlots + u * kSolveSlotBytes),
                                         src, objActive, st, r);
          else
            recordState<kCoherent, false>(b, p, v, rec, nullptr, src, objActive, st, r);
          if (st.w > 0.0f) {
            const float w = st.w;
            const M3& F = st.F;
            const M3 &dF0 = st.dF0, &dF1 = st.dF1, &dF2 = st.dF2;
            const PiolaTerms pt = piolaTerms(F, r.lambda, r.mu);
            const M3 P = piola(F, pt);
            float3 pg = r.vol * f3(frob(dF0, P), frob(dF1, P), frob(dF2, P)) + st.gQ;
            // Reduced material Hessian vol <dF_r, DP[dF_c]>; the cofactor
            // term <A, Dcof[B]> is symmetric, so one directional cofactor is
            // live at a time.
            const float p0 = frob(F, dF0), p1 = frob(F, dF1), p2 = frob(F, dF2);
            const float q0 = frob(pt.cof, dF0), q1 = frob(pt.cof, dF1), q2 = frob(pt.cof, dF2);
            S3 ph;
            {
              const M3 D0 = dcofactor(F, dF0);
              ph.xx = pt.b * frob(dF0, D0);
              ph.xy = pt.b * frob(dF1, D0);
              ph.xz = pt.b * frob(dF2, D0);
            }
            {
              const M3 D1 = dcofactor(F, dF1);
              ph.yy = pt.b * frob(dF1, D1);
              ph.yz = pt.b * frob(dF2, D1);
            }
            ph.zz = pt.b * frob(dF2, dcofactor(F, dF2));
            ph.xx += pt.a * frob(dF0, dF0) + pt.c1 * p0 * p0 + r.lambda * q0 * q0;
            ph.yy += pt.a * frob(dF1, dF1) + pt.c1 * p1 * p1 + r.lambda * q1 * q1;
            ph.zz += pt.a * frob(dF2, dF2) + pt.c1 * p2 * p2 + r.lambda * q2 * q2;
            ph.xy += pt.a * frob(dF0, dF1) + pt.c1 * p0 * p1 + r.lambda * q0 * q1;
            ph.xz += pt.a * frob(dF0, dF2) + pt.c1 * p0 * p2 + r.lambda * q0 * q2;
            ph.yz += pt.a * frob(dF1, dF2) + pt.c1 * p1 * p2 + r.lambda * q1 * q2;
            ph.xx *= r.vol; ph.yy *= r.vol; ph.zz *= r.vol; ph.xy *= r.vol; ph.xz *= r.vol; ph.yz *= r.vol;
            sadd(ph, st.HQ);
            cadd(gsum, w * mv(Rs, pg));
            saddScaled(hess, w, srotate(Rs, ph));
            if (st.slot < 4) {
              // Remove the exact source block already in the local gather.
              const float3 gs = st.gs;
              float3 ps = r.vol * mv(P, gs) + dWs * (position - predV);
              if (objActive) ps = ps + objS * (1.0f / nS);
              const float3 u1 = mv(F, gs), w1 = mv(pt.cof, gs);
              S3 blk = szero();
              saddDiag(blk, pt.a * dot3(gs, gs));
              saddOuter(blk, pt.c1, u1);
              saddOuter(blk, r.lambda, w1);
              cadd(gsum, (-w) * ps);
              saddScaled(hess, -w * r.vol, blk);
              saddDiag(hess, -w * (dWs + ktS / nS));
            }
          }
          if constexpr (kCache) *reinterpret_cast<CubState*>(mySlots + u * kSolveSlotBytes) = st;
        }
        if (!cachedIncident) {
          for (uint32_t a = lane; a < info.y; a += W) {
            // ---- incident tetrahedron (jgs2-shader.ts:3097-3111) ----
            const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
            TetRec r;
            if (!incidentTetChecked(b.tets, entry, b.tetTotal, b.vertexTotal, &r)) continue;
            const M3 F = deformationAtT<kCoherent>(r, src);
            const PiolaTerms pt = piolaTerms(F, r.lambda, r.mu);
            const float3 g = shapeGradient(r, entry & 3u);
            cadd(gsum, r.vol * mv(piola(F, pt), g));
            addIncidentBlock(hess, r, F, pt, g);
          }
          // ---- cloth membrane and bending (jgs2-shader.ts:3113-3186) ----
          if (kExt && p.cloth)
            clothLocalSystem<true, kCoherent>(b.clothTris, b.clothHinges, b.clothIncidence, b.clothRange[v], src,
                                   clothMaterial(p), lane, W, gsum, hess);
        }
        // ---- IPC contact (jgs2-shader.ts:3193-3195): the cached source
        // contacts, or fresh ones under the coloured schedule ----
        if (kExt && p.ipc)
          contactLocal<true>(b, p, v, src, !cachedIncident, kContactSource, lane, W, gsum, hess);
        // Group reduction of the gather.
        groupMerge<W>(gsum, mask);
        hess.xx = groupSum<W>(hess.xx, mask);
        hess.yy = groupSum<W>(hess.yy, mask);
        hess.zz = groupSum<W>(hess.zz, mask);
        hess.xy = groupSum<W>(hess.xy, mask);
        hess.xz = groupSum<W>(hess.xz, mask);
        hess.yz = groupSum<W>(hess.yz, mask);
        if (cachedIncident) {
          const float4 i0 = b.incident[3ull * v], i1 = b.incident[3ull * v + 1], i2 = b.incident[3ull * v + 2];
          cadd(gsum, f3(i0.x, i0.y, i0.z));
          hess.xx += i0.w;
          hess.yy += i1.x;
          hess.zz += i1.y;
          hess.xy += i1.z;
          hess.xz += i1.w;
          hess.yz += i2.x;
        }
        // Own terms: inertia, objectives, floor (jgs2-shader.ts:3083-3092, 3188-3191).
        cadd(gsum, inertia * (position - predV));
        saddDiag(hess, inertia);
        if (objActive) cadd(gsum, objS);
        if (p.objectiveFlags & 2u) saddDiag(hess, ktS);
        if (p.floorStiffness > 0.0f && position.y < p.floorHeight) {
          cadd(gsum, f3(0.0f, p.floorStiffness * (position.y - p.floorHeight), 0.0f));
          hess.yy += p.floorStiffness;
        }
        const float3 grad = cvalue(gsum);
        // ---- globalization and line search (jgs2-shader.ts:3265-3473) ----
        const SolveResult dr = globalizationSolve(hess, grad, inertia);
        status = kNonfinite;
        const float3 fullP = position + dr.direction;
        const float3 fullD = fullP - position;
        const float scs = fmaxf(fabsf(position.x), fmaxf(fabsf(position.y), fabsf(position.z)));
        const float resolution =
            fmaxf(p.sceneScale, fmaxf(scs, 1.0e-12f)) * kUnitRoundoff * kPositionResolutionMultiplier;
        const bool below = dr.status == kAccepted && finiteV(fullP) && finiteV(fullD) && scaledLength(fullD) <= resolution;
        if (dr.status == kAccepted) status = below ? kZeroGradient : kLineSearchFailed;
        else if (dr.status == kZeroGradient) status = kZeroGradient;
        else if (dr.status == kShiftLimit) status = kShiftLimit;
        else if (dr.status == kCholeskyFailed) status = kCholeskyFailed;
        else if (dr.status == kNonDescent) status = kNonDescent;
        float alpha = 0.0f, acceptedDelta = 0.0f, bound = 0.0f, minTrialDet = 0.0f;
        float3 acceptedD = f3(0, 0, 0), acceptedP = position;
        if (dr.status == kAccepted && !below) {
          float ta = 1.0f;
          const float dl = scaledLength(dr.direction);
          if (p.maxStep > 0.0f && dl > p.maxStep) ta = p.maxStep / dl;
          const float controlMin = c0.z;  // accepted-source minimum (finite here)
          const uint4 cr = (kExt && p.cloth) ? b.clothRange[v] : make_uint4(0u, 0u, 0u, 0u);
          const uint32_t contactFirst = (kExt && p.ipc) ? b.contactRange[v].x : 0u;
          const uint32_t contactActive = (kExt && p.ipc) ? b.activeCount[v] : 0u;
          const ClothMaterial cmat = clothMaterial(p);
          for (uint32_t bt = 0; bt <= kMaxBacktracks; ++bt) {
            const float3 tp = position + ta * dr.direction;
            const float3 td = tp - position;
            if (!finiteV(tp) || !finiteV(td)) { status = kNonfinite; minTrialDet = 0.f; backtracks = bt; break; }
            const float tl = scaledLength(td);
            if (p.maxStep > 0.0f && tl > p.maxStep) { ta *= kBacktrackFactor; continue; }
            if (tl <= resolution) { status = kZeroGradient; minTrialDet = 0.f; backtracks = bt; break; }
            const float gd = dot3(grad, td);
            if (!finiteS(gd)) { status = kNonfinite; minTrialDet = 0.f; backtracks = bt; break; }
            if (!(gd < 0.0f)) { status = kZeroGradient; minTrialDet = 0.f; backtracks = bt; break; }
            // Restricted geometry and energy in one pass over the items
            // (restrictedMinimumDeformationDeterminant :1980-2118 and
            // restrictedEnergyDelta :2120-2337); the energy is used only
            // when the geometry is feasible, as in the reference order.
            float jmin = kF32Max, de = 0.0f;
            const float3 ts = mtv(Rs, td);
            bool geomFinite = true;
            // A lane's items in order: its cached cubature records, then its
            // incident tets (the same per-lane order as one merged loop).
            for (uint32_t u = lane; u < K; u += W) {
              CubState stLocal;
              if constexpr (!kCache) {
                // No shared cache for wide records: recompute the record's
                // state (the same arithmetic as the gather above).
                TetRec rr;
                recordState<kCoherent, false>(b, p, v, static_cast<size_t>(v) * K + u, nullptr, src, objActive,
                                              stLocal, rr);
              }
              const CubState& st =
                  kCache ? *reinterpret_cast<const CubState*>(mySlots + u * kSolveSlotBytes) : stLocal;
              if (!(st.w > 0.0f)) continue;
              float J = 0.0f;
              // Record state is in the source frame: the trial step there is R_s^T td.
              const M3 D = ts.x * st.dF0 + ts.y * st.dF1 + ts.z * st.dF2;
              const float dm = st.vol * snhEnergyDelta(st.F, st.I0, st.J0, D, st.lambda, st.mu, &J);
              float comp = dm + dot3(ts, st.gQ) + 0.5f * dot3(ts, smv(st.HQ, ts));
              if (st.slot < 4) {
                float Js;
                comp -= st.vol * snhEnergyDelta(st.F, st.I0, st.J0, outer(td, st.gs), st.lambda, st.mu, &Js);
                comp -= dWs * (dot3(position - predV, td) + 0.5f * dot3(td, td));
                if (objActive) comp -= objectiveDelta(p, b, v, position, td) / nS;
              }
              de += st.w * comp;
              if (!finiteS(J)) geomFinite = false;
              jmin = fminf(jmin, J);
            }
            // Incident tets of lane-order index u >= K, i.e. adjacency slot u - K.
            const uint32_t firstInc = lane >= K % W ? lane - K % W : lane + W - K % W;
#if JGS2_CONV_LOOKAHEAD
            // The lane's next incident tet is requested before the current
            // one's arithmetic (as in the convergence gather).
            uint32_t nextEntry = firstInc < info.y ? __ldg(&b.adjacency[info.x + firstInc]) : 0u;
            TetRec nextRec;
            bool nextOk = false;
            if (firstInc < info.y) nextOk = incidentTetChecked(b.tets, nextEntry, b.tetTotal, b.vertexTotal, &nextRec);
#endif
            for (uint32_t a = firstInc; a < info.y; a += W) {
              float J = 0.0f;
#if JGS2_CONV_LOOKAHEAD
              const uint32_t entry = nextEntry;
              const TetRec r = nextRec;
              const bool tetOk = nextOk;
              if (a + W < info.y) {
                nextEntry = __ldg(&b.adjacency[info.x + a + W]);
                nextOk = incidentTetChecked(b.tets, nextEntry, b.tetTotal, b.vertexTotal, &nextRec);
              }
#else
              const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
              TetRec r;
              const bool tetOk = incidentTetChecked(b.tets, entry, b.tetTotal, b.vertexTotal, &r);
#endif
              if (!tetOk) continue;
              const M3 F = deformationAtT<kCoherent>(r, src);
              const float I0 = frob(F, F);
              const float J0 = mdet(F);
#if JGS2_LS_RANK1
              de += r.vol * snhEnergyDeltaRankOne(F, I0, J0, td, shapeGradient(r, entry & 3u), r.lambda, r.mu, &J);
#else
              de += r.vol * snhEnergyDelta(F, I0, J0, outer(td, shapeGradient(r, entry & 3u)), r.lambda, r.mu, &J);
#endif
              if (!finiteS(J)) geomFinite = false;
              jmin = fminf(jmin, J);
            }
            // Cloth: signed area stretch at the source and the trial pose
            // (jgs2-shader.ts:2067-2116) and the membrane / bending energy
            // deltas (:2207-2263) of the incident elements.
            const float3 trialPos = position + td;
            for (uint32_t a = lane; a < cr.y; a += W) {
              const uint32_t entry = __ldg(&b.clothIncidence[cr.x + a]);
              const uint32_t slot = entry & 3u;
              const ClothTri ct = loadClothTri(b.clothTris, entry >> 2);
              const float3 x0 = xyz(ldPos<kCoherent>(src, ct.i0)), x1 = xyz(ldPos<kCoherent>(src, ct.i1)), x2 = xyz(ldPos<kCoherent>(src, ct.i2));
              const float3 y0 = slot == 0u ? trialPos : x0;
              const float3 y1 = slot == 1u ? trialPos : x1;
              const float3 y2 = slot == 2u ? trialPos : x2;
              const float3 sn = clothRawNormal(x0, x1, x2), tn = clothRawNormal(y0, y1, y2);
              const float twice = 2.0f * ct.area;
              const float ss = length3(sn) / twice, tm = length3(tn) / twice;
              const float ts = dot3(sn, tn) > 0.0f ? tm : -tm;
              if (!(twice > 0.0f) || !finiteS(ss) || !finiteS(ts)) geomFinite = false;
              jmin = fminf(jmin, fminf(ss, ts));
              de += clothMembraneEnergy(ct, y0, y1, y2, cmat) - clothMembraneEnergy(ct, x0, x1, x2, cmat);
            }
            for (uint32_t a = lane; a < cr.w; a += W) {
              const uint32_t entry = __ldg(&b.clothIncidence[cr.z + a]);
              const uint32_t slot = entry & 3u, h = entry >> 2;
              const uint4 q = hingeIndices(b.clothHinges, h);
              const float4 rest = __ldg(&b.clothHinges[2ull * h + 1]);
              const float3 x0 = xyz(ldPos<kCoherent>(src, q.x)), x1 = xyz(ldPos<kCoherent>(src, q.y)), x2 = xyz(ldPos<kCoherent>(src, q.z)), x3 = xyz(ldPos<kCoherent>(src, q.w));
              const float es = clothBendingEnergy(x0, x1, x2, x3, rest, cmat.bending);
              const float et = clothBendingEnergy(slot == 0u ? trialPos : x0, slot == 1u ? trialPos : x1,
                                                  slot == 2u ? trialPos : x2, slot == 3u ? trialPos : x3, rest,
                                                  cmat.bending);
              de += et - es;
            }
            // IPC: a trial within the minimum distance of an active candidate
            // is infeasible (jgs2-shader.ts:1997-2038); barrier and lagged
            // friction energy deltas (:2137-2196).
            if (kExt && contactActive) {
              const float dl = length3(td);
              for (uint32_t a = lane; a < contactActive; a += W) {
                const uint32_t c = b.activeIds[contactFirst + a];
                const float4* cst = b.contactState + kContactStateWords * static_cast<size_t>(c);
                const ContactData source = cachedIncident ? ipcCached(cst[kContactSource], cst[kContactSourceWeights])
                                                          : contactAt(b, c, src, p.ipcActivation);
                if (!source.valid) {
                  geomFinite = false;
                  continue;
                }
                uint32_t ctype;
                const uint4 cq = contactIndices(b, c, &ctype);
                if (ipcWeightFor(cq, make_float4(1.f, 1.f, 1.f, 1.f), v) == 0.0f) continue;
                const bool nearMinimum = !(source.distance - dl > p.ipcMinDistance);
                const bool mayChange = source.distance - dl < p.ipcActivation;
                const bool friction = p.ipcFriction > 0.0f && cst[kContactLagged].w > 0.0f;
                ContactData trial = {p.ipcActivation, f3(1, 0, 0), make_float4(0, 0, 0, 0), true};
                if (nearMinimum || mayChange) trial = contactAt(b, c, src, p.ipcActivation, v, trialPos);
                if (nearMinimum) {
                  if (!trial.valid) geomFinite = false;
                  else if (!(trial.distance > p.ipcMinDistance)) jmin = fminf(jmin, 0.0f);
                }
                if (mayChange || friction)
                  de += contactEnergy(b, p, c, trial, src, v, trialPos) -
                        contactEnergy(b, p, c, source, src, 0xffffffffu, f3(0, 0, 0));
              }
            }
            jmin = groupMin<W>(jmin, mask);
            const bool allFinite = __all_sync(mask, geomFinite);
            de = groupSum<W>(de, mask);
            if (!allFinite) { status = kNonfinite; minTrialDet = 0.f; backtracks = bt; break; }
            const float trialMin = fminf(controlMin, jmin);
            minTrialDet = trialMin;
            if (trialMin > kDeterminantFloor) {
              de += inertia * (dot3(position - predV, td) + 0.5f * dot3(td, td)) + floorDelta(p, position.y, td.y);
              if (objActive) de += objectiveDelta(p, b, v, position, td);
              evals += 1;
              if (!finiteS(de)) { status = kNonfinite; backtracks = bt; break; }
              const float tb = kArmijoC1 * gd;
              if (de <= tb) {
                alpha = ta; acceptedDelta = de; bound = tb; backtracks = bt; status = kAccepted;
                acceptedD = td; acceptedP = tp;
                break;
              }
            }
            ta *= kBacktrackFactor;
          }
          if (status == kLineSearchFailed) backtracks = kMaxBacktracks;
        }
        if (lane == 0) {
          tgt[v] = make_float4(acceptedP.x, acceptedP.y, acceptedP.z, 1.0f);
          b.finalUpdate[v] = scaledLength(acceptedD);
          float4* L = &b.local[4ull * v];
          const float4 l0 = make_float4(dr.direction.x, dr.direction.y, dr.direction.z, alpha);
          const float4 l1 = make_float4(dr.minEig * dr.scale, dr.scale, dr.shift * dr.scale, dr.shift);
          const float4 l2 = make_float4(acceptedDelta, bound, dr.gdd, dr.residual);
          const float4 l3 = make_float4(minTrialDet, float(backtracks), float(evals), float(status));
          L[0] = l0; L[1] = l1; L[2] = l2; L[3] = l3;
          localValid = finiteS(l0.x) && finiteS(l0.y) && finiteS(l0.z) && finiteS(l0.w) && finiteS(l1.x) &&
                       finiteS(l1.y) && finiteS(l1.z) && finiteS(l1.w) && finiteS(l2.x) && finiteS(l2.y) &&
                       finiteS(l2.z) && finiteS(l2.w) && finiteS(l3.x) && status != kNonfinite && l1.w >= 0.0f;
          shiftN = dr.shift;
          haveRecord = true;
        }
      }
    }
  }
  // Local aggregates of reduceCandidate's vertex loop (jgs2-shader.ts:3689-3790),
  // per scene: folded in shared memory when the block's vertices share one
  // scene, otherwise added per vertex.
  const bool oneScene = __syncthreads_and(!haveVertex || scene == sScene) != 0;
  if (haveRecord && lane == 0) {
    const bool failure = status == kShiftLimit || status == kNonDescent || status == kLineSearchFailed ||
                         status == kNonfinite || status == kCholeskyFailed;
    uint32_t trials = 0;
    if (status == kAccepted) trials = backtracks + 1;
    else if (status == kLineSearchFailed && backtracks == kMaxBacktracks) trials = kTrialCount;
    else if (status == kZeroGradient && backtracks > 0) trials = backtracks;
    else if (status == kNonfinite) trials = backtracks;  // a nonfinite trial never has J above the floor here
    const uint32_t skipped = trials - (trials < evals ? trials : evals);
    const uint32_t shiftBits = (shiftN > 0.0f && finiteS(shiftN)) ? __float_as_uint(shiftN) : 0u;
    if (oneScene) {
      if (failure) atomicAdd(&sFail, 1u);
      if (backtracks) atomicMax(&sMaxBack, backtracks);
      if (skipped) atomicAdd(&sSkip, skipped);
      if (evals) atomicAdd(&sEvals, evals);
      if (shiftBits) atomicMax(&sMaxShift, shiftBits);
      if (!localValid) sValid = 0;
    } else {
      FrameState* fs = &b.frames[scene];
      if (failure) atomicAdd(&fs->localFailures, 1u);
      if (backtracks) atomicMax(&fs->localMaxBacktracks, backtracks);
      if (skipped) atomicAdd(&fs->localSkipped, skipped);
      if (evals) atomicAdd(&fs->localEvaluations, evals);
      if (shiftBits) atomicMax(&fs->localMaxShift, shiftBits);
      if (!localValid) atomicAnd(&fs->localNumericsValid, 0u);
    }
  }
  __syncthreads();
  if (oneScene && threadIdx.x == 0) {
    FrameState* fs = &b.frames[sScene];
    if (sFail) atomicAdd(&fs->localFailures, sFail);
    if (sMaxBack) atomicMax(&fs->localMaxBacktracks, sMaxBack);
    if (sSkip) atomicAdd(&fs->localSkipped, sSkip);
    if (sEvals) atomicAdd(&fs->localEvaluations, sEvals);
    if (sMaxShift) atomicMax(&fs->localMaxShift, sMaxShift);
    if (!sValid) atomicAnd(&fs->localNumericsValid, 0u);
  }
}

// kCache: the records' line-search state is cached in shared memory (and the
// records are staged there); wide records (an exact complement) recompute it
// per trial instead, so a block needs no shared memory per vertex.
template <int W, bool kExt, bool kCache>
__global__ void __launch_bounds__(kBlock, JGS2_SOLVE_MIN_BLOCKS) solveKernel(Buffers b, const DevParams* __restrict__ pp,
                                                      const float4* __restrict__ src, float4* tgt,
                                                      const uint32_t* __restrict__ list, uint32_t count,
                                                      uint32_t K, int cachedIncident, uint32_t groupsPerBlock) {
  solveChunk<W, kExt, false, kCache>(b, pp, src, tgt, list, count, K, cachedIncident, groupsPerBlock, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Graph-coloured sweep as one persistent kernel (jgs2-solver.ts:2275-2325,
// colour masks jgs2-shader.ts:3004-3012): for each colour, the vertex frames
// of the vertices the colour's solves read, a grid barrier, the in-place
// local solves of the colour's vertices, a grid barrier.  The grid is
// launched cooperatively (all blocks resident).  Each barrier is a bounded
// spin: a block that waits longer than `spinLimit` polls sets the sweep's
// error word and every block leaves at its next barrier, so the kernel always
// returns; the host reports JGS2_TIMEOUT at its next synchronisation.
struct SweepBarrier {
  uint32_t arrived, generation, error, pad;
};

// Bounded grid barrier; false when the sweep has failed (by this block's
// timeout or another's).
__device__ __forceinline__ bool gridBarrier(SweepBarrier* bar, uint32_t spinLimit) {
  __shared__ uint32_t sOk;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile SweepBarrier* vb = bar;
    const uint32_t gen = vb->generation;
    __threadfence();
    const uint32_t before = atomicAdd(&bar->arrived, 1u);
    if (before == gridDim.x - 1) {
      bar->arrived = 0u;
      __threadfence();
      atomicAdd(&bar->generation, 1u);
    } else {
      uint32_t spins = 0;
      while (vb->generation == gen && vb->error == 0u) {
        if (++spins > spinLimit) {
          atomicOr(&bar->error, 1u);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    sOk = vb->error == 0u ? 1u : 0u;
  }
  __syncthreads();
  return sOk != 0u;
}

template <int W, bool kExt>
__global__ void __launch_bounds__(kBlock, JGS2_SOLVE_MIN_BLOCKS)
    coloredSweepKernel(Buffers b, const DevParams* __restrict__ pp, float4* x, const uint32_t* __restrict__ colorVertices,
                       const uint32_t* __restrict__ colorOffsets, const uint32_t* __restrict__ needVertices,
                       const uint32_t* __restrict__ needOffsets, uint32_t colorCount, uint32_t V, uint32_t K,
                       uint32_t groupsPerBlock, int refreshAllFrames, SweepBarrier* bar, uint32_t spinLimit) {
  for (uint32_t c = 0; c < colorCount; ++c) {
    // Frames of the vertices this colour reads (every vertex after the
    // frame's last colour, so the stored frames match a full pass).
    const bool all = refreshAllFrames && c + 1 == colorCount;
    const uint32_t nb = needOffsets[c], ne = all ? nb + V : needOffsets[c + 1];
    for (uint32_t i = nb + blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
      const uint32_t v = all ? i - nb : needVertices[i];
      const uint32_t scene = b.vertexScene[v];
      const DevParams& p = pp[scene];
      if (!p.active || latched(p, &b.frames[scene])) continue;
      storeFrame(b.vertexRot, v, vertexFrame<true>(b, x, v, p.rotationEpsilon));
    }
    if (!gridBarrier(bar, spinLimit)) return;
    const uint32_t cb = colorOffsets[c], count = colorOffsets[c + 1] - cb;
    const uint32_t chunks = (count + groupsPerBlock - 1) / groupsPerBlock;
    for (uint32_t chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x)
      solveChunk<W, kExt, true>(b, pp, x, x, colorVertices + cb, count, K, 0, groupsPerBlock, chunk);
    if (!gridBarrier(bar, spinLimit)) return;
  }
}

// ---------------------------------------------------------------------------
// Grid-wide reductions.  Each of the prologue, gate and convergence kernels
// runs on a persistent grid (a few blocks per SM, grid-stride loops), folds
// its elements into one partial per block with a fixed tree, writes the
// partial, and the last block to take a ticket folds all partials in block
// order.  Results are deterministic for a given device; nothing waits.
struct GatePartial {
  double e0, e1;      // source / candidate assembled energy
  float minS, minC;   // minimum determinant, source / candidate
  uint32_t bits;      // AND of geometry / energy validity bits
  uint32_t pad;
};
constexpr uint32_t kGateBits = kSourceGeometryValid | kCandidateGeometryValid | kSourceEnergyValid |
                               kCandidateEnergyValid;

__device__ __forceinline__ GatePartial gateIdentity() { return {0.0, 0.0, kF32Max, kF32Max, kGateBits, 0u}; }
__device__ __forceinline__ void gateCombine(GatePartial& a, const GatePartial& b) {
  a.e0 += b.e0;
  a.e1 += b.e1;
  a.minS = fminf(a.minS, b.minS);
  a.minC = fminf(a.minC, b.minC);
  a.bits &= b.bits;
}

struct ConvPartial {
  double sq[6];     // squared norms: five components and their sum
  float scale[6];   // max-abs entries (validity of the robust norm)
  float maxUpdate;
  uint32_t valid;
};
__device__ __forceinline__ ConvPartial convIdentity() {
  ConvPartial p;
  for (int c = 0; c < 6; ++c) { p.sq[c] = 0.0; p.scale[c] = 0.0f; }
  p.maxUpdate = 0.0f;
  p.valid = 1u;
  return p;
}
__device__ __forceinline__ void convCombine(ConvPartial& a, const ConvPartial& b) {
  for (int c = 0; c < 6; ++c) {
    a.sq[c] += b.sq[c];
    a.scale[c] = fmaxf(a.scale[c], b.scale[c]);
  }
  a.maxUpdate = fmaxf(a.maxUpdate, b.maxUpdate);
  a.valid &= b.valid;
}

template <class P, class C>
__device__ __forceinline__ P blockFold(P v, P* smem, C combine) {
  smem[threadIdx.x] = v;
  __syncthreads();
  for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) combine(smem[threadIdx.x], smem[threadIdx.x + s]);
    __syncthreads();
  }
  P r = smem[0];
  __syncthreads();
  return r;
}

// Publishes the block partial at `slot`; returns true in every thread of the
// last of the `count` blocks sharing `ticket`.
template <class P>
__device__ __forceinline__ bool publishPartial(const P& blockValue, P* partials, uint32_t slot, uint32_t count,
                                               uint32_t* ticket, bool* isLast) {
  if (threadIdx.x == 0) {
    partials[slot] = blockValue;
    __threadfence();
    *isLast = atomicAdd(ticket, 1u) == count - 1;
  }
  __syncthreads();
  const bool last = *isLast;
  if (last) __threadfence();
  return last;
}

// Folds partials[0, count) in index order (deterministic).
template <class P, class I, class C>
__device__ __forceinline__ P foldPartials(const P* partials, uint32_t count, P* smem, I identity, C combine) {
  P acc = identity();
  static_assert(sizeof(P) % 4 == 0, "partials are read as 32-bit words");
  for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
    // Other blocks wrote these partials: read them from L2.
    uint32_t words[sizeof(P) / 4];
    const uint32_t* w = reinterpret_cast<const uint32_t*>(partials + k);
#pragma unroll
    for (unsigned i = 0; i < sizeof(P) / 4; ++i) words[i] = __ldcg(w + i);
    P v;
    memcpy(&v, words, sizeof(P));
    combine(acc, v);
  }
  return blockFold(acc, smem, combine);
}

__device__ __forceinline__ void accumulateTet(GatePartial& acc, const TetRec& r, const M3& sF, const M3& cF) {
  const float sJ = mdet(sF), cJ = mdet(cF);
  const bool sgv = finiteS(sJ), cgv = finiteS(cJ);
  if (sgv) acc.minS = fminf(acc.minS, sJ); else acc.bits &= ~kSourceGeometryValid;
  if (cgv) acc.minC = fminf(acc.minC, cJ); else acc.bits &= ~kCandidateGeometryValid;
  bool sev = false, cev = false;
  if (sgv && sJ > kDeterminantFloor) {
    const float e = r.vol * snhEnergy(sF, r.lambda, r.mu);
    sev = finiteS(e);
    if (sev) acc.e0 += e;
  }
  if (cgv && cJ > kDeterminantFloor) {
    const float e = r.vol * snhEnergy(cF, r.lambda, r.mu);
    cev = finiteS(e);
    if (cev) acc.e1 += e;
  }
  if (!sev) acc.bits &= ~kSourceEnergyValid;
  if (!cev) acc.bits &= ~kCandidateEnergyValid;
}

// A cloth triangle as a gate element: its signed area stretch at the source
// and the candidate (candidateTetrahedron, jgs2-shader.ts:3507-3549), and its
// membrane energy, which the reference adds to the energy of the triangle's
// lowest vertex when that vertex's area stretch is above the floor and
// replaces the vertex energy by kF32Max otherwise (:2585-2621).
__device__ __forceinline__ void accumulateClothTri(GatePartial& acc, const ClothTri& t, const float4* __restrict__ s,
                                                   const float4* __restrict__ c, const ClothMaterial& m) {
  const float3 s0 = xyz(s[t.i0]), s1 = xyz(s[t.i1]), s2 = xyz(s[t.i2]);
  const float3 c0 = xyz(c[t.i0]), c1 = xyz(c[t.i1]), c2 = xyz(c[t.i2]);
  const float3 sn = clothRawNormal(s0, s1, s2), cn = clothRawNormal(c0, c1, c2);
  const float twice = 2.0f * t.area;
  const float ss = length3(sn) / twice;
  const float cm = length3(cn) / twice;
  const float cs = dot3(sn, cn) > 0.0f ? cm : -cm;
  const bool sgv = twice > 0.0f && finiteV(sn) && finiteS(ss);
  const bool cgv = twice > 0.0f && finiteV(cn) && finiteS(cs);
  if (sgv) acc.minS = fminf(acc.minS, ss); else acc.bits &= ~kSourceGeometryValid;
  if (cgv) acc.minC = fminf(acc.minC, cs); else acc.bits &= ~kCandidateGeometryValid;
  const float es = (twice > 0.0f && finiteS(ss) && ss > kDeterminantFloor) ? clothMembraneEnergy(t, s0, s1, s2, m)
                                                                            : kF32Max;
  const float ec = (twice > 0.0f && finiteS(cm) && cm > kDeterminantFloor) ? clothMembraneEnergy(t, c0, c1, c2, m)
                                                                            : kF32Max;
  if (finiteS(es)) acc.e0 += es; else acc.bits &= ~kSourceEnergyValid;
  if (finiteS(ec)) acc.e1 += ec; else acc.bits &= ~kCandidateEnergyValid;
}

// An active IPC candidate's barrier and friction energy at the source
// (source contact cache) and the candidate (target cache, or the source cache
// when the contact step collapsed to zero): ipcOwnedEnergy (:751-781), which
// the reference adds to the energy of the candidate's first unpinned vertex,
// and which becomes kF32Max for an invalid contact.
__device__ __forceinline__ void accumulateContact(GatePartial& acc, const Buffers& b, const DevParams& p,
                                                  float contactAlpha, uint32_t c, const float4* __restrict__ src,
                                                  const float4* __restrict__ tgt) {
  if (!b.contactFlag[c]) return;  // not in the active rows of this iteration
  const float4* st = b.contactState + kContactStateWords * static_cast<size_t>(c);
  const ContactData ks = ipcCached(st[kContactSource], st[kContactSourceWeights]);
  const ContactData kc = contactAlpha != 0.0f ? ipcCached(st[kContactTarget], st[kContactTargetWeights]) : ks;
  const bool friction = p.ipcFriction > 0.0f && st[kContactLagged].w > 0.0f;
  auto energy = [&](const ContactData& k, const float4* __restrict__ x) {
    if (!k.valid) return kF32Max;
    if (!ipcBarrierActive(k.distance, p.ipcActivation) && !friction) return 0.0f;
    const float e = contactEnergy(b, p, c, k, x, 0xffffffffu, f3(0, 0, 0));
    return finiteS(e) ? e : kF32Max;
  };
  const float es = energy(ks, src), ec = energy(kc, tgt);
  if (finiteS(es)) acc.e0 += es; else acc.bits &= ~kSourceEnergyValid;
  if (finiteS(ec)) acc.e1 += ec; else acc.bits &= ~kCandidateEnergyValid;
}

// A hinge's bending energy at the source and the candidate (owned by its
// lowest vertex in the reference, :2623-2642).
__device__ __forceinline__ void accumulateHinge(GatePartial& acc, const float4* __restrict__ hinges, uint32_t h,
                                                const float4* __restrict__ s, const float4* __restrict__ c,
                                                float bending) {
  const uint4 q = hingeIndices(hinges, h);
  const float4 rest = __ldg(&hinges[2ull * h + 1]);
  const float es = clothBendingEnergy(xyz(s[q.x]), xyz(s[q.y]), xyz(s[q.z]), xyz(s[q.w]), rest, bending);
  const float ec = clothBendingEnergy(xyz(c[q.x]), xyz(c[q.y]), xyz(c[q.z]), xyz(c[q.w]), rest, bending);
  if (finiteS(es)) acc.e0 += es; else acc.bits &= ~kSourceEnergyValid;
  if (finiteS(ec)) acc.e1 += ec; else acc.bits &= ~kCandidateEnergyValid;
}

// ---------------------------------------------------------------------------
// Prologue: predict (jgs2-shader.ts:2660-2692), iteration-0 vertex frames and
// the source feasibility preflight (candidateTetrahedron + reduceCandidate on
// the accepted pose, jgs2-solver.ts:2240-2259).
__global__ void __launch_bounds__(kBlock) prologueKernel(Buffers b, const DevParams* __restrict__ pp) {
  __shared__ GatePartial smem[kBlock];
  __shared__ bool isLast;
  const RedBlock rb = b.gateTable[blockIdx.x];
  const SceneRange sr = b.scenes[rb.scene];
  const DevParams p = pp[rb.scene];
  if (!p.active) return;  // uniform across the scene's blocks
  FrameState* fs = &b.frames[rb.scene];
  GatePartial acc = gateIdentity();
  for (uint32_t k = rb.begin + threadIdx.x; k < rb.end; k += blockDim.x) {
    if (k < sr.V) {
      const uint32_t i = sr.vOff + k;
      const float4 o = b.pos[0][i];
      b.old[i] = make_float4(o.x, o.y, o.z, 1.0f);
      const uint4 info = b.vinfo[i];
      const float4 rm = b.restMass[i];
      float3 pred = xyz(rm);
      if (!isPinned(info)) {
        const float3 vel = p.velocityDamping * xyz(b.velocity[i]);
        pred = xyz(o) + p.dt * vel + (p.dt * p.dt) * f3(p.gravity[0], p.gravity[1], p.gravity[2]);
      } else {
        b.velocity[i] = make_float4(0, 0, 0, 0);
      }
      b.predicted[i] = make_float4(pred.x, pred.y, pred.z, distributedInertiaWeight(rm, info, p.invDt2));
      b.finalUpdate[i] = 0.0f;
      if (!p.globalization) {
        // Co-rotated path: the iteration source is the inertial prediction.
        b.pos[1][i] = make_float4(pred.x, pred.y, pred.z, 1.0f);
        continue;
      }
      // The stable iteration source is the accepted pose.
      b.pos[1][i] = make_float4(o.x, o.y, o.z, 1.0f);
      // Iteration-0 frames (and, for free vertices, the incident system).
      if (isPinned(info)) storeFrame(b.vertexRot, i, vertexFrame(b, b.pos[0], i, p.rotationEpsilon));
      else frameAndIncident(b, p, b.pos[0], i, info, p.rotationEpsilon);
      const float e = implicitEnergy(p, b, i, xyz(o), info);
      if (finiteS(e)) { acc.e0 += e; acc.e1 += e; }
      else acc.bits &= ~(kSourceEnergyValid | kCandidateEnergyValid);
    }
    if (p.globalization && k < sr.T) {
      const TetRec r = loadTet(b.tets, sr.tOff + k);
      if (tetVerticesInBounds(r.idx, b.vertexTotal)) {
        const M3 F = deformationAt(r, b.pos[0]);
        accumulateTet(acc, r, F, F);
      }
    }
    if (p.cloth) {
      if (k < sr.C) accumulateClothTri(acc, loadClothTri(b.clothTris, sr.cOff + k), b.pos[0], b.pos[0], clothMaterial(p));
      if (k < sr.H) accumulateHinge(acc, b.clothHinges, sr.hOff + k, b.pos[0], b.pos[0], p.clothBending);
    }
  }
  if (!p.globalization) return;  // no preflight on the co-rotated path (uniform)
  const GatePartial blk = blockFold(acc, smem, gateCombine);
  GatePartial* partials = reinterpret_cast<GatePartial*>(b.gatePartials);
  if (!publishPartial(blk, partials, rb.slot, sr.gateBlocks, &fs->prologueTicket, &isLast)) return;
  const GatePartial tot = foldPartials(partials + sr.gateBase, sr.gateBlocks, smem, gateIdentity, gateCombine);
  if (threadIdx.x != 0) return;
  uint32_t vb = tot.bits;
  if (sr.T == 0) vb &= ~(kSourceGeometryValid | kCandidateGeometryValid);
  const bool gv = (vb & kSourceGeometryValid) != 0u;
  const float e0 = float(tot.e0);
  const bool ev = (vb & kSourceEnergyValid) != 0u && finiteS(e0);
  const float m = tot.minS;
  const bool accepted = gv && m > kDeterminantFloor;
  uint32_t cbits = (vb & (kSourceGeometryValid | kCandidateGeometryValid)) | kLocalNumericsValid;
  if (gv) cbits |= kAcceptedMinimumValid;
  // predict clears the control records; the preflight then writes them with
  // history index 0 (jgs2-shader.ts:2687-2691, 3916-3953).
  fs->control[0] = make_float4(gv ? m : 0.f, gv ? m : 0.f, gv ? m : 0.f, float(cbits));
  fs->control[1] = make_float4(accepted ? 1.f : 0.f, accepted ? 0.f : 1.f, 0.f, 0.f);
  fs->control[2] = make_float4(ev ? e0 : 0.f, ev ? e0 : 0.f, ev ? e0 : 0.f, ev ? 1.f : 0.f);
  fs->control[3] = make_float4(0, 0, 0, 0);
  fs->prologueTicket = 0u;
}

// ---------------------------------------------------------------------------
// Gate: candidateTetrahedron (jgs2-shader.ts:3498-3601) + vertex energies
// (assembledVertexEnergy :3489-3496) + reduceCandidate (:3611-3955).
// kExt: some scene of the engine has cloth or contact candidates (their
// terms are compiled out otherwise).  JGS2_GATE_MIN_BLOCKS and
// JGS2_GATE_EXT_MIN_BLOCKS: blocks per SM each instantiation's register
// budget must allow.  For the tetrahedral gate, eight blocks (32 warps per SM
// for this gather-bound kernel) measured 22 % faster on the 100^3 cube than
// the compiler's choice (5 blocks), with bitwise the same results, and six
// and ten slower than eight; with the cloth and contact terms eight blocks
// cost the cloth drape 6 % of its gate time, so that instantiation keeps the
// five blocks the compiler chose for the kernel before the split.
#ifndef JGS2_GATE_MIN_BLOCKS
#define JGS2_GATE_MIN_BLOCKS 8
#endif
#ifndef JGS2_GATE_EXT_MIN_BLOCKS
#define JGS2_GATE_EXT_MIN_BLOCKS 5
#endif
template <bool kExt>
__global__ void __launch_bounds__(kBlock, kExt ? JGS2_GATE_EXT_MIN_BLOCKS : JGS2_GATE_MIN_BLOCKS)
    gateKernel(Buffers b, const DevParams* __restrict__ pp, const float4* __restrict__ src,
               const float4* __restrict__ tgt) {
  __shared__ GatePartial smem[kBlock];
  __shared__ bool isLast;
  const RedBlock rb = b.gateTable[blockIdx.x];
  const SceneRange sr = b.scenes[rb.scene];
  const DevParams p = pp[rb.scene];
  FrameState* fs = &b.frames[rb.scene];
  if (!p.active || latched(p, fs)) return;  // uniform across the scene's blocks
  GatePartial acc = gateIdentity();
  // Contacts: element k takes candidates k, k + span, ... of the scene's
  // list (a single pass for static candidates, which the table covers).
  const uint32_t span = max(sr.gateSpan, 1u);
  const uint2 contacts =
      !kExt ? make_uint2(0u, 0u) : b.contactDynamic ? b.bpSpan[rb.scene] : make_uint2(sr.kOff, sr.KC);
  for (uint32_t k = rb.begin + threadIdx.x; k < rb.end; k += blockDim.x) {
    if (k < sr.T) {
      const TetRec r = loadTet(b.tets, sr.tOff + k);
      if (tetVerticesInBounds(r.idx, b.vertexTotal)) accumulateTet(acc, r, deformationAt(r, src), deformationAt(r, tgt));
    }
    if (k < sr.V) {
      const uint32_t i = sr.vOff + k;
      const uint4 info = b.vinfo[i];
      const float es = implicitEnergy(p, b, i, xyz(src[i]), info);
      const float ec = implicitEnergy(p, b, i, xyz(tgt[i]), info);
      if (finiteS(es)) acc.e0 += es; else acc.bits &= ~kSourceEnergyValid;
      if (finiteS(ec)) acc.e1 += ec; else acc.bits &= ~kCandidateEnergyValid;
    }
    if (kExt && p.cloth) {
      if (k < sr.C) accumulateClothTri(acc, loadClothTri(b.clothTris, sr.cOff + k), src, tgt, clothMaterial(p));
      if (k < sr.H) accumulateHinge(acc, b.clothHinges, sr.hOff + k, src, tgt, p.clothBending);
    }
    if (kExt && p.ipc)
      for (uint32_t c = k; c < contacts.y; c += span)
        accumulateContact(acc, b, p, fs->contactAlpha, contacts.x + c, src, tgt);
  }
  const GatePartial blk = blockFold(acc, smem, gateCombine);
  GatePartial* partials = reinterpret_cast<GatePartial*>(b.gatePartials);
  if (!publishPartial(blk, partials, rb.slot, sr.gateBlocks, &fs->gateTicket, &isLast)) return;
  const GatePartial tot = foldPartials(partials + sr.gateBase, sr.gateBlocks, smem, gateIdentity, gateCombine);
  if (threadIdx.x != 0) return;
  uint32_t vb = tot.bits;
  if (__ldcg(&fs->localNumericsValid)) vb |= kLocalNumericsValid;
  const float eS = float(tot.e0), eC = float(tot.e1);
  if (!finiteS(eS)) vb &= ~kSourceEnergyValid;
  if (!finiteS(eC)) vb &= ~kCandidateEnergyValid;
  if (sr.T == 0) vb &= ~(kSourceGeometryValid | kCandidateGeometryValid);
  const float sm = tot.minS, cm = tot.minC;
  const bool sgv = (vb & kSourceGeometryValid) != 0u, cgv = (vb & kCandidateGeometryValid) != 0u;
  const bool sev = (vb & kSourceEnergyValid) != 0u, cev = (vb & kCandidateEnergyValid) != 0u;
  const bool accepted = (sgv && sm > kDeterminantFloor) && (cgv && cm > kDeterminantFloor);
  const float am = accepted ? cm : sm;
  const bool amv = accepted ? cgv : sgv;
  const float ae = accepted ? eC : eS;
  const bool aev = accepted ? cev : sev;
  if (amv) vb |= kAcceptedMinimumValid;
  uint32_t historyIndex = 0;
  const float packed = fs->control[1].w;
  if (finiteNonnegInt(packed, float(kHistoryCapacity))) historyIndex = static_cast<uint32_t>(packed);
  else vb &= ~kLocalNumericsValid;
  const uint32_t cb = vb & kValidityMask;
  const uint32_t failures = __ldcg(&fs->localFailures);
  fs->control[0] = make_float4(sgv ? sm : 0.f, cgv ? cm : 0.f, amv ? am : 0.f, float(cb));
  fs->control[1] = make_float4(accepted ? 1.f : 0.f, accepted ? 0.f : 1.f, float(failures), float(historyIndex));
  fs->control[2] = make_float4(sev ? eS : 0.f, cev ? eC : 0.f, aev ? ae : 0.f, (sev && cev) ? 1.f : 0.f);
  fs->control[3] = make_float4(__uint_as_float(__ldcg(&fs->localMaxShift)), float(__ldcg(&fs->localMaxBacktracks)),
                               float(__ldcg(&fs->localSkipped)), float(__ldcg(&fs->localEvaluations)));
  // Reset the sweep accumulators for the next iteration.
  fs->localFailures = 0u;
  fs->localMaxBacktracks = 0u;
  fs->localSkipped = 0u;
  fs->localEvaluations = 0u;
  fs->localMaxShift = 0u;
  fs->localNumericsValid = 1u;
  fs->gateTicket = 0u;
}

// ---------------------------------------------------------------------------
// applyCandidate (:3957-3983) + convergenceGradient (:3985-4097) +
// reduceConvergence (:4105-4486), and the next iteration's vertex frames.
// The five component norms are exact Euclidean norms accumulated in double;
// the reference forms the same norms in f32 as scale * sqrt(sum((g/scale)^2)).
// JGS2_CONV_MIN_BLOCKS: blocks per SM the convergence kernel's register
// budget must allow (0: the compiler's choice, 151 registers and 3 blocks).
// Four blocks (128 registers) measured 5 % faster on the 100^3 cube than the
// compiler's choice, with bitwise the same results; five and six were slower.
#ifndef JGS2_CONV_MIN_BLOCKS
#define JGS2_CONV_MIN_BLOCKS 4
#endif
#if JGS2_CONV_MIN_BLOCKS > 0
#define JGS2_CONV_BOUNDS __launch_bounds__(kBlock, JGS2_CONV_MIN_BLOCKS)
#else
#define JGS2_CONV_BOUNDS __launch_bounds__(kBlock)
#endif

__global__ void JGS2_CONV_BOUNDS convergenceKernel(Buffers b, const DevParams* __restrict__ pp,
                                                            const float4* __restrict__ src, float4* tgt,
                                                            int nextRotations) {
  __shared__ ConvPartial smem[kBlock];
  __shared__ bool isLast;
  const RedBlock rb = b.convTable[blockIdx.x];
  const SceneRange sr = b.scenes[rb.scene];
  const DevParams p = pp[rb.scene];
  FrameState* fs = &b.frames[rb.scene];
  if (!p.active || latched(p, fs)) return;  // uniform across the scene's blocks
  const bool accepted = fs->control[1].x == 1.0f;
  const float4* __restrict__ acc = accepted ? tgt : src;
  const uint32_t V = sr.V;
  ConvPartial part = convIdentity();
  for (uint32_t k = rb.begin + threadIdx.x; k < rb.end; k += blockDim.x) {
    const uint32_t v = sr.vOff + k;
    float upd = 0.0f;
    if (!accepted) {
      tgt[v] = src[v];
    } else {
      upd = scaledLength(xyz(tgt[v]) - xyz(src[v]));
    }
    b.finalUpdate[v] = upd;
    if (!(finiteS(upd) && upd >= 0.0f)) part.valid = 0u; else part.maxUpdate = fmaxf(part.maxUpdate, upd);
    const uint4 info = b.vinfo[v];
    if (!isPinned(info)) {
      const float3 x = xyz(acc[v]);
      float3 comps[5];
      comps[0] = (b.restMass[v].w * p.invDt2) * (x - xyz(b.predicted[v]));
      Comp3 material = czero();  // compensated gradient gather
      M3 avg = mzero();
      float total = 0.0f;
      S3 hess = szero();
#if JGS2_CONV_LOOKAHEAD
      // The next incident tet's record is requested before the current
      // one's arithmetic, so its latency overlaps the work.
      uint32_t nextEntry = info.y ? __ldg(&b.adjacency[info.x]) : 0u;
      TetRec nextRec;
      bool nextOk = false;
  if (info.y) nextOk = incidentTetChecked(b.tets, nextEntry, b.tetTotal, b.vertexTotal, &nextRec);
#endif
      for (uint32_t a = 0; a < info.y; ++a) {
#if JGS2_CONV_LOOKAHEAD
        const uint32_t entry = nextEntry;
        const TetRec r = nextRec;
        const bool tetOk = nextOk;
        if (a + 1 < info.y) {
          nextEntry = __ldg(&b.adjacency[info.x + a + 1]);
          nextOk = incidentTetChecked(b.tets, nextEntry, b.tetTotal, b.vertexTotal, &nextRec);
        }
#else
        const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
        TetRec r;
        const bool tetOk = incidentTetChecked(b.tets, entry, b.tetTotal, b.vertexTotal, &r);
#endif
        if (!tetOk) continue;
        const M3 F = deformationAt(r, acc);
        const PiolaTerms pt = piolaTerms(F, r.lambda, r.mu);
        const float3 g = shapeGradient(r, entry & 3u);
        cadd(material, r.vol * mv(piola(F, pt), g));
        if (nextRotations) addIncidentBlock(hess, r, F, pt, g);
        avg = avg + r.vol * F;
        total += r.vol;
      }
      if (p.cloth) {
        const uint4 cr = b.clothRange[v];
        if (nextRotations)
          clothLocalSystem<true>(b.clothTris, b.clothHinges, b.clothIncidence, cr, acc, clothMaterial(p), 0u, 1u,
                                 material, hess);
        else
          clothLocalSystem<false>(b.clothTris, b.clothHinges, b.clothIncidence, cr, acc, clothMaterial(p), 0u, 1u,
                                  material, hess);
      }
      comps[1] = cvalue(material);
      comps[2] = f3(0, 0, 0);
      comps[3] = f3(0, 0, 0);
      if (p.objectiveFlags != 0u) {
        if (p.objectiveFlags & 1u) comps[2] = -xyz(b.forces[v]);
        if (p.objectiveFlags & 2u) {
          const float4 t = b.targets[v];
          if (t.w > 0.0f) comps[3] = t.w * (x - xyz(t));
        }
      }
      comps[4] = f3(0, 0, 0);
      if (p.floorStiffness > 0.0f && x.y < p.floorHeight) comps[4].y = p.floorStiffness * (x.y - p.floorHeight);
      if (p.ipc) comps[4] = comps[4] + xyz(b.contactGrad[v]);  // contactGradientKernel
      float3 totalG = f3(0, 0, 0);
      bool tv = true;
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const bool ok = finiteV(comps[c]);
        const float3 val = ok ? comps[c] : f3(0, 0, 0);
        part.scale[c] = fmaxf(part.scale[c], fmaxf(fabsf(val.x), fmaxf(fabsf(val.y), fabsf(val.z))));
        part.sq[c] += double(val.x) * val.x + double(val.y) * val.y + double(val.z) * val.z;
        totalG = totalG + val;
        tv = tv && ok;
      }
      tv = tv && finiteV(totalG);
      if (tv) {
        part.scale[5] = fmaxf(part.scale[5], fmaxf(fabsf(totalG.x), fmaxf(fabsf(totalG.y), fabsf(totalG.z))));
        part.sq[5] += double(totalG.x) * totalG.x + double(totalG.y) * totalG.y + double(totalG.z) * totalG.z;
      } else {
        part.valid = 0u;
      }
      // The next iteration's frame and incident system from the same
      // deformation gradients (the accepted pose is the next source).
      if (nextRotations) {
        const M3 favg = total > 0.0f ? (1.0f / total) * avg : midentity();
        storeFrame(b.vertexRot, v, info.y == 0u ? midentity() : polarRotation(favg, p.rotationEpsilon));
        storeIncident(b.incident, v, comps[1], hess);
      }
    } else if (nextRotations) {
      storeFrame(b.vertexRot, v, vertexFrame(b, acc, v, p.rotationEpsilon));
    }
  }
  const ConvPartial blk = blockFold(part, smem, convCombine);
  ConvPartial* partials = reinterpret_cast<ConvPartial*>(b.convPartials);
  if (!publishPartial(blk, partials, rb.slot, sr.convBlocks, &fs->convTicket, &isLast)) return;
  const ConvPartial tot = foldPartials(partials + sr.convBase, sr.convBlocks, smem, convIdentity, convCombine);
  if (threadIdx.x != 0) return;
  float norms[5];
  bool cnv = tot.valid != 0u;
  for (int c = 0; c < 5; ++c) {
    norms[c] = float(sqrt(tot.sq[c]));
    cnv = cnv && finiteS(norms[c]) && norms[c] >= 0.0f;
  }
  const float gnorm = float(sqrt(tot.sq[5]));
  const float den = fmaxf(1.0f, norms[0] + norms[1] + norms[2] + norms[3] + norms[4]);
  const float rel = gnorm / den;
  const bool rnv = cnv && finiteS(gnorm) && finiteS(den) && den >= 1.0f && finiteS(rel) && rel >= 0.0f;
  const float mu = tot.maxUpdate;
  const bool ssv = finiteS(p.sceneScale) && p.sceneScale >= 0.0f;
  const float nmu = mu / fmaxf(ssv ? p.sceneScale : 1.0e-12f, 1.0e-12f);
  const bool unv = tot.valid != 0u && ssv && finiteS(mu) && mu >= 0.0f && finiteS(nmu);
  const float4 geometry = fs->control[0];
  const uint32_t cb = controlBits(geometry.w) & kValidityMask;
  const bool sgv = (cb & kSourceGeometryValid) != 0u && finiteS(geometry.x);
  const bool cgv = (cb & kCandidateGeometryValid) != 0u && finiteS(geometry.y);
  const bool amv = (cb & kAcceptedMinimumValid) != 0u && finiteS(geometry.z);
  const bool lnv = (cb & kLocalNumericsValid) != 0u;
  const float4 accept = fs->control[1];
  const bool aav = finiteNonnegInt(accept.x, 1.0f), arv = finiteNonnegInt(accept.y, 1.0f);
  const bool lfv = finiteNonnegInt(accept.z, float(V));
  const bool hiv = finiteNonnegInt(accept.w, float(kHistoryCapacity));
  const bool aa = aav && accept.x == 1.0f, ar = arv && accept.y == 1.0f;
  const uint32_t failures = lfv ? static_cast<uint32_t>(accept.z) : 0u;
  const uint32_t hi = hiv ? static_cast<uint32_t>(accept.w) : 0u;
  const float4 cmx = fs->control[3];
  const bool cmv = finiteS(cmx.x) && cmx.x >= 0.0f && finiteNonnegInt(cmx.y, float(kMaxBacktracks)) &&
                   finiteNonnegInt(cmx.z, float(V) * float(kTrialCount)) &&
                   finiteNonnegInt(cmx.w, float(V) * float(kTrialCount));
  const bool fin = rnv && unv && sgv && cgv && amv && lnv && aav && arv && lfv && hiv && cmv;
  const bool rs = fin && rel <= p.residualTolerance;
  const bool us = fin && nmu <= p.normalizedUpdateTolerance;
  const bool conv = rs && us && aa && !ar && failures == 0u;
  if (hiv && hi < kHistoryCapacity) {
    float4* h = &fs->history[8 * hi];
    h[0] = fs->control[0];
    h[1] = make_float4(accept.x, accept.y, accept.z, ar ? 1.f : 0.f);
    h[2] = fs->control[2];
    h[3] = make_float4(cnv ? norms[0] : 0.f, cnv ? norms[1] : 0.f, cnv ? norms[2] : 0.f, cnv ? norms[3] : 0.f);
    h[4] = make_float4(cnv ? norms[4] : 0.f, rnv ? gnorm : 0.f, rnv ? den : 0.f, rnv ? rel : 0.f);
    h[5] = make_float4(unv ? mu : 0.f, unv ? nmu : 0.f, rs ? 1.f : 0.f, us ? 1.f : 0.f);
    h[6] = make_float4(conv ? 1.f : 0.f, fin ? 1.f : 0.f, float(hi), cmv ? cmx.x : 0.f);
    h[7] = make_float4(cmv ? cmx.y : 0.f, cmv ? cmx.z : 0.f, cmv ? cmx.w : 0.f, 1.f);
  }
  fs->control[1].w = float(hi + 1);
  if (conv && p.stopEnabled) fs->control[0].w = float(cb | kStopLatchBit);
  fs->convTicket = 0u;
}

// ---------------------------------------------------------------------------
// Epilogue: even-count copy (copyPosition, :4488-4496), optional body
// correction (:4498-4551), finalize (:4553-4589).
__global__ void __launch_bounds__(kBlock) bodyAccumulateKernel(Buffers b, const DevParams* __restrict__ pp,
                                                               const float4* __restrict__ finalPos, uint32_t V) {
  const uint32_t v = blockIdx.x * kBlock + threadIdx.x;
  if (v >= V || !pp[b.vertexScene[v]].active) return;
  float4 x = finalPos[v];
  if (finalPos != b.pos[0]) b.pos[0][v] = make_float4(x.x, x.y, x.z, 1.0f);
  const uint4 info = b.vinfo[v];
  const double m = fmax(double(b.restMass[v].w), 0.0);
  const float4 pr = b.predicted[v];
  // Per body: total mass, solved x/z moments, predicted x/z moments, pinned
  // count.  Double atomics: the summation order varies from run to run, so
  // the correction is reproducible to double rounding, not bitwise.
  double* acc = &b.bodyAccum[6ull * info.w];
  atomicAdd(&acc[0], m);
  atomicAdd(&acc[1], m * x.x);
  atomicAdd(&acc[2], m * x.z);
  atomicAdd(&acc[3], m * pr.x);
  atomicAdd(&acc[4], m * pr.z);
  if (isPinned(info)) atomicAdd(&acc[5], 1.0);
}

// accumulated: bodyAccumulateKernel ran (and left the final pose in pos[0]).
__global__ void __launch_bounds__(kBlock) finalizeKernel(Buffers b, const DevParams* __restrict__ pp,
                                                         const float4* __restrict__ finalPos, uint32_t V,
                                                         int accumulated) {
  const uint32_t v = blockIdx.x * kBlock + threadIdx.x;
  if (v >= V) return;
  const DevParams& p = pp[b.vertexScene[v]];
  if (!p.active) return;
  const uint4 info = b.vinfo[v];
  float4 x = accumulated ? b.pos[0][v] : finalPos[v];
  if (isPinned(info)) {
    if (!p.globalization) {
      const float4 rm = b.restMass[v];
      x = make_float4(rm.x, rm.y, rm.z, 1.0f);
    }
    b.pos[0][v] = make_float4(x.x, x.y, x.z, 1.0f);
    b.velocity[v] = make_float4(0, 0, 0, 0);
    return;
  }
  if (accumulated && p.bodyCorrection) {
    const double* acc = &b.bodyAccum[6ull * info.w];
    if (acc[5] == 0.0 && acc[0] > 0.0) {
      x.x += float((acc[3] - acc[1]) / acc[0]);
      x.z += float((acc[4] - acc[2]) / acc[0]);
    }
  }
  b.pos[0][v] = make_float4(x.x, x.y, x.z, 1.0f);
  const float3 o = xyz(b.old[v]);
  float3 vel = (xyz(x) - o) * p.invDt;
  if (p.floorStiffness > 0.0f && p.contactTangentialDamping > 0.0f && x.y <= p.floorHeight + p.contactMargin) {
    const float s = expf(-p.contactTangentialDamping * p.dt);
    vel.x *= s;
    vel.z *= s;
  }
  b.velocity[v] = make_float4(vel.x, vel.y, vel.z, 0.0f);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the gate.  Its reduction scratch is a static
// device array instead of solver buffers: a 256-byte header whose first word
// is the block ticket, then one GatePartial per block.  The ticket must be
// zero when a launch starts; module load zero-fills the array and the last
// block of every launch writes the ticket back to zero.  Two launches that
// overlap in time share the array and corrupt each other's result.
static_assert(sizeof(GatePartial) == kGatePartialBytes, "partial size");
static __device__ __align__(256) unsigned char gGateScratch[kGateScratchBytes];

// One element per thread (tet i and vertex i), so the grid, and with it the
// number of partials, grows with max(V, T); the launcher rejects sizes whose
// partials do not fit.  The sweep records are taken as cleared: no local
// failures, valid numerics, history slot 0, one skipped trial per vertex.
__global__ void __launch_bounds__(kBlock) gateScratchKernel(Buffers b, DevParams p, const float4* __restrict__ src,
                                                            const float4* __restrict__ tgt, uint32_t V, uint32_t T,
                                                            uint32_t C, uint32_t H, float4* __restrict__ control,
                                                            unsigned char* __restrict__ scratch) {
  __shared__ GatePartial smem[kBlock];
  __shared__ bool isLast;
  uint32_t* ticket = reinterpret_cast<uint32_t*>(scratch);
  GatePartial* partials = reinterpret_cast<GatePartial*>(scratch + kGateScratchHeaderBytes);
  GatePartial acc = gateIdentity();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < T) {
    const TetRec r = loadTet(b.tets, i);
    accumulateTet(acc, r, deformationAt(r, src), deformationAt(r, tgt));
  }
  if (i < V) {
    const uint4 info = b.vinfo[i];
    const float es = implicitEnergy(p, b, i, xyz(src[i]), info);
    const float ec = implicitEnergy(p, b, i, xyz(tgt[i]), info);
    if (finiteS(es)) acc.e0 += es; else acc.bits &= ~kSourceEnergyValid;
    if (finiteS(ec)) acc.e1 += ec; else acc.bits &= ~kCandidateEnergyValid;
  }
  if (i < C) accumulateClothTri(acc, loadClothTri(b.clothTris, i), src, tgt, clothMaterial(p));
  if (i < H) accumulateHinge(acc, b.clothHinges, i, src, tgt, p.clothBending);
  const GatePartial blk = blockFold(acc, smem, gateCombine);
  if (!publishPartial(blk, partials, blockIdx.x, gridDim.x, ticket, &isLast)) return;
  const GatePartial tot = foldPartials(partials, gridDim.x, smem, gateIdentity, gateCombine);
  if (threadIdx.x != 0) return;
  uint32_t vb = tot.bits | kLocalNumericsValid;
  const float eS = float(tot.e0), eC = float(tot.e1);
  if (!finiteS(eS)) vb &= ~kSourceEnergyValid;
  if (!finiteS(eC)) vb &= ~kCandidateEnergyValid;
  if (T == 0) vb &= ~(kSourceGeometryValid | kCandidateGeometryValid);
  const float sm = tot.minS, cm = tot.minC;
  const bool sgv = (vb & kSourceGeometryValid) != 0u, cgv = (vb & kCandidateGeometryValid) != 0u;
  const bool sev = (vb & kSourceEnergyValid) != 0u, cev = (vb & kCandidateEnergyValid) != 0u;
  const bool accepted = (sgv && sm > kDeterminantFloor) && (cgv && cm > kDeterminantFloor);
  const float am = accepted ? cm : sm;
  const bool amv = accepted ? cgv : sgv;
  const float ae = accepted ? eC : eS;
  const bool aev = accepted ? cev : sev;
  if (amv) vb |= kAcceptedMinimumValid;
  const uint32_t cb = vb & kValidityMask;
  control[0] = make_float4(sgv ? sm : 0.f, cgv ? cm : 0.f, amv ? am : 0.f, float(cb));
  control[1] = make_float4(accepted ? 1.f : 0.f, accepted ? 0.f : 1.f, 0.f, 0.f);
  control[2] = make_float4(sev ? eS : 0.f, cev ? eC : 0.f, aev ? ae : 0.f, (sev && cev) ? 1.f : 0.f);
  control[3] = make_float4(0.f, 0.f, float(V), 0.f);
  *ticket = 0u;
}

}  // namespace

// ---------------------------------------------------------------------------
// Exact all-element oracle diagnostics (JGS2GpuOracleEvaluator,
// jgs2-diagnostics.ts:388-1146): per tet its frozen frame (the step's
// seven-step polar), energy, determinant and finiteness; per vertex the exact
// active-coordinate gradient, the diagonal block of the frozen global
// Hessian, the inertia, objective and floor energies and norms; one
// fixed-order reduction.  Opt-in; the frame loop never runs it.

__device__ __forceinline__ float finiteOr0(float v) { return finiteS(v) ? v : 0.0f; }
__device__ __forceinline__ float4 finite4(float3 v, float w) {
  return make_float4(finiteOr0(v.x), finiteOr0(v.y), finiteOr0(v.z), w);
}

// Co-rotated displacement of a tet's vertices in its frame R:
// R^T (x_l - centroid) - (X_l - rest centroid).
__device__ __forceinline__ void oracleDisplacement(const Buffers& b, const float4* __restrict__ x, const uint4& q,
                                                   const M3& R, float3 d[4], bool* finite) {
  float3 cur[4], rest[4];
  float3 cc = f3(0, 0, 0), rc = f3(0, 0, 0);
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const uint32_t v = idxAt(q, l);
    cur[l] = xyz(x[v]);
    rest[l] = xyz(b.restMass[v]);
    cc = cc + 0.25f * cur[l];
    rc = rc + 0.25f * rest[l];
  }
  const M3 Rt = mtrans(R);
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    d[l] = mv(Rt, cur[l] - cc) - (rest[l] - rc);
    *finite = *finite && finiteV(cur[l]) && finiteV(rest[l]) && finiteV(d[l]);
  }
}

__global__ void __launch_bounds__(kBlock) oracleTetKernel(Buffers b, OracleParams q, const float4* __restrict__ x,
                                                          float4* __restrict__ rot, float4* __restrict__ metric) {
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= q.T) return;
  const uint32_t t = q.tOff + k;
  const TetRec r = loadTet(b.tets, t);
  const M3 F = deformationAt(r, x);
  const float det = mdet(F);
  const M3 R = polarRotation(F, q.rotationEpsilon);
  bool finite = finiteM(F) && finiteS(det) && finiteM(R);
  float energy = 0.0f;
  if (q.corotated) {
    float3 d[4];
    oracleDisplacement(b, x, r.idx, R, d, &finite);
    const float* K = b.stiffness + 144ull * t;
#pragma unroll
    for (int row = 0; row < 4; ++row) {
      float3 lg = f3(0, 0, 0);
#pragma unroll
      for (int col = 0; col < 4; ++col) lg = lg + mv(stiffnessBlock(K, row, col), d[col]);
      finite = finite && finiteV(lg);
      energy += 0.5f * dot3(d[row], lg);
    }
  } else {
    energy = r.vol * snhEnergy(F, r.lambda, r.mu);
    const PiolaTerms pt = piolaTerms(F, r.lambda, r.mu);
    finite = finite && finiteM(piola(F, pt));
  }
  finite = finite && finiteS(energy);
  rot[3ull * k] = finite4(R.c0, 0.0f);
  rot[3ull * k + 1] = finite4(R.c1, 0.0f);
  rot[3ull * k + 2] = finite4(R.c2, 0.0f);
  metric[k] = make_float4(finiteOr0(energy), finiteOr0(det), finite ? 1.0f : 0.0f, 0.0f);
}

__global__ void __launch_bounds__(kBlock) oracleVertexKernel(Buffers b, OracleParams q, const float4* __restrict__ x,
                                                             const float4* __restrict__ rot,
                                                             float4* __restrict__ rec) {
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= q.V) return;
  const uint32_t v = q.vOff + k;
  const uint4 info = b.vinfo[v];
  const float4 rm = b.restMass[v];
  const float3 cur = xyz(x[v]), pred = xyz(b.predicted[v]);
  const float3 diff = cur - pred;
  const float update = b.finalUpdate[v];
  const float floorDistance = cur.y - q.floorHeight;
  const bool active = !isPinned(info);
  float3 grad = f3(0, 0, 0), gIn = f3(0, 0, 0), gEl = f3(0, 0, 0), gExt = f3(0, 0, 0), gTgt = f3(0, 0, 0);
  float3 gFloor = f3(0, 0, 0);
  M3 H = mzero();
  float eIn = 0.0f, eExt = 0.0f, eTgt = 0.0f, eFloor = 0.0f, weight = 0.0f, mag = 0.0f;
  bool updateValid = false, floorActive = false;
  bool finite = finiteV(cur) && finiteV(pred) && finiteV(xyz(rm)) && finiteS(rm.w) && finiteS(update) &&
                finiteS(floorDistance);
  if (active) {
    weight = rm.w * q.invDt2;
    gIn = weight * diff;
    grad = gIn;
    H = weight * midentity();
    eIn = 0.5f * weight * dot3(diff, diff);
    mag = update;
    updateValid = update >= 0.0f;
    const float3 force = (q.objectiveFlags & 1u) ? xyz(b.forces[v]) : f3(0, 0, 0);
    gExt = -1.0f * force;
    eExt = -dot3(force, cur);
    grad = grad + gExt;
    const float4 target = (q.objectiveFlags & 2u) ? b.targets[v] : make_float4(0, 0, 0, 0);
    finite = finite && finiteV(force) && finiteS(target.w) && target.w >= 0.0f;
    if (target.w > 0.0f) {
      finite = finite && finiteV(xyz(target));
      const float3 res = cur - xyz(target);
      gTgt = target.w * res;
      eTgt = 0.5f * target.w * dot3(res, res);
      grad = grad + gTgt;
      H = H + target.w * midentity();
    }
    for (uint32_t a = 0; a < info.y; ++a) {
      const uint32_t entry = __ldg(&b.adjacency[info.x + a]);
      const uint32_t t = entry >> 2, slot = entry & 3u;
      const TetRec r = loadTet(b.tets, t);
      if (q.corotated) {
        const uint32_t kt = t - q.tOff;
        const M3 R = {xyz(rot[3ull * kt]), xyz(rot[3ull * kt + 1]), xyz(rot[3ull * kt + 2])};
        float3 d[4];
        oracleDisplacement(b, x, r.idx, R, d, &finite);
        const float* K = b.stiffness + 144ull * t;
        float3 lg = f3(0, 0, 0);
#pragma unroll
        for (int col = 0; col < 4; ++col) lg = lg + mv(stiffnessBlock(K, slot, col), d[col]);
        gEl = gEl + mv(R, lg);
        H = H + mm(mm(R, stiffnessBlock(K, slot, slot)), mtrans(R));
      } else {
        const M3 F = deformationAt(r, x);
        const PiolaTerms pt = piolaTerms(F, r.lambda, r.mu);
        const float3 g = shapeGradient(r, slot);
        gEl = gEl + r.vol * mv(piola(F, pt), g);
        S3 blk = szero();
        addIncidentBlock(blk, r, F, pt, g);
        H.c0 = H.c0 + f3(blk.xx, blk.xy, blk.xz);
        H.c1 = H.c1 + f3(blk.xy, blk.yy, blk.yz);
        H.c2 = H.c2 + f3(blk.xz, blk.yz, blk.zz);
      }
    }
    grad = grad + gEl;
    floorActive = q.floorStiffness > 0.0f && floorDistance < 0.0f;
    if (floorActive) {
      eFloor = 0.5f * q.floorStiffness * floorDistance * floorDistance;
      gFloor.y = q.floorStiffness * floorDistance;
      grad = grad + gFloor;
      H.c1.y += q.floorStiffness;
    }
  }
  const float gSq = dot3(grad, grad), inSq = dot3(gIn, gIn), elSq = dot3(gEl, gEl), flSq = dot3(gFloor, gFloor);
  finite = finite && finiteS(weight) && finiteS(eIn) && finiteS(eExt) && finiteS(eTgt) && finiteS(eFloor) &&
           finiteS(mag) && finiteV(grad) && finiteV(gIn) && finiteV(gEl) && finiteV(gExt) && finiteV(gTgt) &&
           finiteV(gFloor) && finiteM(H) && finiteS(gSq) && finiteS(inSq) && finiteS(elSq) &&
           finiteS(dot3(gExt, gExt)) && finiteS(dot3(gTgt, gTgt)) && finiteS(flSq);
  float4* o = rec + 9ull * k;
  o[0] = finite4(grad, active ? 1.0f : 0.0f);
  // Rows of the (symmetric) block with the energies beside them.
  o[1] = make_float4(finiteOr0(H.c0.x), finiteOr0(H.c1.x), finiteOr0(H.c2.x), finiteOr0(eIn));
  o[2] = make_float4(finiteOr0(H.c0.y), finiteOr0(H.c1.y), finiteOr0(H.c2.y), finiteOr0(eFloor));
  o[3] = make_float4(finiteOr0(H.c0.z), finiteOr0(H.c1.z), finiteOr0(H.c2.z), finiteOr0(mag));
  o[4] = make_float4(finiteOr0(gSq), finite ? 1.0f : 0.0f, finiteOr0(weight), updateValid ? 1.0f : 0.0f);
  o[5] = make_float4(finiteOr0(inSq), finiteOr0(elSq), finiteOr0(flSq), finiteOr0(floorDistance));
  o[6] = make_float4(floorActive ? 1.0f : 0.0f, 0.0f, 0.0f, 0.0f);
  o[7] = finite4(gExt, finiteOr0(eExt));
  o[8] = finite4(gTgt, finiteOr0(eTgt));
}

// reduceDiagnostics in one block: each thread folds a fixed stride of the
// records in double, then a fixed-order tree; deterministic.
__global__ void __launch_bounds__(1024) oracleReduceKernel(OracleParams q, const float4* __restrict__ metric,
                                                           const float4* __restrict__ rec, double* out) {
  __shared__ double sh[1024];
  double acc[kOracleSummaryWords];
#pragma unroll
  for (int i = 0; i < kOracleSummaryWords; ++i) acc[i] = 0.0;
  acc[11] = 0.0;                 // largest update
  acc[12] = 3.0e38;              // smallest determinant
  acc[13] = 3.0e38;              // smallest floor distance
  acc[16] = 1.0;                 // all active updates valid
  acc[17] = 1.0;                 // all finite
  for (uint32_t t = threadIdx.x; t < q.T; t += blockDim.x) {
    const float4 m = metric[t];
    acc[1] += m.x;
    acc[12] = fmin(acc[12], double(m.y));
    if (!(m.z >= 0.5f)) acc[17] = 0.0;
  }
  for (uint32_t v = threadIdx.x; v < q.V; v += blockDim.x) {
    const float4* o = rec + 9ull * v;
    const float4 g = o[0], r0 = o[1], r1 = o[2], r2 = o[3], m = o[4], c = o[5], fl = o[6], ext = o[7], tg = o[8];
    const bool active = g.w >= 0.5f;
    acc[0] += r0.w;
    acc[2] += ext.w;
    acc[3] += tg.w;
    acc[4] += r1.w;
    acc[5] += m.x;
    acc[6] += c.x;
    acc[7] += c.y;
    acc[8] += double(ext.x) * ext.x + double(ext.y) * ext.y + double(ext.z) * ext.z;
    acc[9] += double(tg.x) * tg.x + double(tg.y) * tg.y + double(tg.z) * tg.z;
    acc[10] += c.z;
    if (active) {
      acc[11] = fmax(acc[11], double(r2.w));
      acc[13] = fmin(acc[13], double(c.w));
      acc[15] += fl.x >= 0.5f ? 1.0 : 0.0;
      if (!(m.w >= 0.5f)) acc[16] = 0.0;
      acc[14] += 1.0;
    }
    if (!(m.y >= 0.5f)) acc[17] = 0.0;
  }
  for (int i = 0; i < kOracleSummaryWords; ++i) {
    sh[threadIdx.x] = acc[i];
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const double a = sh[threadIdx.x], c = sh[threadIdx.x + o];
        sh[threadIdx.x] = (i == 11) ? fmax(a, c) : (i == 12 || i == 13 || i == 16 || i == 17) ? fmin(a, c) : a + c;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = sh[0];
    __syncthreads();
  }
}

inline uint32_t blocksFor(uint32_t n) { return (n + kBlock - 1) / kBlock; }

uint32_t smCount() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return static_cast<uint32_t>(sms);
}

int launchPrologue(const Buffers& b, const DevParams* p, cudaStream_t s) {
  prologueKernel<<<b.gateBlocks, kBlock, 0, s>>>(b, p);
  return 1;
}

int launchTetPolar(const Buffers& b, const DevParams* p, const float4* src, uint32_t T, cudaStream_t s) {
  if (T == 0) return 0;
  tetPolarKernel<<<blocksFor(T), kBlock, 0, s>>>(b, p, src, T);
  return 1;
}

int launchCorotatedSolve(const Buffers& b, const DevParams* p, const float4* src, float4* tgt, const uint32_t* list,
                         uint32_t count, uint32_t K, cudaStream_t s) {
  if (count == 0) return 0;
  corotatedSolveKernel<<<blocksFor(count), kBlock, 0, s>>>(b, p, src, tgt, list, count, K);
  return 1;
}

int launchVertexPolar(const Buffers& b, const DevParams* p, const float4* src, const uint32_t* list,
                      uint32_t count, cudaStream_t s) {
  if (count == 0) return 0;
  vertexPolarKernel<<<blocksFor(count), kBlock, 0, s>>>(b, p, src, list, count);
  return 1;
}

int launchSolve(const Buffers& b, const DevParams* p, const float4* src, float4* tgt, const uint32_t* list,
                uint32_t count, uint32_t K, bool cachedIncident, cudaStream_t s) {
  if (count == 0) return 0;
  const bool cache = solveCachesRecords(K);
  const uint32_t fit = solveGroupsPerBlock(K);
  if (fit == 0) return 0;
  const uint32_t shift = std::min(b.solveShift, 2u);
  const uint32_t groups = std::max(1u, fit >> shift);
  const size_t smem = cache ? static_cast<size_t>(groups) * K * kSolveSlotBytes : 0;
  constexpr uint32_t perWarp = 32u / kGroup;
  const uint32_t threads = (groups + perWarp - 1) / perWarp * 32u;
  // One vertex per lane group: the line search makes per-vertex work uneven,
  // and the block scheduler balances it better than a fixed grid stride.
  const uint32_t blocks = std::max(1u, (count + groups - 1) / groups);
  // Contact-heavy engines (more than 64 candidate incidences of the static
  // superset per solved vertex on average, listed or not): a whole warp per
  // vertex over its active candidates.  A broad-phase engine decides on the
  // superset too, so it runs the variant its static twin runs.
  const uint64_t superset = b.contactDynamic ? b.bpSuperset : b.contactCount;
  const int ci = cachedIncident ? 1 : 0;
  if (b.contactIdx && superset * 4u > uint64_t(64) * count) {
    // Warps per block: an eighth of the vertices a 4-lane block of the same
    // cache budget would take (at most a full block).
    const uint32_t perVertex = static_cast<uint32_t>(K * kSolveSlotBytes);
    const uint32_t fit4 = std::min<uint32_t>(32u, (cache && perVertex) ? solveSharedBytes() / perVertex : 32u);
    const uint32_t wg = std::max(1u, std::min(std::max(1u, fit4 >> shift) * 4u / 32u, kBlock / 32u));
    const size_t wsmem = cache ? static_cast<size_t>(wg) * K * kSolveSlotBytes : 0;
    const uint32_t wb = std::max(1u, (count + wg - 1) / wg);
    if (cache)
      solveKernel<32, true, true><<<wb, wg * 32, wsmem, s>>>(b, p, src, tgt, list, count, K, ci, wg);
    else
      solveKernel<32, true, false><<<wb, wg * 32, 0, s>>>(b, p, src, tgt, list, count, K, ci, wg);
  } else if (b.clothRange || b.contactIdx) {
    if (cache) solveKernel<kGroup, true, true><<<blocks, threads, smem, s>>>(b, p, src, tgt, list, count, K, ci, groups);
    else solveKernel<kGroup, true, false><<<blocks, threads, 0, s>>>(b, p, src, tgt, list, count, K, ci, groups);
  } else {
    if (cache) solveKernel<kGroup, false, true><<<blocks, threads, smem, s>>>(b, p, src, tgt, list, count, K, ci, groups);
    else solveKernel<kGroup, false, false><<<blocks, threads, 0, s>>>(b, p, src, tgt, list, count, K, ci, groups);
  }
  return 1;
}

// Dynamic shared memory a solve block may use (the device's opt-in limit less
// the kernel's static shared memory); sets the kernels' attribute once.
int launchColoredSweep(const Buffers& b, const DevParams* p, float4* x, const uint32_t* colorVertices,
                       const uint32_t* colorOffsets, const uint32_t* needVertices, const uint32_t* needOffsets,
                       uint32_t colorCount, uint32_t V, uint32_t K, uint32_t largestColor, uint32_t largestNeed,
                       bool refreshAllFrames, void* barrier, uint32_t spinLimit, cudaStream_t s) {
  const uint32_t fit = solveGroupsPerBlock(K);
  if (fit == 0 || colorCount == 0) return 0;
  if (!solveCachesRecords(K)) return -1;  // the sweep kernel caches records
  const uint32_t groups = std::max(1u, fit >> std::min(b.solveShift, 2u));
  const size_t smem = static_cast<size_t>(groups) * K * kSolveSlotBytes;
  constexpr uint32_t perWarp = 32u / kGroup;
  const uint32_t threads = (groups + perWarp - 1) / perWarp * 32u;
  const bool ext = b.clothRange || b.contactIdx;
  const void* fn = ext ? reinterpret_cast<const void*>(coloredSweepKernel<kGroup, true>)
                       : reinterpret_cast<const void*>(coloredSweepKernel<kGroup, false>);
  static int attr = -1;
  if (attr < 0) {
    attr = static_cast<int>(solveSharedBytes());
    cudaFuncSetAttribute(coloredSweepKernel<kGroup, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, attr);
    cudaFuncSetAttribute(coloredSweepKernel<kGroup, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, attr);
  }
  int device = 0, sms = 0, perSm = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, static_cast<int>(threads), smem) != cudaSuccess ||
      perSm <= 0 || sms <= 0)
    return -1;
  // As many blocks as the widest phase can use: every colour's solves in one
  // wave of chunks (else the launch-per-colour encoding is the better one),
  // the frames spread at one vertex per thread.
  const uint32_t capacity = static_cast<uint32_t>(perSm * sms);
  const uint32_t chunks = (largestColor + groups - 1) / groups;
  if (chunks > capacity) return -1;
  const uint32_t frameBlocks = (std::max(largestNeed, refreshAllFrames ? V : 0u) + threads - 1) / threads;
  const uint32_t grid = std::max(1u, std::min(capacity, std::max(chunks, frameBlocks)));
  // A cooperative grid: every block resident, so the barriers can complete.
  cudaMemsetAsync(barrier, 0, sizeof(SweepBarrier), s);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  SweepBarrier* bar = static_cast<SweepBarrier*>(barrier);
  const int all = refreshAllFrames ? 1 : 0;
  cudaError_t e;
  if (ext)
    e = cudaLaunchKernelEx(&cfg, coloredSweepKernel<kGroup, true>, b, p, x, colorVertices, colorOffsets, needVertices,
                           needOffsets, colorCount, V, K, groups, all, bar, spinLimit);
  else
    e = cudaLaunchKernelEx(&cfg, coloredSweepKernel<kGroup, false>, b, p, x, colorVertices, colorOffsets,
                           needVertices, needOffsets, colorCount, V, K, groups, all, bar, spinLimit);
  return e == cudaSuccess ? 2 : -1;
}

size_t sweepBarrierBytes() { return sizeof(SweepBarrier); }

bool boundsChecked() { return JGS2_BOUNDS_CHECKS != 0; }

cudaError_t takeBoundsViolation(uint32_t* site) {
  *site = 0;
#if JGS2_BOUNDS_CHECKS
  cudaError_t e = cudaMemcpyFromSymbol(site, gBoundsViolation, sizeof(uint32_t));
  if (e != cudaSuccess || *site == 0) return e;
  const uint32_t zero = 0;
  return cudaMemcpyToSymbol(gBoundsViolation, &zero, sizeof(uint32_t));
#else
  return cudaSuccess;
#endif
}

uint32_t solveSharedBytes() {
  static int optin = -1;
  if (optin < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) optin = 48 * 1024;
    optin -= 1024;  // static shared memory of the kernel
    cudaFuncSetAttribute(solveKernel<kGroup, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    cudaFuncSetAttribute(solveKernel<kGroup, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    cudaFuncSetAttribute(solveKernel<32, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  }
  return static_cast<uint32_t>(optin);
}

bool solveCachesRecords(uint32_t K) { return static_cast<size_t>(K) * kSolveSlotBytes <= kSolveCacheBytesPerVertex; }

uint32_t solveGroupsPerBlock(uint32_t K) {
  // Shared memory holds one cached record state per cubature record of each
  // vertex in the block; wide records are recomputed instead of cached.
  uint32_t groups = (kBlock / 32) * (32 / kGroup);
  if (!solveCachesRecords(K)) return groups;
  const uint32_t perVertex = static_cast<uint32_t>(K * kSolveSlotBytes);
  if (perVertex > 0) groups = std::min<uint32_t>(groups, solveSharedBytes() / perVertex);
  return groups;
}

int launchContactLag(const Buffers& b, const DevParams* p, cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactLagKernel<<<blocksFor(b.contactCount), kBlock, 0, s>>>(b, p);
  return 1;
}

int launchContactRows(const Buffers& b, const DevParams* p, const float4* src, uint32_t V, cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactFlagKernel<<<blocksFor(b.contactCount), kBlock, 0, s>>>(b, p, src);
  contactRowsKernel<<<(V + kBlock / 32 - 1) / (kBlock / 32), kBlock, 0, s>>>(b, p, V);
  return 2;
}

int launchContactGradient(const Buffers& b, const DevParams* p, const float4* src, const float4* tgt, uint32_t V,
                          cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactGradientKernel<<<(V + kBlock / 32 - 1) / (kBlock / 32), kBlock, 0, s>>>(b, p, src, tgt, V);
  return 1;
}

// Candidate kernels: one thread per static candidate, or a grid that strides
// over the broad phase's list (its count is on the device).
uint32_t candidateBlocks(const Buffers& b) {
  const uint32_t n = blocksFor(b.contactCount);
  return b.contactDynamic ? std::min(n, smCount() * 16u) : n;
}

int launchContactStep(const Buffers& b, const DevParams* p, const float4* src, const float4* tgt, cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactStepKernel<<<candidateBlocks(b), kBlock, 0, s>>>(b, p, src, tgt);
  return 1;
}

int launchContactApply(const Buffers& b, const DevParams* p, const float4* src, float4* tgt, uint32_t V,
                       bool validated, cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactApplyKernel<<<blocksFor(V), kBlock, 0, s>>>(b, p, src, tgt, V, validated ? 1 : 0);
  return 1;
}

int launchContactValidate(const Buffers& b, const DevParams* p, const float4* tgt, cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactValidateKernel<<<candidateBlocks(b), kBlock, 0, s>>>(b, p, tgt);
  return 1;
}

int launchContactFeatures(const float* points, const uint32_t* types, uint32_t n, float* out, uint32_t* wide,
                          cudaStream_t s) {
  if (n == 0) return 0;
  contactFeatureKernel<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(points, types, n, out, wide);
  return 1;
}

int launchContactPromote(const Buffers& b, const DevParams* p, cudaStream_t s) {
  if (b.contactCount == 0) return 0;
  contactPromoteKernel<<<candidateBlocks(b), kBlock, 0, s>>>(b, p);
  return 1;
}

uint32_t broadPhaseSortPasses(uint32_t V) {
  uint32_t bits = 1;
  while (bits < 32 && (V >> bits) != 0u) ++bits;  // keys 0..V, the sentinel V included
  return (bits + 7) / 8;
}

int launchBroadPhase(const Buffers& b, const DevParams* p, const float4* src, uint32_t V, bool first,
                     cudaStream_t s) {
  if (!b.contactDynamic || b.contactCount == 0) return 0;
  const uint32_t triBlocks = blocksFor(b.bpTriTotal), edgeBlocks = blocksFor(b.bpEdgeTotal);
  bpBoxesKernel<<<triBlocks + edgeBlocks + blocksFor(V), kBlock, 0, s>>>(b, p, src, triBlocks, edgeBlocks, V);
  const uint32_t triSupers = (b.bpTriTotal + kBpChunk * kBpChunk - 1) / (kBpChunk * kBpChunk);
  const uint32_t edgeSupers = (b.bpEdgeTotal + kBpChunk * kBpChunk - 1) / (kBpChunk * kBpChunk);
  bpSuperKernel<<<(triSupers + edgeSupers + kBlock / 32 - 1) / (kBlock / 32), kBlock, 0, s>>>(b, triSupers,
                                                                                              edgeSupers);
  const uint32_t rowBlocks = (b.bpRowTotal + kBlock / 32 - 1) / (kBlock / 32);
  const int f = first ? 1 : 0;
  bpRowsKernel<false><<<rowBlocks, kBlock, 0, s>>>(b, p, src, f);
  bpScanKernel<<<1, kScanThreads, 0, s>>>(b, p, f);
  bpRowsKernel<true><<<rowBlocks, kBlock, 0, s>>>(b, p, src, f);
  bpInitKernel<<<candidateBlocks(b), kBlock, 0, s>>>(b, p, src, f);
  const uint32_t tiles = static_cast<uint32_t>((4ull * b.contactCount + kSortTile - 1) / kSortTile);
  for (uint32_t pass = 0; pass < b.bpSortPasses; ++pass) {
    const uint32_t in = pass & 1u, out = in ^ 1u;
    bpSortHistKernel<<<tiles, kSortThreads, 0, s>>>(b.bpKeys[in], b.bpStatus, 8u * pass, b.bpHist);
    bpSortScanKernel<<<256, kScanThreads, 0, s>>>(b.bpStatus, b.bpHist);
    bpSortScatterKernel<<<tiles, kSortThreads, 0, s>>>(b.bpKeys[in], b.bpVals[in], b.bpKeys[out], b.bpVals[out],
                                                       b.bpStatus, 8u * pass, b.bpHist);
  }
  const uint32_t segBlocks = std::min(blocksFor(4u * b.contactCount), smCount() * 8u);
  bpSegmentsKernel<<<segBlocks, kBlock, 0, s>>>(b, b.bpKeys[b.bpSortPasses & 1u]);
  return 7 + 3 * static_cast<int>(b.bpSortPasses);
}

int launchOracleDiagnostics(const Buffers& b, const OracleParams& q, float4* tetRot, float4* tetMetric,
                            float4* vertexRecords, double* summary, cudaStream_t s) {
  int n = 0;
  if (q.T) {
    oracleTetKernel<<<blocksFor(q.T), kBlock, 0, s>>>(b, q, b.pos[0], tetRot, tetMetric);
    ++n;
  }
  if (q.V) {
    oracleVertexKernel<<<blocksFor(q.V), kBlock, 0, s>>>(b, q, b.pos[0], tetRot, vertexRecords);
    ++n;
  }
  oracleReduceKernel<<<1, 1024, 0, s>>>(q, tetMetric, vertexRecords, summary);
  return n + 1;
}

int launchCopy(const Buffers& b, const DevParams* p, const float4* src, float4* dst, uint32_t V, cudaStream_t s) {
  copyKernel<<<blocksFor(V), kBlock, 0, s>>>(b, p, src, dst, V);
  return 1;
}

int launchGate(const Buffers& b, const DevParams* p, const float4* src, const float4* tgt, cudaStream_t s) {
  if (b.clothRange || b.contactIdx)
    gateKernel<true><<<b.gateBlocks, kBlock, 0, s>>>(b, p, src, tgt);
  else
    gateKernel<false><<<b.gateBlocks, kBlock, 0, s>>>(b, p, src, tgt);
  return 1;
}

int launchConvergence(const Buffers& b, const DevParams* p, const float4* src, float4* tgt,
                      bool computeNextRotations, cudaStream_t s) {
  convergenceKernel<<<b.convBlocks, kBlock, 0, s>>>(b, p, src, tgt, computeNextRotations ? 1 : 0);
  return 1;
}

int launchEpilogue(const Buffers& b, const DevParams* p, const float4* finalPos, uint32_t V, bool bodyCorrection,
                   uint32_t bodies, cudaStream_t s) {
  int n = 0;
  if (bodyCorrection) {
    cudaMemsetAsync(b.bodyAccum, 0, sizeof(double) * 6ull * bodies, s);
    bodyAccumulateKernel<<<blocksFor(V), kBlock, 0, s>>>(b, p, finalPos, V);
    ++n;
  }
  finalizeKernel<<<blocksFor(V), kBlock, 0, s>>>(b, p, finalPos, V, bodyCorrection ? 1 : 0);
  return n + 1;
}

cudaError_t gateScratchAddress(void** out) { return cudaGetSymbolAddress(out, gGateScratch); }

uint32_t gateScratchMaxElements() { return kGateScratchMaxBlocks * static_cast<uint32_t>(kBlock); }

int launchGateScratch(const Buffers& b, const DevParams& p, const float4* predicted, const float4* src,
                      const float4* tgt, uint32_t V, uint32_t T, uint32_t C, uint32_t H, float4* control,
                      void* scratch, cudaStream_t s) {
  const uint32_t n = std::max(std::max(T, V), std::max(C, H));
  if (n == 0 || n > gateScratchMaxElements()) return 0;
  Buffers view = b;
  view.predicted = const_cast<float4*>(predicted);
  gateScratchKernel<<<blocksFor(n), kBlock, 0, s>>>(view, p, src, tgt, V, T, C, H, control,
                                                   static_cast<unsigned char*>(scratch));
  return 1;
}

}  // namespace jgs2
