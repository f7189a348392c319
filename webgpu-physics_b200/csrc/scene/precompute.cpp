// JGS2 precompute: exact full-coordinate bases and nonlinear cubature
// training, restated from
//   src/simulation/cpu/fem.ts:238-335            (rest linear system)
//   src/simulation/cpu/precompute.ts:141-206     (computeExactVertexBasis)
//   src/simulation/cpu/cubature.ts:55-297        (low-frequency modes)
//   src/simulation/cpu/cubature.ts:371-690       (greedy NNLS selection)
//   src/simulation/cpu/cubature.ts:312-369, 714-820 (co-rotated linear training)
//   src/simulation/cpu/nonlinear-cubature.ts:140-620 (pose corpus)
//   src/simulation/cpu/nonlinear-cubature-training.ts:189-843 (training)
//
// The same routines run either on the whole mesh (the reference's method) or
// on a local patch around each source vertex, with patches of identical
// signature sharing one training result.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <unordered_map>

#include "scene_internal.hpp"
#include "select_gpu.hpp"

namespace jgs2scene {
namespace {

constexpr double kMinimumPoseDeterminant = 0.5;        // nonlinear-cubature.ts:24
constexpr uint32_t kValidationOnlyModes = 4;           // nonlinear-cubature.ts:14
constexpr int kLinearRefinementPasses = 4;             // cubature.ts:52

// ---- dense linear algebra -------------------------------------------------

// choleskyFactor (src/simulation/cpu/math.ts:56-99).
bool choleskyFactor(const std::vector<double>& a, int n, std::vector<double>& L) {
  L.assign(static_cast<size_t>(n) * n, 0.0);
  double largest = 0;
  for (int i = 0; i < n; ++i) largest = std::max(largest, std::fabs(a[static_cast<size_t>(i) * n + i]));
  const double tol = std::max(largest, 1.0) * 1e-13;
  for (int r = 0; r < n; ++r) {
    double* Lr = &L[static_cast<size_t>(r) * n];
    for (int c = 0; c <= r; ++c) {
      const double* Lc = &L[static_cast<size_t>(c) * n];
      double v = a[static_cast<size_t>(r) * n + c];
      for (int k = 0; k < c; ++k) v -= Lr[k] * Lc[k];
      if (r == c) {
        if (!(v > tol) || !std::isfinite(v)) return false;
        Lr[c] = std::sqrt(v);
      } else {
        Lr[c] = v / Lc[c];
      }
    }
  }
  return true;
}

// solveCholesky (src/simulation/cpu/math.ts:101-132).
void solveCholesky(const std::vector<double>& L, int n, const double* rhs, double* x) {
  for (int r = 0; r < n; ++r) {
    const double* Lr = &L[static_cast<size_t>(r) * n];
    double v = rhs[r];
    for (int c = 0; c < r; ++c) v -= Lr[c] * x[c];
    x[r] = v / Lr[r];
  }
  for (int r = n - 1; r >= 0; --r) {
    double v = x[r];
    for (int c = r + 1; c < n; ++c) v -= L[static_cast<size_t>(c) * n + r] * x[c];
    x[r] = v / L[static_cast<size_t>(r) * n + r];
  }
}

double dotv(const double* a, const double* b, size_t n) {
  double s = 0;
  for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

// canonicalizeVectorSign (src/simulation/cpu/cubature.ts:55-67).
void canonicalizeLargest(std::vector<double>& v) {
  size_t big = 0;
  for (size_t i = 1; i < v.size(); ++i)
    if (std::fabs(v[i]) > std::fabs(v[big])) big = i;
  if (!v.empty() && v[big] < 0)
    for (double& x : v) x = -x;
}

// orthonormalizeBlock (src/simulation/cpu/cubature.ts:69-122).
std::vector<std::vector<double>> orthonormalizeBlock(const std::vector<std::vector<double>>& in,
                                                     int n) {
  std::vector<std::vector<double>> out;
  for (size_t ci = 0; ci < in.size(); ++ci) {
    std::vector<double> cand = in[ci];
    for (int pass = 0; pass < 2; ++pass)
      for (const auto& b : out) {
        const double p = dotv(cand.data(), b.data(), n);
        for (int r = 0; r < n; ++r) cand[r] -= p * b[r];
      }
    double norm = std::sqrt(dotv(cand.data(), cand.data(), n));
    if (norm <= 1e-11) {
      bool found = false;
      for (int off = 0; off < n && !found; ++off) {
        std::vector<double> trial(n, 0.0);
        trial[(ci + off) % n] = 1;
        for (const auto& b : out) {
          const double p = dotv(trial.data(), b.data(), n);
          for (int r = 0; r < n; ++r) trial[r] -= p * b[r];
        }
        const double tn = std::sqrt(dotv(trial.data(), trial.data(), n));
        if (tn > 1e-11) {
          for (double& x : trial) x /= tn;
          cand = trial;
          found = true;
        }
      }
      if (!found) throw std::runtime_error("Could not construct the requested low-frequency basis.");
      norm = 1;
    }
    for (double& x : cand) x /= norm;
    canonicalizeLargest(cand);
    out.push_back(std::move(cand));
  }
  return out;
}

// jacobiSymmetricEigendecomposition (src/simulation/cpu/cubature.ts:130-218).
void jacobiEigen(std::vector<double> a, int n, std::vector<double>& values,
                 std::vector<double>& vectors) {
  std::vector<double> v(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) v[i * n + i] = 1;
  for (int it = 0; it < n * n * 16; ++it) {
    int p = 0, q = 1;
    double largest = 0;
    for (int r = 0; r < n; ++r)
      for (int c = r + 1; c < n; ++c) {
        const double m = std::fabs(a[r * n + c]);
        if (m > largest) { largest = m; p = r; q = c; }
      }
    const double ds = std::max({std::fabs(a[p * n + p]), std::fabs(a[q * n + q]), 1.0});
    if (largest <= 1e-12 * ds) break;
    const double app = a[p * n + p], aqq = a[q * n + q], apq = a[p * n + q];
    const double angle = 0.5 * std::atan2(2 * apq, aqq - app);
    const double c = std::cos(angle), s = std::sin(angle);
    for (int i = 0; i < n; ++i) {
      if (i == p || i == q) continue;
      const double aip = a[i * n + p], aiq = a[i * n + q];
      const double rp = c * aip - s * aiq, rq = s * aip + c * aiq;
      a[i * n + p] = rp; a[p * n + i] = rp;
      a[i * n + q] = rq; a[q * n + i] = rq;
    }
    a[p * n + p] = c * c * app - 2 * s * c * apq + s * s * aqq;
    a[q * n + q] = s * s * app + 2 * s * c * apq + c * c * aqq;
    a[p * n + q] = 0; a[q * n + p] = 0;
    for (int r = 0; r < n; ++r) {
      const double vip = v[r * n + p], viq = v[r * n + q];
      v[r * n + p] = c * vip - s * viq;
      v[r * n + q] = s * vip + c * viq;
    }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int l, int r) {
    const double dl = a[l * n + l], dr = a[r * n + r];
    if (dl != dr) return dl < dr;
    return l < r;
  });
  values.assign(n, 0);
  vectors.assign(static_cast<size_t>(n) * n, 0);
  for (int c = 0; c < n; ++c) {
    values[c] = a[order[c] * n + order[c]];
    for (int r = 0; r < n; ++r) vectors[r * n + c] = v[r * n + order[c]];
  }
}

// ---- local problem ----------------------------------------------------------

struct Problem {
  uint32_t Vp = 0, Tp = 0;
  std::vector<uint32_t> globalVertex, globalTet;
  std::vector<double> rest;            // 3 * Vp
  std::vector<double> mass;            // Vp (global lumped masses)
  std::vector<uint32_t> incident;      // Vp (global incident tet counts)
  std::vector<uint8_t> freeMask;       // Vp
  std::vector<uint32_t> tets;          // 4 * Tp local
  std::vector<double> vol, invRest;    // Tp, 9 * Tp
  std::vector<const Material*> mats;   // Tp
};

struct Context {
  const Problem* pb = nullptr;
  double h = 0;
  int n = 0;
  std::vector<int> dof;  // Vp -> first active dof or -1
  std::vector<double> H, L;
  // Per training pose: vertex frames (9 * Vp) and element gradients with the
  // distributed inertia folded in (12 * Tp).
  int poses = 0;
  std::vector<std::vector<double>> frames, elemGrad;
  bool amplitudeReduced = false;
  // Co-rotated linear training: low-frequency displacement poses (3 * Vp
  // each) and the rest stiffness of every tetrahedron (144 * Tp).
  bool linear = false;
  std::vector<std::vector<double>> linearPoses;
  std::vector<double> stiffness;
};

void deformationGradient(const Problem& pb, uint32_t t, const double* x, double* F) {
  const uint32_t* q = &pb.tets[4ull * t];
  const double* a = &x[3ull * q[0]];
  const double ds[9] = {x[3ull * q[1]] - a[0], x[3ull * q[2]] - a[0], x[3ull * q[3]] - a[0],
                        x[3ull * q[1] + 1] - a[1], x[3ull * q[2] + 1] - a[1], x[3ull * q[3] + 1] - a[1],
                        x[3ull * q[1] + 2] - a[2], x[3ull * q[2] + 2] - a[2], x[3ull * q[3] + 2] - a[2]};
  mul3(ds, &pb.invRest[9ull * t], F);
}

// Stable Neo-Hookean first Piola stress in the reference's CPU form
// (evaluateStableNeoHookeanDensity, src/simulation/cpu/stable-neo-hookean.ts:225-288).
void stablePiola(const Material& m, const double* F, double* P, double* J) {
  double lambda, mu;
  stableLame(m, &lambda, &mu);
  const double alpha = 1 + mu / lambda - mu / (4 * lambda);
  double I1 = 0;
  for (int i = 0; i < 9; ++i) I1 += F[i] * F[i];
  const double cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                         F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                         F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  const double d = det3(F);
  const double shear = mu * (1 - 1 / (I1 + 1));
  const double volume = lambda * (d - alpha);
  for (int i = 0; i < 9; ++i) P[i] = shear * F[i] + volume * cof[i];
  *J = d;
}

// assembleRestLinearSystem (src/simulation/cpu/fem.ts:238-335) on the problem.
bool buildSystem(Context& ctx) {
  const Problem& pb = *ctx.pb;
  ctx.dof.assign(pb.Vp, -1);
  int n = 0;
  for (uint32_t v = 0; v < pb.Vp; ++v)
    if (pb.freeMask[v]) { ctx.dof[v] = n; n += 3; }
  ctx.n = n;
  if (n == 0) return false;
  ctx.H.assign(static_cast<size_t>(n) * n, 0.0);
  double k[144];
  for (uint32_t t = 0; t < pb.Tp; ++t) {
    linearStiffness(&pb.invRest[9ull * t], pb.vol[t], *pb.mats[t], k);
    for (int lr = 0; lr < 4; ++lr) {
      const int rb = ctx.dof[pb.tets[4ull * t + lr]];
      if (rb < 0) continue;
      for (int lc = 0; lc < 4; ++lc) {
        const int cb = ctx.dof[pb.tets[4ull * t + lc]];
        if (cb < 0) continue;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            ctx.H[static_cast<size_t>(rb + i) * n + cb + j] += k[(lr * 3 + i) * 12 + lc * 3 + j];
      }
    }
  }
  const double invH2 = 1.0 / (ctx.h * ctx.h);
  for (uint32_t v = 0; v < pb.Vp; ++v) {
    const int b = ctx.dof[v];
    if (b < 0) continue;
    const double inertia = pb.mass[v] * invH2;
    if (!(inertia > 0) || !std::isfinite(inertia))
      throw std::runtime_error("Movable vertex has invalid lumped mass.");
    for (int c = 0; c < 3; ++c) ctx.H[static_cast<size_t>(b + c) * n + b + c] += inertia;
  }
  if (!choleskyFactor(ctx.H, n, ctx.L))
    throw std::runtime_error("Rest Hessian is not positive definite.");
  return true;
}

// buildLowFrequencyTrainingPoses (src/simulation/cpu/cubature.ts:224-297):
// block inverse iteration then Rayleigh-Ritz.  Returns full-length modes.
std::vector<std::vector<double>> lowFrequencyModes(const Context& ctx, int requested,
                                                   int iterations) {
  const int n = ctx.n;
  const int m = std::min(requested, n);
  std::vector<std::vector<double>> modes(m, std::vector<double>(n));
  for (int k = 0; k < m; ++k)
    for (int r = 0; r < n; ++r)
      modes[k][r] = std::sin((r + 1.0) * (k + 1.0) * 0.754877666) +
                    0.5 * std::cos((r + 1.0) * (k + 3.0) * 0.569840291);
  modes = orthonormalizeBlock(modes, n);
  for (int it = 0; it < iterations; ++it) {
    std::vector<std::vector<double>> next(m, std::vector<double>(n));
    for (int k = 0; k < m; ++k) solveCholesky(ctx.L, n, modes[k].data(), next[k].data());
    modes = orthonormalizeBlock(next, n);
  }
  std::vector<std::vector<double>> Hm(m, std::vector<double>(n, 0.0));
  for (int k = 0; k < m; ++k)
    for (int r = 0; r < n; ++r) Hm[k][r] = dotv(&ctx.H[static_cast<size_t>(r) * n], modes[k].data(), n);
  std::vector<double> proj(static_cast<size_t>(m) * m);
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < m; ++c) proj[r * m + c] = dotv(modes[r].data(), Hm[c].data(), n);
  std::vector<double> values, vecs;
  jacobiEigen(proj, m, values, vecs);
  const Problem& pb = *ctx.pb;
  std::vector<std::vector<double>> out;
  for (int k = 0; k < m; ++k) {
    std::vector<double> v(n, 0.0);
    for (int b = 0; b < m; ++b) {
      const double c = vecs[b * m + k];
      for (int r = 0; r < n; ++r) v[r] += modes[b][r] * c;
    }
    canonicalizeLargest(v);
    std::vector<double> full(3ull * pb.Vp, 0.0);
    for (uint32_t vert = 0; vert < pb.Vp; ++vert)
      if (ctx.dof[vert] >= 0)
        for (int c = 0; c < 3; ++c) full[3ull * vert + c] = v[ctx.dof[vert] + c];
    out.push_back(std::move(full));
  }
  return out;
}

// normalizeAndAppendMode (src/simulation/cpu/nonlinear-cubature.ts:308-333).
bool normalizeAndAppend(std::vector<std::vector<double>>& dst, std::vector<double> cand) {
  for (const auto& e : dst) {
    const double p = dotv(cand.data(), e.data(), cand.size());
    for (size_t i = 0; i < cand.size(); ++i) cand[i] -= p * e[i];
  }
  const double norm = std::sqrt(dotv(cand.data(), cand.data(), cand.size()));
  if (!(norm > 1e-10) || !std::isfinite(norm)) return false;
  for (double& x : cand) x /= norm;
  for (double x : cand) {
    if (std::fabs(x) <= 1e-12) continue;
    if (x < 0)
      for (double& y : cand) y = -y;
    break;
  }
  dst.push_back(std::move(cand));
  return true;
}

// buildFreeComponentRigidDisplacementModes (nonlinear-cubature.ts:335-416).
std::vector<std::vector<double>> rigidModes(const Problem& pb) {
  std::vector<uint32_t> parent(pb.Vp);
  std::iota(parent.begin(), parent.end(), 0u);
  auto find = [&](uint32_t v) {
    uint32_t r = v;
    while (parent[r] != r) r = parent[r];
    while (parent[v] != v) { const uint32_t nx = parent[v]; parent[v] = r; v = nx; }
    return r;
  };
  for (uint32_t t = 0; t < pb.Tp; ++t) {
    const uint32_t f = pb.tets[4ull * t];
    for (int l = 1; l < 4; ++l) {
      const uint32_t a = find(f), b = find(pb.tets[4ull * t + l]);
      if (a != b) parent[std::max(a, b)] = std::min(a, b);
    }
  }
  std::vector<std::vector<uint32_t>> comps;
  std::unordered_map<uint32_t, size_t> index;
  for (uint32_t v = 0; v < pb.Vp; ++v) {
    const uint32_t r = find(v);
    auto it = index.find(r);
    if (it == index.end()) { index[r] = comps.size(); comps.push_back({v}); }
    else comps[it->second].push_back(v);
  }
  std::vector<std::vector<double>> out;
  for (const auto& verts : comps) {
    bool anyFixed = false;
    for (uint32_t v : verts) anyFixed |= !pb.freeMask[v];
    if (anyFixed) continue;
    double total = 0, c[3] = {0, 0, 0};
    for (uint32_t v : verts) {
      total += pb.mass[v];
      for (int k = 0; k < 3; ++k) c[k] += pb.mass[v] * pb.rest[3ull * v + k];
    }
    for (double& x : c) x /= total;
    std::vector<std::vector<double>> cands(6, std::vector<double>(3ull * pb.Vp, 0.0));
    for (uint32_t v : verts) {
      const double x = pb.rest[3ull * v] - c[0], y = pb.rest[3ull * v + 1] - c[1],
                   z = pb.rest[3ull * v + 2] - c[2];
      for (int k = 0; k < 3; ++k) cands[k][3ull * v + k] = 1;
      cands[3][3ull * v] = 0; cands[3][3ull * v + 1] = -z; cands[3][3ull * v + 2] = y;
      cands[4][3ull * v] = z; cands[4][3ull * v + 1] = 0; cands[4][3ull * v + 2] = -x;
      cands[5][3ull * v] = -y; cands[5][3ull * v + 1] = x; cands[5][3ull * v + 2] = 0;
    }
    for (auto& cd : cands) normalizeAndAppend(out, cd);
  }
  return out;
}

double sceneScale(const Problem& pb) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (uint32_t v = 0; v < pb.Vp; ++v)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pb.rest[3ull * v + k]);
      hi[k] = std::max(hi[k], pb.rest[3ull * v + k]);
    }
  return std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                   (hi[2] - lo[2]) * (hi[2] - lo[2]));
}

// displacementDirectionMeasure (nonlinear-cubature.ts:140-178).
double directionMeasure(const Problem& pb, const std::vector<double>& d, double scale) {
  double maxGrad = 0, maxDisp = 0;
  for (uint32_t t = 0; t < pb.Tp; ++t) {
    double G[9];
    deformationGradient(pb, t, d.data(), G);
    double s = 0;
    for (double x : G) s += x * x;
    maxGrad = std::max(maxGrad, std::sqrt(s));
  }
  for (uint32_t v = 0; v < pb.Vp; ++v)
    maxDisp = std::max(maxDisp, std::sqrt(d[3ull * v] * d[3ull * v] + d[3ull * v + 1] * d[3ull * v + 1] +
                                          d[3ull * v + 2] * d[3ull * v + 2]));
  return std::max(maxGrad, maxDisp / scale);
}

// Build the training corpus (buildNonlinearCubaturePoseCorpus, training split,
// nonlinear-cubature.ts:452-552) and cache frames and element gradients.
void buildCorpus(Context& ctx, const jgs2_precompute_options& opt) {
  const Problem& pb = *ctx.pb;
  const double scale = sceneScale(pb);
  if (!(scale > 0)) throw std::runtime_error("Nonlinear Cubature scene scale must be positive.");
  const auto rigid = rigidModes(pb);
  const int requested = static_cast<int>(opt.mode_count + kValidationOnlyModes);
  auto raw = lowFrequencyModes(ctx, requested + static_cast<int>(rigid.size()),
                               static_cast<int>(opt.inverse_iterations));
  std::vector<std::vector<double>> modes;
  if (rigid.empty()) {
    modes = raw;
  } else {
    // removeRigidDisplacementModes (nonlinear-cubature.ts:418-441).
    for (auto src : raw) {
      for (const auto& r : rigid) {
        const double p = dotv(src.data(), r.data(), src.size());
        for (size_t i = 0; i < src.size(); ++i) src[i] -= p * r[i];
      }
      normalizeAndAppend(modes, src);
      if (static_cast<int>(modes.size()) >= requested) break;
    }
    if (modes.empty()) throw std::runtime_error("Nonlinear Cubature free components have no deformational modes.");
  }
  const size_t trainModes = std::min<size_t>(opt.mode_count, modes.size());
  std::vector<std::vector<double>> posePositions;
  double amplitude = opt.training_amplitude;
  for (int attempt = 0; attempt < 6; ++attempt) {
    posePositions.clear();
    bool ok = true;
    for (size_t k = 0; k < trainModes && ok; ++k)
      for (int sign : {1, -1}) {
        std::vector<double> dir(modes[k].size());
        for (size_t i = 0; i < dir.size(); ++i) dir[i] = sign * modes[k][i];
        const double measure = directionMeasure(pb, dir, scale);
        if (!(measure > 1e-14) || !std::isfinite(measure))
          throw std::runtime_error("Nonlinear Cubature training mode has zero direction.");
        const double s = amplitude / measure;
        std::vector<double> x(pb.rest);
        for (size_t i = 0; i < x.size(); ++i) x[i] += dir[i] * s;
        double minJ = 1e300;
        for (uint32_t t = 0; t < pb.Tp; ++t) {
          double F[9];
          deformationGradient(pb, t, x.data(), F);
          minJ = std::min(minJ, det3(F));
        }
        if (!(minJ >= kMinimumPoseDeterminant)) { ok = false; break; }
        posePositions.push_back(std::move(x));
      }
    if (ok) break;
    // The reference throws here; a halved amplitude keeps the training pose
    // admissible and is counted in the statistics.
    amplitude *= 0.5;
    ctx.amplitudeReduced = true;
  }
  ctx.poses = static_cast<int>(posePositions.size());
  ctx.frames.assign(ctx.poses, std::vector<double>(9ull * pb.Vp, 0.0));
  ctx.elemGrad.assign(ctx.poses, std::vector<double>(12ull * pb.Tp, 0.0));
  const double invH2 = 1.0 / (ctx.h * ctx.h);
  for (int p = 0; p < ctx.poses; ++p) {
    const double* x = posePositions[p].data();
    // Vertex frames: polar of the rest-volume-weighted average F over the
    // vertex's incident tetrahedra in the problem (computeVertexPolarFrames,
    // src/simulation/cpu/deformation-gradient.ts:22-172).
    std::vector<double> avg(9ull * pb.Vp, 0.0), wsum(pb.Vp, 0.0);
    for (uint32_t t = 0; t < pb.Tp; ++t) {
      double F[9], P[9], J;
      deformationGradient(pb, t, x, F);
      for (int l = 0; l < 4; ++l) {
        const uint32_t v = pb.tets[4ull * t + l];
        for (int i = 0; i < 9; ++i) avg[9ull * v + i] += pb.vol[t] * F[i];
        wsum[v] += pb.vol[t];
      }
      stablePiola(*pb.mats[t], F, P, &J);
      double g[12];
      shapeGradients(&pb.invRest[9ull * t], g);
      double* eg = &ctx.elemGrad[p][12ull * t];
      for (int l = 0; l < 4; ++l) {
        const uint32_t v = pb.tets[4ull * t + l];
        const double dist = pb.mass[v] * invH2 / pb.incident[v];
        for (int r = 0; r < 3; ++r) {
          double s = 0;
          for (int c = 0; c < 3; ++c) s += P[r * 3 + c] * g[l * 3 + c];
          eg[l * 3 + r] = pb.vol[t] * s + dist * (x[3ull * v + r] - pb.rest[3ull * v + r]);
        }
      }
    }
    for (uint32_t v = 0; v < pb.Vp; ++v) {
      if (wsum[v] > 0)
        for (int i = 0; i < 9; ++i) avg[9ull * v + i] /= wsum[v];
      polarRotation3(&avg[9ull * v], &ctx.frames[p][9ull * v]);
    }
  }
}

// Training data of the co-rotated linear path (precompute.ts:261-268): the
// low-frequency modes of the rest system as displacement poses, and each
// tetrahedron's rest stiffness.
void buildLinearPoses(Context& ctx, const jgs2_precompute_options& opt) {
  const Problem& pb = *ctx.pb;
  ctx.linear = true;
  ctx.linearPoses = lowFrequencyModes(ctx, static_cast<int>(opt.mode_count),
                                      static_cast<int>(opt.inverse_iterations));
  ctx.stiffness.assign(144ull * pb.Tp, 0.0);
  for (uint32_t t = 0; t < pb.Tp; ++t)
    linearStiffness(&pb.invRest[9ull * t], pb.vol[t], *pb.mats[t], &ctx.stiffness[144ull * t]);
}

void prepareTraining(Context& ctx, const jgs2_precompute_options& opt, bool linear) {
  if (opt.exact_complement) return;
  if (linear) buildLinearPoses(ctx, opt);
  else buildCorpus(ctx, opt);
}

// ---- greedy nonnegative selection ------------------------------------------

using jgs2select::Gram;
using jgs2select::kMaxColumns;
using jgs2select::kResidualTolerance;
using jgs2select::maxd;

struct Selection {
  std::vector<int> tets;  // local tet ids in selection order
  std::vector<double> weights;
  double residual = 0;    // normalized
};

// A training system ready for selection: one column per local tetrahedron
// (its reduced gradients stacked over the training poses) and the summed
// target, with the selection's column limit and refinement passes.
struct Training {
  std::vector<std::vector<double>> cols;
  std::vector<double> target;
  int maxColumns = 0;
  int passes = 0;
  bool audit = false;  // small-mesh subset audit after the selection
};

// The candidate filter of selectGreedyNonnegativeColumns (cubature.ts:
// 508-560): columns with |c|² > 1e-18 in index order, their squared norms and
// target dot products.
struct Candidates {
  enum Status { kReady, kFlatTarget, kEmpty } status = kReady;
  double tt = 0, tn = 0;
  int limit = 0;
  std::vector<int> ids;
  std::vector<double> cc, ct;
};

Candidates candidates(const Training& tr) {
  Candidates c;
  const size_t rows = tr.target.size();
  c.tt = dotv(tr.target.data(), tr.target.data(), rows);
  c.tn = std::sqrt(c.tt);
  if (c.tn <= 1e-12) {
    c.status = Candidates::kFlatTarget;
    return c;
  }
  for (size_t i = 0; i < tr.cols.size(); ++i) {
    const double n2 = dotv(tr.cols[i].data(), tr.cols[i].data(), rows);
    if (n2 > 1e-18) {
      c.ids.push_back(static_cast<int>(i));
      c.cc.push_back(n2);
    }
  }
  c.limit = std::min<int>(tr.maxColumns, static_cast<int>(c.ids.size()));
  if (c.limit > kMaxColumns) throw std::runtime_error("Exhaustive NNLS supports at most 12 selected columns.");
  if (c.ids.empty() || c.limit == 0) {
    c.status = Candidates::kEmpty;
    return c;
  }
  c.ct.resize(c.ids.size());
  for (size_t i = 0; i < c.ids.size(); ++i) c.ct[i] = dotv(tr.cols[c.ids[i]].data(), tr.target.data(), rows);
  return c;
}

// Greedy growth (each step appends the candidate whose exhaustive NNLS fit
// leaves the smallest residual) until the limit or a residual below 1%, then
// refinement passes that swap one chosen slot for an unchosen candidate while
// that helps (selectGreedyNonnegativeColumns, cubature.ts:508-690).  The
// trial systems, the NNLS and the scan rule are cubature_select.hpp's, shared
// with the GPU selection.
SelectOutput selectOnCpu(const Training& tr, const Candidates& cs, double tolerance = kResidualTolerance) {
  using namespace jgs2select;
  SelectOutput ch;
  if (cs.status != Candidates::kReady) return ch;
  const size_t rows = tr.target.size(), C = cs.ids.size();
  const int n = static_cast<int>(C);
  std::vector<double> dsel(kMaxColumns * C);
  auto setRow = [&](int slot) {
    const double* a = tr.cols[cs.ids[ch.sel[slot]]].data();
    for (size_t i = 0; i < C; ++i) dsel[slot * C + i] = dotv(a, tr.cols[cs.ids[i]].data(), rows);
  };
  auto chosen = [&](int ci) {
    for (int s = 0; s < ch.count; ++s)
      if (ch.sel[s] == ci) return true;
    return false;
  };
  Gram<kMaxColumns> g;
  double w[kMaxColumns];
  double err = cs.tt;
  for (int step = 0; step < cs.limit; ++step) {
    const int k = ch.count;
    int best = -1;
    double bestErr = err;
    for (int ci = 0; ci < n; ++ci) {
      if (chosen(ci)) continue;
      swapGram(g, ch.sel, k + 1, k, ci, dsel.data(), C, cs.cc.data(), cs.ct.data(), cs.tt);
      const double e = smallNnls(g, w);
      if (improves(e, bestErr, best >= 0, ci, best)) {
        best = ci;
        bestErr = e;
      }
    }
    if (best < 0) break;
    swapGram(g, ch.sel, k + 1, k, best, dsel.data(), C, cs.cc.data(), cs.ct.data(), cs.tt);
    smallNnls(g, ch.weights);
    ch.sel[k] = best;
    ch.count = k + 1;
    setRow(k);
    err = bestErr;
    if (std::sqrt(maxd(err, 0.0)) / cs.tn < tolerance) break;
  }
  for (int pass = 0; pass < tr.passes && ch.count > 0; ++pass) {
    const int k = ch.count;
    int rslot = -1, rcand = -1;
    double rerr = err;
    for (int slot = 0; slot < k; ++slot) {
      for (int ci = 0; ci < n; ++ci) {
        if (chosen(ci)) continue;
        swapGram(g, ch.sel, k, slot, ci, dsel.data(), C, cs.cc.data(), cs.ct.data(), cs.tt);
        const double e = smallNnls(g, w);
        if (improves(e, rerr, rcand >= 0, ci, rcand)) {
          rslot = slot;
          rcand = ci;
          rerr = e;
        }
      }
    }
    if (rslot < 0) break;
    swapGram(g, ch.sel, k, rslot, rcand, dsel.data(), C, cs.cc.data(), cs.ct.data(), cs.tt);
    smallNnls(g, ch.weights);
    ch.sel[rslot] = rcand;
    setRow(rslot);
    err = rerr;
  }
  return ch;
}

// Exhaustive subset audit for meshes of at most 12 tetrahedra
// (nonlinear-cubature-training.ts:738-771).
void subsetAudit(const std::vector<std::vector<double>>& cols, const std::vector<double>& t,
                 int maxSamples, Selection& sel) {
  const int T = static_cast<int>(cols.size());
  if (!(T <= 12 && maxSamples < T)) return;
  const size_t rows = t.size();
  const double tt = dotv(t.data(), t.data(), rows), tn = std::sqrt(tt);
  if (tn <= 1e-12) return;
  const int size = std::min(maxSamples, T);
  std::vector<int> subset;
  std::function<void(int)> visit = [&](int next) {
    if (static_cast<int>(subset.size()) == size) {
      Gram<kMaxColumns> g;
      g.k = size;
      g.tt = tt;
      for (int r = 0; r < size; ++r) {
        g.b[r] = dotv(cols[subset[r]].data(), t.data(), rows);
        for (int c = 0; c < size; ++c) g.G[r][c] = dotv(cols[subset[r]].data(), cols[subset[c]].data(), rows);
      }
      double w[kMaxColumns];
      jgs2select::smallNnls(g, w);
      std::vector<double> res(t);
      for (int i = 0; i < size; ++i)
        for (size_t r = 0; r < rows; ++r) res[r] -= cols[subset[i]][r] * w[i];
      const double nr = std::sqrt(dotv(res.data(), res.data(), rows)) / tn;
      if (nr < sel.residual - 1e-14) {
        sel.residual = nr;
        sel.tets = subset;
        sel.weights.assign(w, w + size);
      }
      return;
    }
    const int remaining = size - static_cast<int>(subset.size());
    for (int tt2 = next; tt2 <= T - remaining; ++tt2) {
      subset.push_back(tt2);
      visit(tt2 + 1);
      subset.pop_back();
    }
  };
  visit(0);
}

// The chosen tetrahedra and weights with the fit's direct residual, then the
// subset audit where it applies.
Selection finishSelection(const Training& tr, const Candidates& cs, const SelectOutput& ch) {
  Selection out;
  if (cs.status == Candidates::kEmpty) out.residual = 1;
  if (cs.status == Candidates::kReady) {
    for (int i = 0; i < ch.count; ++i) {
      out.tets.push_back(cs.ids[ch.sel[i]]);
      out.weights.push_back(ch.weights[i]);
    }
    const size_t rows = tr.target.size();
    std::vector<double> res(tr.target);
    for (size_t i = 0; i < out.tets.size(); ++i)
      for (size_t r = 0; r < rows; ++r) res[r] -= tr.cols[out.tets[i]][r] * out.weights[i];
    out.residual = std::sqrt(dotv(res.data(), res.data(), rows)) / cs.tn;
  }
  if (tr.audit) subsetAudit(tr.cols, tr.target, tr.maxColumns, out);
  return out;
}

// The selection's input on the GPU: the candidate columns row-major.
std::vector<double> candidateRows(const Training& tr, const Candidates& cs) {
  const size_t rows = tr.target.size(), C = cs.ids.size();
  std::vector<double> out(rows * C);
  for (size_t i = 0; i < C; ++i) {
    const double* col = tr.cols[cs.ids[i]].data();
    for (size_t r = 0; r < rows; ++r) out[r * C + i] = col[r];
  }
  return out;
}

struct LocalRecord {
  int tet;  // local tet id
  double weight;
  std::array<double, 36> basis;
};

// Records of the positive weights (nonlinear-cubature-training.ts:785-792),
// each with the four vertices' basis blocks.
void keepPositive(const Problem& pb, const std::vector<double>& ubar, const Selection& sel,
                  std::vector<LocalRecord>& records) {
  for (size_t i = 0; i < sel.tets.size(); ++i) {
    if (!(sel.weights[i] > 1e-10)) continue;
    LocalRecord rec;
    rec.tet = sel.tets[i];
    rec.weight = sel.weights[i];
    for (int l = 0; l < 4; ++l) {
      const uint32_t v = pb.tets[4ull * rec.tet + l];
      for (int e = 0; e < 9; ++e) rec.basis[l * 9 + e] = ubar[9ull * v + e];
    }
    records.push_back(rec);
  }
}

// selectCubatureSamples (src/simulation/cpu/cubature.ts:714-820): one column
// per tetrahedron holding, at every training pose, its reduced gradient
// (evaluateReducedTetGradient, cubature.ts:312-369: rest stiffness times the
// pose plus the tetrahedron's share of the inertia, projected by the exact
// basis, less the source slot's own row); per-pose normalisation by the norm
// of the summed target.  False when there is nothing to fit.
bool linearTraining(const Context& ctx, uint32_t s, const std::vector<double>& ubar,
                    const jgs2_precompute_options& opt, Training& tr);

// computeExactVertexBasis (precompute.ts:141-206) and the training system of
// one source vertex (selectStableNeoHookeanCubatureSamples,
// nonlinear-cubature-training.ts:689-843, or the co-rotated linear
// training).  Returns false when the source is finished without a selection
// (the exact complement's records, or nothing to fit).
bool buildTraining(const Context& ctx, uint32_t s, const jgs2_precompute_options& opt, std::vector<double>& ubar,
                   Training& tr, std::vector<LocalRecord>& records) {
  const Problem& pb = *ctx.pb;
  const int n = ctx.n;
  const int sb = ctx.dof[s];
  records.clear();
  if (sb < 0) return false;
  // Exact basis Ubar = H^-1 S^T (S H^-1 S^T)^-1, one 3x3 block per vertex.
  std::vector<double> X(static_cast<size_t>(n) * 3, 0.0), rhs(n), sol(n);
  for (int c = 0; c < 3; ++c) {
    std::fill(rhs.begin(), rhs.end(), 0.0);
    rhs[sb + c] = 1;
    solveCholesky(ctx.L, n, rhs.data(), sol.data());
    for (int r = 0; r < n; ++r) X[static_cast<size_t>(r) * 3 + c] = sol[r];
  }
  double comp[9], schur[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      comp[r * 3 + c] = 0.5 * (X[static_cast<size_t>(sb + r) * 3 + c] + X[static_cast<size_t>(sb + c) * 3 + r]);
  if (!inv3(comp, schur)) throw std::runtime_error("Cannot invert a singular 3 by 3 matrix.");
  ubar.assign(9ull * pb.Vp, 0.0);
  for (uint32_t v = 0; v < pb.Vp; ++v) {
    const int b = ctx.dof[v];
    if (b < 0) continue;
    for (int coord = 0; coord < 3; ++coord)
      for (int col = 0; col < 3; ++col) {
        double val = 0;
        for (int in = 0; in < 3; ++in) val += X[static_cast<size_t>(b + coord) * 3 + in] * schur[in * 3 + col];
        ubar[9ull * v + coord * 3 + col] = val;
      }
  }
  if (opt.exact_complement) {
    // Exact remainder: every candidate tetrahedron with weight one.
    for (uint32_t t = 0; t < pb.Tp; ++t) {
      LocalRecord rec;
      rec.tet = static_cast<int>(t);
      rec.weight = 1.0;
      for (int l = 0; l < 4; ++l) {
        const uint32_t v = pb.tets[4ull * t + l];
        for (int e = 0; e < 9; ++e) rec.basis[l * 9 + e] = ubar[9ull * v + e];
      }
      records.push_back(rec);
    }
    return false;
  }
  if (ctx.linear) return linearTraining(ctx, s, ubar, opt, tr);
  // Stacked training system (buildStackedTrainingSystem,
  // nonlinear-cubature-training.ts:473-552) with per-pose normalisation.
  const int P = ctx.poses;
  std::vector<std::vector<double>>& cols = tr.cols;
  std::vector<double>& target = tr.target;
  cols.assign(pb.Tp, std::vector<double>(3ull * P, 0.0));
  target.assign(3ull * P, 0.0);
  std::vector<double> B(9ull * pb.Vp);
  std::vector<double> rem(3ull * pb.Tp);
  for (int p = 0; p < P; ++p) {
    const double* Rs = &ctx.frames[p][9ull * s];
    double RsT[9];
    transpose3(Rs, RsT);
    for (uint32_t v = 0; v < pb.Vp; ++v) {
      if (ctx.dof[v] < 0) { std::fill(&B[9ull * v], &B[9ull * v] + 9, 0.0); continue; }
      double left[9];
      mul3(&ctx.frames[p][9ull * v], &ubar[9ull * v], left);
      mul3(left, RsT, &B[9ull * v]);
    }
    double poseTarget[3] = {0, 0, 0}, scaleSq = 0;
    for (uint32_t t = 0; t < pb.Tp; ++t) {
      const double* eg = &ctx.elemGrad[p][12ull * t];
      double pr[3] = {0, 0, 0};
      int slot = -1;
      for (int l = 0; l < 4; ++l) {
        const uint32_t v = pb.tets[4ull * t + l];
        if (v == s) slot = l;
        const double* Bl = &B[9ull * v];
        for (int r = 0; r < 3; ++r)
          for (int row = 0; row < 3; ++row) pr[r] += Bl[row * 3 + r] * eg[l * 3 + row];
      }
      if (slot >= 0)
        for (int r = 0; r < 3; ++r) pr[r] -= eg[slot * 3 + r];
      for (int r = 0; r < 3; ++r) {
        rem[3ull * t + r] = pr[r];
        poseTarget[r] += pr[r];
        scaleSq += pr[r] * pr[r];
      }
    }
    const double poseNorm = std::sqrt(poseTarget[0] * poseTarget[0] + poseTarget[1] * poseTarget[1] +
                                      poseTarget[2] * poseTarget[2]);
    if (scaleSq == 0) continue;  // trivial pose
    // Cancellation-dominated target.  The reference throws below 1e-12
    // relative; between 1e-12 and 1e-6 the per-pose normalisation scales the
    // columns by up to 1e12 and the least-squares fit loses every digit, so
    // such poses are skipped like trivial ones.
    if (poseNorm <= 1e-6 * std::sqrt(scaleSq)) continue;
    for (int r = 0; r < 3; ++r) {
      target[3ull * p + r] = poseTarget[r] / poseNorm;
      for (uint32_t t = 0; t < pb.Tp; ++t) cols[t][3ull * p + r] = rem[3ull * t + r] / poseNorm;
    }
  }
  tr.maxColumns = static_cast<int>(opt.cubature_k);
  tr.passes = static_cast<int>(opt.refinement_passes);
  tr.audit = true;
  return true;
}

bool linearTraining(const Context& ctx, uint32_t s, const std::vector<double>& ubar,
                    const jgs2_precompute_options& opt, Training& tr) {
  const Problem& pb = *ctx.pb;
  const int P = static_cast<int>(ctx.linearPoses.size());
  const double invH2 = 1.0 / (ctx.h * ctx.h);
  std::vector<std::vector<double>>& cols = tr.cols;
  std::vector<double>& target = tr.target;
  cols.assign(pb.Tp, std::vector<double>(3ull * P, 0.0));
  target.assign(3ull * P, 0.0);
  for (int p = 0; p < P; ++p) {
    const double* pose = ctx.linearPoses[p].data();
    double poseTarget[3] = {0, 0, 0}, scaleSq = 0;
    for (uint32_t t = 0; t < pb.Tp; ++t) {
      const uint32_t* q = &pb.tets[4ull * t];
      const double* k = &ctx.stiffness[144ull * t];
      double u[12], g[12];
      for (int c = 0; c < 12; ++c) u[c] = pose[3ull * q[c / 3] + c % 3];
      for (int r = 0; r < 12; ++r) {
        double val = 0;
        for (int c = 0; c < 12; ++c) val += k[r * 12 + c] * u[c];
        const uint32_t v = q[r / 3];
        g[r] = val + pb.mass[v] * invH2 * u[r] / pb.incident[v];
      }
      double red[3] = {0, 0, 0};
      for (int l = 0; l < 4; ++l) {
        const double* U = &ubar[9ull * q[l]];
        for (int rc = 0; rc < 3; ++rc)
          for (int c = 0; c < 3; ++c) red[c] += U[rc * 3 + c] * g[l * 3 + rc];
      }
      for (int l = 0; l < 4; ++l)
        if (q[l] == s) {
          for (int c = 0; c < 3; ++c) red[c] -= g[l * 3 + c];
          break;
        }
      for (int c = 0; c < 3; ++c) {
        cols[t][3ull * p + c] = red[c];
        poseTarget[c] += red[c];
        scaleSq += red[c] * red[c];
      }
    }
    const double poseNorm = std::sqrt(poseTarget[0] * poseTarget[0] + poseTarget[1] * poseTarget[1] +
                                      poseTarget[2] * poseTarget[2]);
    // A target that cancels to below 1e-6 of its terms (seen on local
    // patches) would scale its rows by up to 1e12 and swamp the fit, so such
    // a pose is dropped; the reference normalises every pose above 1e-12.
    if (poseNorm <= 1e-6 * std::sqrt(scaleSq)) {
      for (uint32_t t = 0; t < pb.Tp; ++t)
        for (int c = 0; c < 3; ++c) cols[t][3ull * p + c] = 0.0;
      continue;
    }
    if (poseNorm > 1e-12)
      for (int c = 0; c < 3; ++c) {
        target[3ull * p + c] = poseTarget[c] / poseNorm;
        for (uint32_t t = 0; t < pb.Tp; ++t) cols[t][3ull * p + c] /= poseNorm;
      }
  }
  bool anyColumn = false;
  for (const auto& col : cols) anyColumn |= dotv(col.data(), col.data(), col.size()) > 1e-18;
  if (!(std::sqrt(dotv(target.data(), target.data(), target.size())) > 1e-12) || !anyColumn) return false;
  tr.maxColumns = static_cast<int>(opt.cubature_k);
  tr.passes = kLinearRefinementPasses;
  tr.audit = false;
  return true;
}

// One source vertex trained start to finish on this CPU thread; returns the
// normalized residual.
double trainSource(const Context& ctx, uint32_t s, const jgs2_precompute_options& opt,
                   std::vector<LocalRecord>& records) {
  std::vector<double> ubar;
  Training tr;
  if (!buildTraining(ctx, s, opt, ubar, tr, records)) return 0.0;
  const Candidates cs = candidates(tr);
  const Selection sel = finishSelection(tr, cs, selectOnCpu(tr, cs));
  keepPositive(*ctx.pb, ubar, sel, records);
  return sel.residual;
}

// A source vertex whose selection runs in a GPU batch: its training system is
// built on a CPU thread, selected with the other jobs of its batch, then
// finished on a CPU thread.
struct TrainingJob {
  Problem pb;                 // the patch (patch method); unused with a shared context
  uint32_t source = 0;        // source vertex, local to the problem
  bool trained = false;       // the problem had a system to train
  bool reduced = false;       // the corpus amplitude was halved
  bool select = false;        // a selection is pending
  std::vector<double> ubar;
  Training tr;
  Candidates cs;
  std::vector<double> rows;   // candidate columns, row-major
  std::vector<LocalRecord> records;
  double residual = 0;
  size_t bytes() const {
    size_t b = rows.size() * sizeof(double);
    for (const auto& c : tr.cols) b += c.size() * sizeof(double);
    return b;
  }
};

// Builds job j's training system (on the given context) and its candidate
// filter; a job that needs no selection is finished here.
void buildJob(const Context& ctx, const jgs2_precompute_options& opt, TrainingJob& job) {
  job.trained = true;
  job.select = buildTraining(ctx, job.source, opt, job.ubar, job.tr, job.records);
  if (!job.select) return;
  job.cs = candidates(job.tr);
  if (job.cs.status != Candidates::kReady) {
    job.select = false;
    const Selection sel = finishSelection(job.tr, job.cs, SelectOutput{});
    keepPositive(*ctx.pb, job.ubar, sel, job.records);
    job.residual = sel.residual;
    return;
  }
  job.rows = candidateRows(job.tr, job.cs);
}

// Selects every pending job of the batch in one GPU launch, then finishes
// them (direct residuals, audits, records) on the CPU threads; the jobs'
// training data is released.
std::string selectBatchOnGpu(std::vector<TrainingJob*>& batch, const Problem* shared) {
  std::vector<SelectInput> in;
  std::vector<TrainingJob*> pending;
  for (TrainingJob* j : batch) {
    if (!j->select) continue;
    SelectInput p;
    p.cols = j->rows.data();
    p.cc = j->cs.cc.data();
    p.ct = j->cs.ct.data();
    p.rows = static_cast<uint32_t>(j->tr.target.size());
    p.cand = static_cast<uint32_t>(j->cs.ids.size());
    p.limit = static_cast<uint32_t>(j->cs.limit);
    p.passes = static_cast<uint32_t>(j->tr.passes);
    p.tt = j->cs.tt;
    p.tn = j->cs.tn;
    in.push_back(p);
    pending.push_back(j);
  }
  std::vector<SelectOutput> out;
  const std::string err = selectOnGpu(in, out);
  if (!err.empty()) return err;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < static_cast<int64_t>(pending.size()); ++i) {
    TrainingJob& j = *pending[i];
    const Selection sel = finishSelection(j.tr, j.cs, out[i]);
    keepPositive(shared ? *shared : j.pb, j.ubar, sel, j.records);
    j.residual = sel.residual;
    j.select = false;
  }
  for (TrainingJob* j : batch) {
    j->tr = Training{};
    j->rows = {};
    j->cs = Candidates{};
    j->ubar = {};
  }
  return {};
}

double secondsSince(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Bytes of training data gathered before a GPU selection batch runs.
constexpr size_t kSelectionBatchBytes = size_t(1) << 30;

// The batch budget: kSelectionBatchBytes, or JGS2_SELECTION_BATCH_BYTES when
// set (smaller budgets split a precompute into more GPU launches).
size_t selectionBatchBytes() {
  const char* e = std::getenv("JGS2_SELECTION_BATCH_BYTES");
  if (!e || !*e) return kSelectionBatchBytes;
  const unsigned long long v = std::strtoull(e, nullptr, 10);
  return v > 0 ? static_cast<size_t>(v) : kSelectionBatchBytes;
}

// ---- patch extraction and signatures ----------------------------------------

struct MeshGraph {
  std::vector<uint64_t> adjStart;    // incident tets CSR
  std::vector<uint32_t> adjTets;
  std::vector<uint64_t> nbrStart;    // vertex neighbours CSR
  std::vector<uint32_t> nbrs;
};

MeshGraph buildGraph(const Mesh& m) {
  MeshGraph g;
  const uint32_t V = m.vertexCount(), T = m.tetCount();
  g.adjStart.assign(V + 1ull, 0);
  for (uint32_t v : m.tets) g.adjStart[v + 1]++;
  for (uint32_t v = 0; v < V; ++v) g.adjStart[v + 1] += g.adjStart[v];
  g.adjTets.assign(g.adjStart[V], 0);
  std::vector<uint64_t> cur(g.adjStart.begin(), g.adjStart.end() - 1);
  for (uint32_t t = 0; t < T; ++t)
    for (int l = 0; l < 4; ++l) g.adjTets[cur[m.tets[4ull * t + l]]++] = t;
  g.nbrStart.assign(V + 1ull, 0);
  std::vector<std::vector<uint32_t>> tmp(omp_get_max_threads());
  std::vector<std::vector<uint32_t>> per(V);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < static_cast<int64_t>(V); ++v) {
    std::vector<uint32_t>& list = per[v];
    for (uint64_t i = g.adjStart[v]; i < g.adjStart[v + 1]; ++i) {
      const uint32_t t = g.adjTets[i];
      for (int l = 0; l < 4; ++l) {
        const uint32_t u = m.tets[4ull * t + l];
        if (u != static_cast<uint32_t>(v)) list.push_back(u);
      }
    }
    std::sort(list.begin(), list.end());
    list.erase(std::unique(list.begin(), list.end()), list.end());
  }
  for (uint32_t v = 0; v < V; ++v) g.nbrStart[v + 1] = g.nbrStart[v] + per[v].size();
  g.nbrs.resize(g.nbrStart[V]);
  for (uint32_t v = 0; v < V; ++v) {
    std::copy(per[v].begin(), per[v].end(), g.nbrs.begin() + g.nbrStart[v]);
    std::vector<uint32_t>().swap(per[v]);
  }
  return g;
}

// Patch around s: free vertices within `radius` rings (not globally fixed),
// tetrahedra incident to them, and every vertex those tetrahedra touch.
// Per-thread scratch of the patch extraction: epoch marks over the mesh's
// vertices and tetrahedra (a vertex or tetrahedron is in the current set when
// its mark equals the current epoch), a global-to-local vertex map and
// reusable lists.  Replaces per-patch searches and sorts of duplicates.
struct PatchScratch {
  std::vector<uint32_t> vertexMark, tetMark, local;
  uint32_t epoch = 0;
  std::vector<uint32_t> frontier, next, visited, freeVerts, tets, verts;
  std::vector<int64_t> signature;
  Problem pb;  // the patch of the classification passes

  uint32_t nextEpoch(uint32_t V, uint32_t T) {
    if (vertexMark.size() != V || tetMark.size() != T) {
      vertexMark.assign(V, 0);
      tetMark.assign(T, 0);
      local.assign(V, 0);
      epoch = 0;
    }
    if (++epoch == 0) {
      std::fill(vertexMark.begin(), vertexMark.end(), 0u);
      std::fill(tetMark.begin(), tetMark.end(), 0u);
      epoch = 1;
    }
    return epoch;
  }
};

// The patch of source vertex s: the vertices within `radius` rings (breadth
// first over the vertex graph), the tetrahedra incident to its free vertices,
// and every vertex of those tetrahedra, each list in ascending global order
// (local ids follow it).  Rest volumes and inverse rest matrices are copied
// only when the patch is trained.
void extractPatch(const Scene& sc, const MeshGraph& g, uint32_t s, uint32_t radius, Problem& pb,
                  uint32_t* sLocal, PatchScratch& ps, bool forTraining) {
  const Mesh& m = sc.mesh;
  const uint32_t V = m.vertexCount(), T = m.tetCount();
  uint32_t e = ps.nextEpoch(V, T);
  ps.frontier.assign(1, s);
  ps.visited.assign(1, s);
  ps.vertexMark[s] = e;
  for (uint32_t r = 0; r < radius; ++r) {
    ps.next.clear();
    for (uint32_t v : ps.frontier)
      for (uint64_t i = g.nbrStart[v]; i < g.nbrStart[v + 1]; ++i) {
        const uint32_t u = g.nbrs[i];
        if (ps.vertexMark[u] != e) {
          ps.vertexMark[u] = e;
          ps.visited.push_back(u);
          ps.next.push_back(u);
        }
      }
    ps.frontier.swap(ps.next);
  }
  ps.freeVerts.clear();
  for (uint32_t v : ps.visited)
    if (!m.fixed[v]) ps.freeVerts.push_back(v);
  e = ps.nextEpoch(V, T);
  ps.tets.clear();
  for (uint32_t v : ps.freeVerts)
    for (uint64_t i = g.adjStart[v]; i < g.adjStart[v + 1]; ++i) {
      const uint32_t t = g.adjTets[i];
      if (ps.tetMark[t] != e) {
        ps.tetMark[t] = e;
        ps.tets.push_back(t);
      }
    }
  std::sort(ps.tets.begin(), ps.tets.end());
  ps.verts.clear();
  for (uint32_t t : ps.tets)
    for (int l = 0; l < 4; ++l) {
      const uint32_t u = m.tets[4ull * t + l];
      if (ps.vertexMark[u] != e) {
        ps.vertexMark[u] = e;
        ps.verts.push_back(u);
      }
    }
  std::sort(ps.verts.begin(), ps.verts.end());
  e = ps.nextEpoch(V, T);
  for (uint32_t v : ps.freeVerts) ps.vertexMark[v] = e;
  const std::vector<uint32_t>& verts = ps.verts;
  const std::vector<uint32_t>& tets = ps.tets;
  pb.Vp = static_cast<uint32_t>(verts.size());
  pb.Tp = static_cast<uint32_t>(tets.size());
  pb.globalVertex = verts;
  pb.globalTet = tets;
  pb.rest.resize(3ull * pb.Vp);
  pb.mass.resize(pb.Vp);
  pb.incident.resize(pb.Vp);
  pb.freeMask.resize(pb.Vp);
  for (uint32_t i = 0; i < pb.Vp; ++i) {
    const uint32_t v = verts[i];
    ps.local[v] = i;
    for (int k = 0; k < 3; ++k) pb.rest[3ull * i + k] = m.positions[3ull * v + k];
    pb.mass[i] = sc.masses[v];
    pb.incident[i] = static_cast<uint32_t>(g.adjStart[v + 1] - g.adjStart[v]);
    pb.freeMask[i] = ps.vertexMark[v] == e ? 1 : 0;
    if (v == s) *sLocal = i;
  }
  pb.tets.resize(4ull * pb.Tp);
  pb.mats.resize(pb.Tp);
  pb.vol.resize(forTraining ? pb.Tp : 0);
  pb.invRest.resize(forTraining ? 9ull * pb.Tp : 0);
  for (uint32_t i = 0; i < pb.Tp; ++i) {
    const uint32_t t = tets[i];
    for (int l = 0; l < 4; ++l) pb.tets[4ull * i + l] = ps.local[m.tets[4ull * t + l]];
    pb.mats[i] = &sc.materialTable[m.materials[t]];
    if (!forTraining) continue;
    pb.vol[i] = sc.rest.volumes[t];
    std::memcpy(&pb.invRest[9ull * i], &sc.rest.inverseRest[9ull * t], 9 * sizeof(double));
  }
}

// Quantised signature of a patch relative to its source vertex: sizes, the
// source's local id, every vertex's offset from the source (quantised to
// 1e-9 of the patch extent), mass ratio, incident count and free flag, and
// every tetrahedron's local vertices and material.
void patchSignature(const Scene& sc, const Problem& pb, uint32_t sLocal, std::vector<int64_t>& sig) {
  sig.clear();
  sig.reserve(8 + 6ull * pb.Vp + 5ull * pb.Tp);
  sig.push_back(pb.Vp);
  sig.push_back(pb.Tp);
  sig.push_back(sLocal);
  double scale = 0;
  for (uint32_t i = 0; i < pb.Vp; ++i)
    for (int k = 0; k < 3; ++k)
      scale = std::max(scale, std::fabs(pb.rest[3ull * i + k] - pb.rest[3ull * sLocal + k]));
  const double q = std::max(scale, 1e-300) * 1e-9;
  for (uint32_t i = 0; i < pb.Vp; ++i) {
    for (int k = 0; k < 3; ++k)
      sig.push_back(std::llround((pb.rest[3ull * i + k] - pb.rest[3ull * sLocal + k]) / q));
    sig.push_back(std::llround(pb.mass[i] * 1e9 / std::max(pb.mass[sLocal], 1e-300)));
    sig.push_back(pb.incident[i]);
    sig.push_back(pb.freeMask[i]);
  }
  for (uint32_t i = 0; i < pb.Tp; ++i) {
    for (int l = 0; l < 4; ++l) sig.push_back(pb.tets[4ull * i + l]);
    sig.push_back(pb.mats[i] - sc.materialTable.data());
  }
}

// 64-bit hash of a signature, one multiply-xorshift round per word; equal
// hashes are confirmed by comparing the signatures themselves.
uint64_t hashSignature(const std::vector<int64_t>& sig) {
  uint64_t h = 0x9e3779b97f4a7c15ull ^ sig.size();
  for (int64_t v : sig) {
    h ^= static_cast<uint64_t>(v);
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 32;
  }
  return h;
}

void writeRecords(Scene& sc, uint32_t globalVertex, const Problem& pb,
                  const std::vector<LocalRecord>& recs, uint32_t K) {
  for (size_t i = 0; i < recs.size() && i < K; ++i) {
    const size_t r = static_cast<size_t>(globalVertex) * K + i;
    sc.recordTets[r] = pb.globalTet[recs[i].tet];
    sc.recordWeights[r] = static_cast<float>(recs[i].weight);
    for (int e = 0; e < 36; ++e) sc.recordBasis[36 * r + e] = static_cast<float>(recs[i].basis[e]);
  }
}

}  // namespace

bool runPrecompute(Scene& sc, const jgs2_precompute_options& opt, jgs2_precompute_stats* stats) {
  const auto start = std::chrono::steady_clock::now();
  const Mesh& m = sc.mesh;
  const uint32_t V = m.vertexCount();
  const uint32_t K = opt.cubature_k;
  // The thread count applies to this precompute only; the process's OpenMP
  // setting is restored on every return.
  struct ThreadCount {
    int saved = omp_get_max_threads();
    ~ThreadCount() { omp_set_num_threads(saved); }
  } threadCount;
  if (opt.threads > 0) omp_set_num_threads(static_cast<int>(opt.threads));
  sc.timestep = opt.timestep;
  sc.cubatureK = K;
  sc.recordTets.assign(static_cast<size_t>(V) * K, 0xffffffffu);
  sc.recordWeights.assign(static_cast<size_t>(V) * K, 0.f);
  sc.recordBasis.assign(static_cast<size_t>(V) * K * 36, 0.f);
  bool anyStable = false, anyCorotated = false;
  for (uint32_t t = 0; t < m.tetCount(); ++t) {
    if (sc.materialTable[m.materials[t]].model == JGS2_MATERIAL_STABLE_NEO_HOOKEAN) anyStable = true;
    else anyCorotated = true;
  }
  if (anyStable && anyCorotated) {
    sc.error = "Mixed stable Neo-Hookean/co-rotated nonlinear Cubature preprocessing is not implemented.";
    return false;
  }
  jgs2_precompute_stats st{};
  bool gpu = false;
  if (!opt.exact_complement && opt.selection_device != JGS2_SELECTION_CPU) {
    const SelectionDevice device = selectionDevice();
    if (opt.selection_device == JGS2_SELECTION_GPU && device != SelectionDevice::kUsable) {
      sc.error = device == SelectionDevice::kNone
                     ? "GPU cubature selection was requested, but no CUDA device is visible."
                     : "GPU cubature selection was requested, but the current CUDA device is not sm_100.";
      return false;
    }
    gpu = device == SelectionDevice::kUsable;
  }
  st.selection_on_gpu = gpu ? 1 : 0;
  std::vector<double> residuals(V, -1.0);
  std::vector<uint32_t> incident(V, 0);
  for (uint32_t v : m.tets) incident[v]++;
  if (opt.method == JGS2_PRECOMPUTE_EXACT) {
    Problem pb;
    pb.Vp = V;
    pb.Tp = m.tetCount();
    pb.globalVertex.resize(V);
    std::iota(pb.globalVertex.begin(), pb.globalVertex.end(), 0u);
    pb.globalTet.resize(pb.Tp);
    std::iota(pb.globalTet.begin(), pb.globalTet.end(), 0u);
    pb.rest = m.positions;
    pb.mass = sc.masses;
    pb.incident = incident;
    pb.freeMask.resize(V);
    for (uint32_t v = 0; v < V; ++v) pb.freeMask[v] = m.fixed[v] ? 0 : 1;
    pb.tets = m.tets;
    pb.vol = sc.rest.volumes;
    pb.invRest = sc.rest.inverseRest;
    pb.mats.resize(pb.Tp);
    for (uint32_t t = 0; t < pb.Tp; ++t) pb.mats[t] = &sc.materialTable[m.materials[t]];
    Context ctx;
    ctx.pb = &pb;
    ctx.h = opt.timestep;
    if (!buildSystem(ctx)) { sc.error = "A simulation scene must have at least one movable vertex."; return false; }
    prepareTraining(ctx, opt, anyCorotated);
    st.training_classes = 1;
    st.reduced_amplitude_classes = ctx.amplitudeReduced ? 1 : 0;
    std::vector<uint32_t> sources;
    for (uint32_t v = 0; v < V; ++v)
      if (!m.fixed[v] && incident[v] > 0) sources.push_back(v);
    std::vector<std::string> errors(omp_get_max_threads());
    const auto trainStart = std::chrono::steady_clock::now();
    if (!gpu) {
#pragma omp parallel for schedule(dynamic, 1)
      for (int64_t i = 0; i < static_cast<int64_t>(sources.size()); ++i) {
        std::vector<LocalRecord> recs;
        try {
          residuals[sources[i]] = trainSource(ctx, sources[i], opt, recs);
          writeRecords(sc, sources[i], pb, recs, K);
        } catch (const std::exception& e) {
          errors[omp_get_thread_num()] = e.what();
        }
      }
    } else {
      // Training systems built on the CPU threads, selections in GPU batches
      // of about selectionBatchBytes() of columns.
      const size_t S = sources.size(), group = 4 * static_cast<size_t>(omp_get_max_threads());
      const size_t budget = selectionBatchBytes();
      for (size_t next = 0; next < S;) {
        std::vector<std::unique_ptr<TrainingJob>> jobs;
        size_t bytes = 0;
        while (next < S && bytes < budget) {
          const size_t first = jobs.size(), n = std::min(S - next, group);
          for (size_t i = 0; i < n; ++i) {
            jobs.emplace_back(new TrainingJob);
            jobs.back()->source = sources[next + i];
          }
#pragma omp parallel for schedule(dynamic, 1)
          for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
            try {
              buildJob(ctx, opt, *jobs[first + i]);
            } catch (const std::exception& e) {
              errors[omp_get_thread_num()] = e.what();
            }
          }
          for (size_t i = first; i < jobs.size(); ++i) bytes += jobs[i]->bytes();
          next += n;
        }
        for (const auto& e : errors)
          if (!e.empty()) { sc.error = e; return false; }
        std::vector<TrainingJob*> batch;
        for (auto& j : jobs) batch.push_back(j.get());
        const auto selectStart = std::chrono::steady_clock::now();
        const std::string err = selectBatchOnGpu(batch, &pb);
        st.selection_seconds += secondsSince(selectStart);
        if (!err.empty()) { sc.error = err; return false; }
        st.selection_batches++;
        for (auto& j : jobs) {
          residuals[j->source] = j->residual;
          writeRecords(sc, j->source, pb, j->records, K);
        }
      }
    }
    st.training_seconds = secondsSince(trainStart);
    for (const auto& e : errors)
      if (!e.empty()) { sc.error = e; return false; }
  } else {
    const MeshGraph g = buildGraph(m);
    std::vector<uint32_t> sources;
    for (uint32_t v = 0; v < V; ++v)
      if (!m.fixed[v] && incident[v] > 0) sources.push_back(v);
    const size_t S = sources.size();
    std::vector<uint64_t> hashes(S);
    std::vector<PatchScratch> scratch(omp_get_max_threads());
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < static_cast<int64_t>(S); ++i) {
      PatchScratch& ps = scratch[omp_get_thread_num()];
      uint32_t sl = 0;
      extractPatch(sc, g, sources[i], opt.patch_radius, ps.pb, &sl, ps, false);
      patchSignature(sc, ps.pb, sl, ps.signature);
      hashes[i] = hashSignature(ps.signature);
    }
    // Group by hash; the first vertex of each group is its representative.
    std::unordered_map<uint64_t, uint32_t> classOf;
    std::vector<size_t> reps;
    std::vector<uint32_t> cls(S);
    for (size_t i = 0; i < S; ++i) {
      auto it = classOf.find(hashes[i]);
      if (it == classOf.end()) {
        const uint32_t c = static_cast<uint32_t>(reps.size());
        classOf.emplace(hashes[i], c);
        reps.push_back(i);
        cls[i] = c;
      } else {
        cls[i] = it->second;
      }
    }
    const size_t C = reps.size();
    std::vector<std::vector<LocalRecord>> classRecords(C);
    std::vector<std::vector<int64_t>> classSig(C);
    std::vector<double> classResidual(C, 0.0);
    std::vector<uint8_t> classReduced(C, 0);
    std::vector<std::string> errors(omp_get_max_threads());
    const auto trainStart = std::chrono::steady_clock::now();
    if (!gpu) {
#pragma omp parallel for schedule(dynamic, 1)
      for (int64_t c = 0; c < static_cast<int64_t>(C); ++c) {
        try {
          Problem pb;
          uint32_t sl = 0;
          extractPatch(sc, g, sources[reps[c]], opt.patch_radius, pb, &sl, scratch[omp_get_thread_num()], true);
          patchSignature(sc, pb, sl, classSig[c]);
          Context ctx;
          ctx.pb = &pb;
          ctx.h = opt.timestep;
          if (!buildSystem(ctx)) continue;
          prepareTraining(ctx, opt, anyCorotated);
          classReduced[c] = ctx.amplitudeReduced ? 1 : 0;
          classResidual[c] = trainSource(ctx, sl, opt, classRecords[c]);
        } catch (const std::exception& e) {
          errors[omp_get_thread_num()] = e.what();
        }
      }
    } else {
      // Class systems built on the CPU threads, selections in GPU batches of
      // about selectionBatchBytes() of columns.
      const size_t group = 4 * static_cast<size_t>(omp_get_max_threads());
      const size_t budget = selectionBatchBytes();
      for (size_t next = 0; next < C;) {
        std::vector<std::unique_ptr<TrainingJob>> jobs;
        size_t bytes = 0;
        const size_t batchFirst = next;
        while (next < C && bytes < budget) {
          const size_t first = jobs.size(), n = std::min(C - next, group);
          for (size_t i = 0; i < n; ++i) jobs.emplace_back(new TrainingJob);
#pragma omp parallel for schedule(dynamic, 1)
          for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
            const size_t c = next + i;
            TrainingJob& job = *jobs[first + i];
            try {
              extractPatch(sc, g, sources[reps[c]], opt.patch_radius, job.pb, &job.source,
                           scratch[omp_get_thread_num()], true);
              patchSignature(sc, job.pb, job.source, classSig[c]);
              Context ctx;
              ctx.pb = &job.pb;
              ctx.h = opt.timestep;
              if (!buildSystem(ctx)) continue;
              prepareTraining(ctx, opt, anyCorotated);
              job.reduced = ctx.amplitudeReduced;
              buildJob(ctx, opt, job);
            } catch (const std::exception& e) {
              errors[omp_get_thread_num()] = e.what();
            }
          }
          for (size_t i = first; i < jobs.size(); ++i) bytes += jobs[i]->bytes();
          next += n;
        }
        for (const auto& e : errors)
          if (!e.empty()) { sc.error = e; return false; }
        std::vector<TrainingJob*> batch;
        for (auto& j : jobs) batch.push_back(j.get());
        const auto selectStart = std::chrono::steady_clock::now();
        const std::string err = selectBatchOnGpu(batch, nullptr);
        st.selection_seconds += secondsSince(selectStart);
        if (!err.empty()) { sc.error = err; return false; }
        st.selection_batches++;
        for (size_t i = 0; i < jobs.size(); ++i) {
          const size_t c = batchFirst + i;
          if (!jobs[i]->trained) continue;
          classReduced[c] = jobs[i]->reduced ? 1 : 0;
          classResidual[c] = jobs[i]->residual;
          classRecords[c] = std::move(jobs[i]->records);
        }
      }
    }
    st.training_seconds = secondsSince(trainStart);
    for (const auto& e : errors)
      if (!e.empty()) { sc.error = e; return false; }
    std::vector<uint8_t> mismatch(S, 0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < static_cast<int64_t>(S); ++i) {
      PatchScratch& ps = scratch[omp_get_thread_num()];
      uint32_t sl = 0;
      extractPatch(sc, g, sources[i], opt.patch_radius, ps.pb, &sl, ps, false);
      const uint32_t c = cls[i];
      if (static_cast<size_t>(i) != reps[c]) {
        patchSignature(sc, ps.pb, sl, ps.signature);
        if (ps.signature != classSig[c]) {
          mismatch[i] = 1;  // hash collision: train this vertex on its own
          continue;
        }
      }
      writeRecords(sc, sources[i], ps.pb, classRecords[c], K);
      residuals[sources[i]] = classResidual[c];
    }
    for (size_t i = 0; i < S; ++i) {
      if (!mismatch[i]) continue;
      Problem pb;
      uint32_t sl = 0;
      extractPatch(sc, g, sources[i], opt.patch_radius, pb, &sl, scratch[0], true);
      Context ctx;
      ctx.pb = &pb;
      ctx.h = opt.timestep;
      if (!buildSystem(ctx)) continue;
      prepareTraining(ctx, opt, anyCorotated);
      std::vector<LocalRecord> recs;
      residuals[sources[i]] = trainSource(ctx, sl, opt, recs);
      writeRecords(sc, sources[i], pb, recs, K);
      st.training_classes++;
    }
    st.training_classes += static_cast<uint32_t>(C);
    for (uint8_t r : classReduced) st.reduced_amplitude_classes += r;
  }
  double sum = 0;
  uint32_t count = 0;
  for (uint32_t v = 0; v < V; ++v) {
    if (residuals[v] < 0) continue;
    count++;
    sum += residuals[v];
    st.max_residual = std::max(st.max_residual, residuals[v]);
    if (residuals[v] > kResidualTolerance) st.vertices_over_tolerance++;
    uint32_t nrec = 0;
    for (uint32_t k = 0; k < K; ++k)
      if (sc.recordWeights[static_cast<size_t>(v) * K + k] > 0) nrec++;
    st.records_written += nrec;
    st.max_records_per_vertex = std::max(st.max_records_per_vertex, nrec);
  }
  st.source_vertices = count;
  st.mean_residual = count ? sum / count : 0;
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
  if (stats) *stats = st;
  return true;
}

}  // namespace jgs2scene

extern "C" {

// selectGreedyNonnegativeColumns (src/simulation/cpu/cubature.ts:508-690)
// over caller columns, through the cubature trainer's own selection core
// (the candidate filter, the greedy growth by exhaustive NNLS fits, the
// refinement swaps and the final residual), which the GPU selection matches
// bit for bit.
jgs2_status jgs2_select_nonnegative_columns(const double* columns, uint32_t column_count, uint32_t rows,
                                            const double* target, uint32_t max_columns, uint32_t refinement_passes,
                                            double residual_tolerance, uint32_t* selected, double* weights,
                                            uint32_t* selected_count, double* normalized_residual) {
  using namespace jgs2scene;
  if (rows == 0 || !target || !selected_count || !normalized_residual || (column_count > 0 && !columns) ||
      (max_columns > 0 && (!selected || !weights)) || max_columns > static_cast<uint32_t>(jgs2select::kMaxColumns) ||
      !(residual_tolerance >= 0.0 && residual_tolerance <= 1.0))
    return JGS2_INVALID_ARGUMENT;
  const size_t n = static_cast<size_t>(column_count) * rows;
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(columns[i])) return JGS2_INVALID_ARGUMENT;
  for (uint32_t r = 0; r < rows; ++r)
    if (!std::isfinite(target[r])) return JGS2_INVALID_ARGUMENT;
  try {
    Training tr;
    tr.cols.resize(column_count);
    for (uint32_t c = 0; c < column_count; ++c)
      tr.cols[c].assign(columns + static_cast<size_t>(c) * rows, columns + static_cast<size_t>(c + 1) * rows);
    tr.target.assign(target, target + rows);
    tr.maxColumns = static_cast<int>(max_columns);
    tr.passes = static_cast<int>(refinement_passes);
    const Candidates cs = candidates(tr);
    const Selection sel = finishSelection(tr, cs, selectOnCpu(tr, cs, residual_tolerance));
    *selected_count = static_cast<uint32_t>(sel.tets.size());
    for (size_t i = 0; i < sel.tets.size(); ++i) {
      selected[i] = static_cast<uint32_t>(sel.tets[i]);
      weights[i] = sel.weights[i];
    }
    *normalized_residual = sel.residual;
  } catch (const std::exception&) {
    return JGS2_INVALID_ARGUMENT;
  }
  return JGS2_OK;
}

}  // extern "C"
