// Greedy nonnegative column selection for cubature training, shared by the
// CPU trainer (precompute.cpp) and the GPU trainer (select_gpu.cu).
//
// Restated from src/simulation/cpu/cubature.ts:
//   solveDenseLinearSystem      math.ts:134-199   (partial pivoting, pivot floor 1e-14)
//   solveSmallNnls              cubature.ts:387-440 (exhaustive active-set search,
//                                                   errors from the Gram matrix)
//   selectGreedyNonnegativeColumns cubature.ts:508-690 (greedy growth, then
//                                                   swap refinement passes)
//
// Every function here is plain IEEE double arithmetic in source order (no
// library calls beyond fabs); both sides are compiled without multiply-add
// contraction (g++ -ffp-contract=off, nvcc --fmad=false), so a selection made
// on the GPU is bit for bit the one the CPU makes.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstddef>

#if defined(__CUDACC__)
#define JGS2_SELECT_HD __host__ __device__ inline
#else
#define JGS2_SELECT_HD inline
#endif

namespace jgs2select {

constexpr double kPivotFloor = 1e-14;          // math.ts:1 (MATRIX_EPSILON)
constexpr double kResidualTolerance = 0.01;    // nonlinear-cubature-training.ts:23
constexpr int kMaxColumns = 12;                // exhaustive NNLS limit (cubature.ts:395)

// std::max(a, b) for doubles, spelled out so host and device agree on NaN
// and signed zero: (a < b) ? b : a.
JGS2_SELECT_HD double maxd(double a, double b) { return (a < b) ? b : a; }

// Gram system of a column set: G = Cᵀ C, b = Cᵀ t, tt = tᵀ t.  N bounds the
// set size; the arithmetic does not depend on N.
template <int N>
struct Gram {
  int k = 0;
  double G[N][N];
  double b[N];
  double tt;
};

// In-place Gaussian elimination with partial pivoting on an n x n row-major
// system; false when a pivot is at or below the floor or not finite.
JGS2_SELECT_HD bool solveDense(double* a, double* b, int n) {
  for (int p = 0; p < n; ++p) {
    int best = p;
    double bestMag = fabs(a[p * n + p]);
    for (int r = p + 1; r < n; ++r) {
      const double m = fabs(a[r * n + p]);
      if (m > bestMag) { bestMag = m; best = r; }
    }
    if (bestMag <= kPivotFloor || !(bestMag <= DBL_MAX)) return false;
    if (best != p) {
      for (int c = p; c < n; ++c) {
        const double t = a[p * n + c];
        a[p * n + c] = a[best * n + c];
        a[best * n + c] = t;
      }
      const double t = b[p];
      b[p] = b[best];
      b[best] = t;
    }
    const double d = a[p * n + p];
    for (int r = p + 1; r < n; ++r) {
      const double f = a[r * n + p] / d;
      a[r * n + p] = 0;
      for (int c = p + 1; c < n; ++c) a[r * n + c] -= f * a[p * n + c];
      b[r] -= f * b[p];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    double v = b[r];
    for (int c = r + 1; c < n; ++c) v -= a[r * n + c] * b[c];
    b[r] = v / a[r * n + r];
  }
  return true;
}

// Exhaustive active-set NNLS over the k columns of g: every nonempty subset
// is solved unconstrained; subsets with a coefficient below -1e-10 are
// discarded; the smallest squared residual (tt - 2 wᵀb + wᵀGw) wins, a later
// subset only when smaller by more than 1e-14 relative.  Returns the residual
// and writes the weights (zero outside the winning subset).
template <int N>
JGS2_SELECT_HD double smallNnls(const Gram<N>& g, double* w) {
  const int k = g.k;
  double best = g.tt;
  for (int i = 0; i < k; ++i) w[i] = 0;
  double A[N * N], rhs[N], cw[N];
  int active[N];
  for (int mask = 1; mask < (1 << k); ++mask) {
    int d = 0;
    for (int c = 0; c < k; ++c)
      if (mask & (1 << c)) active[d++] = c;
    for (int r = 0; r < d; ++r) {
      rhs[r] = g.b[active[r]];
      for (int c = 0; c < d; ++c) A[r * d + c] = g.G[active[r]][active[c]];
    }
    if (!solveDense(A, rhs, d)) continue;
    bool neg = false;
    for (int r = 0; r < d; ++r) neg |= rhs[r] < -1e-10;
    if (neg) continue;
    for (int c = 0; c < k; ++c) cw[c] = 0;
    for (int r = 0; r < d; ++r) cw[active[r]] = maxd(0.0, rhs[r]);
    double err = g.tt;
    for (int r = 0; r < k; ++r) {
      if (cw[r] == 0) continue;
      err -= 2 * cw[r] * g.b[r];
      for (int c = 0; c < k; ++c) err += cw[r] * g.G[r][c] * cw[c];
    }
    if (err < best - 1e-14 * maxd(1.0, best)) {
      best = err;
      for (int c = 0; c < k; ++c) w[c] = cw[c];
    }
  }
  return best;
}

// The Gram system of the selected set `sel` (kk entries, candidate indices)
// with position `slot` holding candidate `ci` instead.  Growing the set by one
// is the case slot == kk - 1 (sel[kk - 1] is not read).  dsel is row-major,
// dsel[s * stride + i] = col(sel[s]) · col(i); cc[i] = |col(i)|², ct[i] =
// col(i) · t.  The slot's own row and column are read through the other
// rows' dot products, as the reference assembles the trial system.
template <int N>
JGS2_SELECT_HD void swapGram(Gram<N>& g, const int* sel, int kk, int slot, int ci, const double* dsel,
                             size_t stride, const double* cc, const double* ct, double tt) {
  g.k = kk;
  g.tt = tt;
  for (int r = 0; r < kk; ++r) {
    const int a = r == slot ? ci : sel[r];
    g.b[r] = ct[a];
    for (int c = 0; c < kk; ++c) {
      const int b = c == slot ? ci : sel[c];
      if (r != slot) g.G[r][c] = dsel[static_cast<size_t>(r) * stride + b];
      else if (c != slot) g.G[r][c] = dsel[static_cast<size_t>(c) * stride + a];
      else g.G[r][c] = cc[a];
    }
  }
}

// The scan rule of the greedy step and the refinement passes, applied to
// trials in order: a trial replaces the incumbent when its residual is lower
// by more than 1e-14 relative, or within that of it and on a candidate of
// lower index (candidate ids increase with the candidate index).
JGS2_SELECT_HD bool improves(double e, double bestErr, bool haveBest, int ci, int bestCi) {
  const double tol = 1e-14 * maxd(1.0, bestErr);
  return e < bestErr - tol || (fabs(e - bestErr) <= tol && haveBest && ci < bestCi);
}

}  // namespace jgs2select
