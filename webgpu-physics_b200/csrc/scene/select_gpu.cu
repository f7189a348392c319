// Greedy nonnegative cubature selection on the GPU: one thread block per
// training problem (a patch class or a source vertex).  Each greedy step and
// each refinement pass evaluates all its trials in parallel (one exhaustive
// small NNLS per thread), then one warp replays the reference's sequential
// scan over the trial residuals; the winner's dot-product row is recomputed by
// the whole block.  The arithmetic is cubature_select.hpp's, compiled with
// --fmad=false, so every selection equals the CPU trainer's bit for bit.
//
// Restates selectGreedyNonnegativeColumns (src/simulation/cpu/cubature.ts:
// 508-690) with solveSmallNnls (cubature.ts:387-440).
//
// Sets of at most six columns (every reference scene trains K = 6) take a
// register-resident NNLS: each thread's trial Gram sits in shared memory and
// every subset is solved in the full 6 x 6 frame, its inactive rows and
// columns replaced by the identity, with all loops unrolled.  That solve
// performs the subset's own eliminations on the same values in the same
// order; the identity rows never become pivots (their entries in active
// columns are zero and a pivot must be strictly larger) and only add or
// subtract zeros, so every nonzero value, every pivot decision and every
// residual equals the compacted solve's.  Only the sign of a zero can differ,
// and the weights pass through max(0, x), which returns +0 for both.
#include <cuda_runtime.h>

#include <cstring>

#include "select_gpu.hpp"

namespace jgs2scene {
namespace {

using jgs2select::Gram;
using jgs2select::improves;
using jgs2select::kMaxColumns;
using jgs2select::kResidualTolerance;
using jgs2select::maxd;
using jgs2select::smallNnls;
using jgs2select::swapGram;

struct DeviceProblem {
  uint64_t data;     // doubles: rows x cand columns (row-major), cc[cand], ct[cand]
  uint64_t scratch;  // doubles: dot rows of the selected columns [N x cand], trial residuals [N x cand]
  uint32_t rows, cand, limit, passes;
  double tt, tn;
};

constexpr int kThreads = 256;

__device__ bool chosen(const int* sel, int k, int ci) {
  bool hit = false;
  for (int s = 0; s < k; ++s) hit |= sel[s] == ci;
  return hit;
}

// The reference's sequential scan over trials in item order (item = slot *
// cand + ci) under `improves`, replayed by one warp: each round finds the
// first lane past the last winner whose trial beats the incumbent.  The lanes
// before it do not beat the same incumbent, so the sequential scan would pass
// them by unchanged; the result is the scan's.  Each round moves `after`
// forward, so a chunk takes at most 32 rounds.
__device__ void scanTrials(const double* errs, int items, int cand, const int* sel, int k, double startErr,
                           int* winSlot, int* winCi, double* winErr) {
  const int lane = threadIdx.x & 31;
  int best = -1;
  double bestErr = startErr;
  for (int base = 0; base < items; base += 32) {
    const int i = base + lane;
    const int ci = i % cand;
    const bool valid = i < items && !chosen(sel, k, ci);
    const double e = valid ? errs[i] : 0.0;
    int after = -1;
    for (;;) {
      const bool have = best >= 0;
      const bool up = valid && lane > after && improves(e, bestErr, have, ci, have ? best % cand : 0);
      const unsigned m = __ballot_sync(0xffffffffu, up);
      if (m == 0) break;
      const int j = __ffs(m) - 1;
      bestErr = __shfl_sync(0xffffffffu, e, j);
      best = base + j;
      after = j;
    }
  }
  if (lane == 0) {
    *winSlot = best < 0 ? -1 : best / cand;
    *winCi = best < 0 ? -1 : best % cand;
    *winErr = bestErr;
  }
}

using jgs2select::kPivotFloor;

// The Gram system of one trial for the six-column path, written to this
// thread's slice of shared memory: G[r][c] at g[(6r + c) * kThreads], b[r] at
// g[(36 + r) * kThreads].  Same entries as swapGram; rows and columns at and
// past kk are not written and not read.
__device__ void swapGramShared(double* g, const int* sel, int kk, int slot, int ci, const double* dsel,
                               size_t stride, const double* cc, const double* ct) {
  for (int r = 0; r < kk; ++r) {
    const int a = r == slot ? ci : sel[r];
    g[(36 + r) * kThreads] = ct[a];
    for (int c = 0; c < kk; ++c) {
      const int b = c == slot ? ci : sel[c];
      double v;
      if (r != slot) v = dsel[static_cast<size_t>(r) * stride + b];
      else if (c != slot) v = dsel[static_cast<size_t>(c) * stride + a];
      else v = cc[a];
      g[(6 * r + c) * kThreads] = v;
    }
  }
}

// jgs2select::smallNnls for kk <= 6 columns, every subset solved in the
// embedded 6 x 6 frame with unrolled loops (registers only).  Returns the
// best residual; the weights are not needed by the trials.
__device__ double smallNnls6(const double* g, double tt, int kk) {
  double b[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) b[r] = r < kk ? g[(36 + r) * kThreads] : 0.0;
  double best = tt;
  const int masks = 1 << kk;
  for (int mask = 1; mask < masks; ++mask) {
    double A[6][6], x[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const bool ar = (mask >> r) & 1;
      x[r] = ar ? b[r] : 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const bool ac = (mask >> c) & 1;
        A[r][c] = (ar && ac) ? g[(6 * r + c) * kThreads] : (r == c ? 1.0 : 0.0);
      }
    }
    bool ok = true;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      int pivot = p;
      double pivotMag = fabs(A[p][p]);
#pragma unroll
      for (int r = p + 1; r < 6; ++r) {
        const double m = fabs(A[r][p]);
        if (m > pivotMag) {
          pivotMag = m;
          pivot = r;
        }
      }
      ok = ok && !(pivotMag <= kPivotFloor || !(pivotMag <= DBL_MAX));
#pragma unroll
      for (int r = p + 1; r < 6; ++r) {
        if (r == pivot) {
#pragma unroll
          for (int c = p; c < 6; ++c) {
            const double t = A[p][c];
            A[p][c] = A[r][c];
            A[r][c] = t;
          }
          const double t = x[p];
          x[p] = x[r];
          x[r] = t;
        }
      }
      const double d = A[p][p];
#pragma unroll
      for (int r = p + 1; r < 6; ++r) {
        const double f = A[r][p] / d;
        A[r][p] = 0;
#pragma unroll
        for (int c = p + 1; c < 6; ++c) A[r][c] -= f * A[p][c];
        x[r] -= f * x[p];
      }
    }
    if (!ok) continue;
#pragma unroll
    for (int r = 5; r >= 0; --r) {
      double v = x[r];
#pragma unroll
      for (int c = r + 1; c < 6; ++c) v -= A[r][c] * x[c];
      x[r] = v / A[r][r];
    }
    bool neg = false;
#pragma unroll
    for (int r = 0; r < 6; ++r) neg |= x[r] < -1e-10;
    if (neg) continue;
    double cw[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) cw[c] = ((mask >> c) & 1) ? maxd(0.0, x[c]) : 0.0;
    double err = tt;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (r >= kk || cw[r] == 0) continue;
      err -= 2 * cw[r] * b[r];
#pragma unroll
      for (int c = 0; c < 6; ++c)
        if (c < kk) err += cw[r] * g[(6 * r + c) * kThreads] * cw[c];
    }
    if (err < best - 1e-14 * maxd(1.0, best)) best = err;
  }
  return best;
}

// One trial's residual: the six-column path through shared memory, or the
// shared header's NNLS.
template <int N>
__device__ double trialResidual(double* gram, const int* sel, int kk, int slot, int ci, const double* dsel,
                                size_t stride, const double* cc, const double* ct, double tt) {
  if constexpr (N == 6) {
    swapGramShared(gram, sel, kk, slot, ci, dsel, stride, cc, ct);
    return smallNnls6(gram, tt, kk);
  } else {
    Gram<N> g;
    double w[N];
    swapGram(g, sel, kk, slot, ci, dsel, stride, cc, ct, tt);
    return smallNnls(g, w);
  }
}

// Shared memory of the six-column path: each thread's trial Gram (36 + 6).
constexpr size_t kGramSharedBytes = 42 * kThreads * sizeof(double);

template <int N>
__global__ void __launch_bounds__(kThreads) greedySelectKernel(const DeviceProblem* problems, const double* data,
                                                               double* scratch, SelectOutput* out) {
  const DeviceProblem p = problems[blockIdx.x];
  const int C = static_cast<int>(p.cand);
  const size_t R = p.rows;
  const double* cols = data + p.data;
  const double* cc = cols + R * C;
  const double* ct = cc + C;
  double* dsel = scratch + p.scratch;
  double* errs = dsel + static_cast<size_t>(N) * C;
  __shared__ int sel[N];
  __shared__ double weights[N];
  __shared__ int winSlot, winCi;
  __shared__ double winErr;
  extern __shared__ double gramShared[];
  const int tid = threadIdx.x;
  double* gram = gramShared + tid;

  // dsel[slot][i] = col(sel[slot]) · col(i), summed over rows in order.
  auto setRow = [&](int slot) {
    const int a = sel[slot];
    for (int i = tid; i < C; i += kThreads) {
      double s = 0;
      for (size_t r = 0; r < R; ++r) s += cols[r * C + a] * cols[r * C + i];
      dsel[static_cast<size_t>(slot) * C + i] = s;
    }
  };

  int k = 0;
  double err = p.tt;
  // Greedy growth: every unchosen candidate appended as the last slot.
  for (int step = 0; step < static_cast<int>(p.limit); ++step) {
    for (int ci = tid; ci < C; ci += kThreads) {
      if (chosen(sel, k, ci)) continue;
      errs[ci] = trialResidual<N>(gram, sel, k + 1, k, ci, dsel, C, cc, ct, p.tt);
    }
    __syncthreads();
    if (tid < 32) scanTrials(errs, C, C, sel, k, err, &winSlot, &winCi, &winErr);
    __syncthreads();
    if (winCi < 0) break;
    if (tid == 0) {
      Gram<N> g;
      swapGram(g, sel, k + 1, k, winCi, dsel, C, cc, ct, p.tt);
      smallNnls(g, weights);
      sel[k] = winCi;
    }
    __syncthreads();
    setRow(k);
    ++k;
    err = winErr;
    __syncthreads();
    if (sqrt(maxd(err, 0.0)) / p.tn < kResidualTolerance) break;
  }
  // Refinement passes: the best single swap of a chosen slot, until none helps.
  for (int pass = 0; pass < static_cast<int>(p.passes) && k > 0; ++pass) {
    const int items = k * C;
    for (int i = tid; i < items; i += kThreads) {
      const int slot = i / C, ci = i - slot * C;
      if (chosen(sel, k, ci)) continue;
      errs[i] = trialResidual<N>(gram, sel, k, slot, ci, dsel, C, cc, ct, p.tt);
    }
    __syncthreads();
    if (tid < 32) scanTrials(errs, items, C, sel, k, err, &winSlot, &winCi, &winErr);
    __syncthreads();
    if (winCi < 0) break;
    if (tid == 0) {
      Gram<N> g;
      swapGram(g, sel, k, winSlot, winCi, dsel, C, cc, ct, p.tt);
      smallNnls(g, weights);
      sel[winSlot] = winCi;
    }
    __syncthreads();
    setRow(winSlot);
    err = winErr;
    __syncthreads();
  }
  SelectOutput& o = out[blockIdx.x];
  if (tid == 0) o.count = k;
  if (tid < k) {
    o.sel[tid] = sel[tid];
    o.weights[tid] = weights[tid];
  }
}

// Device allocations and the stream of one selection call, released on exit.
struct Resources {
  double* data = nullptr;
  double* scratch = nullptr;
  DeviceProblem* problems = nullptr;
  SelectOutput* out = nullptr;
  cudaStream_t stream = nullptr;
  ~Resources() {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(data);
    cudaFree(scratch);
    cudaFree(problems);
    cudaFree(out);
    if (stream) cudaStreamDestroy(stream);
  }
};

std::string failed(const char* what, cudaError_t e) {
  return std::string("GPU cubature selection: ") + what + " failed: " + cudaGetErrorString(e);
}

}  // namespace

SelectionDevice selectionDevice() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return SelectionDevice::kNone;
  }
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess) {
    cudaGetLastError();
    return SelectionDevice::kNone;
  }
  // The library carries sm_100a code only.
  return major == 10 && minor == 0 ? SelectionDevice::kUsable : SelectionDevice::kOtherArchitecture;
}

std::string selectOnGpu(const std::vector<SelectInput>& in, std::vector<SelectOutput>& out) {
  out.assign(in.size(), SelectOutput{});
  if (in.empty()) return {};
  int width = 6;
  for (const SelectInput& p : in)
    if (p.limit > 6) width = kMaxColumns;
  std::vector<DeviceProblem> desc(in.size());
  uint64_t dataLen = 0, scratchLen = 0;
  for (size_t i = 0; i < in.size(); ++i) {
    const SelectInput& p = in[i];
    if (p.cand == 0 || p.limit == 0 || p.limit > static_cast<uint32_t>(kMaxColumns))
      return "GPU cubature selection: a problem without candidates or with more than 12 columns";
    desc[i] = DeviceProblem{dataLen, scratchLen, p.rows, p.cand, p.limit, p.passes, p.tt, p.tn};
    dataLen += (static_cast<uint64_t>(p.rows) + 2) * p.cand;
    scratchLen += 2ull * width * p.cand;
  }
  std::vector<double> host(dataLen);
  for (size_t i = 0; i < in.size(); ++i) {
    const SelectInput& p = in[i];
    double* d = host.data() + desc[i].data;
    const size_t n = static_cast<size_t>(p.rows) * p.cand;
    std::memcpy(d, p.cols, n * sizeof(double));
    std::memcpy(d + n, p.cc, p.cand * sizeof(double));
    std::memcpy(d + n + p.cand, p.ct, p.cand * sizeof(double));
  }
  Resources res;
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&res.stream, cudaStreamNonBlocking)) != cudaSuccess)
    return failed("cudaStreamCreateWithFlags", e);
  if ((e = cudaMalloc(&res.data, dataLen * sizeof(double))) != cudaSuccess) return failed("cudaMalloc", e);
  if ((e = cudaMalloc(&res.scratch, scratchLen * sizeof(double))) != cudaSuccess) return failed("cudaMalloc", e);
  if ((e = cudaMalloc(&res.problems, desc.size() * sizeof(DeviceProblem))) != cudaSuccess)
    return failed("cudaMalloc", e);
  if ((e = cudaMalloc(&res.out, out.size() * sizeof(SelectOutput))) != cudaSuccess) return failed("cudaMalloc", e);
  if ((e = cudaMemcpyAsync(res.data, host.data(), dataLen * sizeof(double), cudaMemcpyHostToDevice,
                           res.stream)) != cudaSuccess)
    return failed("cudaMemcpyAsync", e);
  if ((e = cudaMemcpyAsync(res.problems, desc.data(), desc.size() * sizeof(DeviceProblem),
                           cudaMemcpyHostToDevice, res.stream)) != cudaSuccess)
    return failed("cudaMemcpyAsync", e);
  const unsigned blocks = static_cast<unsigned>(in.size());
  if (width == 6) {
    if ((e = cudaFuncSetAttribute(greedySelectKernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kGramSharedBytes))) != cudaSuccess)
      return failed("cudaFuncSetAttribute", e);
    greedySelectKernel<6><<<blocks, kThreads, kGramSharedBytes, res.stream>>>(res.problems, res.data, res.scratch,
                                                                              res.out);
  } else
    greedySelectKernel<kMaxColumns><<<blocks, kThreads, 0, res.stream>>>(res.problems, res.data, res.scratch,
                                                                         res.out);
  if ((e = cudaGetLastError()) != cudaSuccess) return failed("greedySelectKernel launch", e);
  if ((e = cudaMemcpyAsync(out.data(), res.out, out.size() * sizeof(SelectOutput), cudaMemcpyDeviceToHost,
                           res.stream)) != cudaSuccess)
    return failed("cudaMemcpyAsync", e);
  if ((e = cudaStreamSynchronize(res.stream)) != cudaSuccess) return failed("greedySelectKernel", e);
  return {};
}

}  // namespace jgs2scene
