// GPU greedy cubature selection (select_gpu.cu): many training problems, one
// thread block each.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "cubature_select.hpp"

namespace jgs2scene {

// One selection problem after the host's candidate filter: `rows` x `cand`
// candidate columns stored row-major (cols[r * cand + i]), their squared norms
// cc[i] and target dot products ct[i], the target's squared norm tt and norm
// tn, the column limit (1..12) and the number of refinement passes.
struct SelectInput {
  const double* cols = nullptr;
  const double* cc = nullptr;
  const double* ct = nullptr;
  uint32_t rows = 0, cand = 0, limit = 0, passes = 0;
  double tt = 0, tn = 0;
};

// The selected candidates (indices into the problem's candidates, in slot
// order) and their weights.
struct SelectOutput {
  int32_t count = 0;
  int32_t sel[jgs2select::kMaxColumns];
  double weights[jgs2select::kMaxColumns];
};

// The calling thread's current CUDA device: none (no device or driver), one
// this library's sm_100a code runs on, or another architecture.
enum class SelectionDevice { kNone, kUsable, kOtherArchitecture };
SelectionDevice selectionDevice();

// Runs every problem's selection on the current CUDA device; returns an empty
// string, or the failing CUDA call and its error.
std::string selectOnGpu(const std::vector<SelectInput>& in, std::vector<SelectOutput>& out);

}  // namespace jgs2scene
