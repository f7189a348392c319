// Device buffers, per-call parameters and kernel launch entry points of the
// JGS2 step.  Shared by jgs2_kernels.cu (device) and jgs2_runtime.cpp (host).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace jgs2 {

// Per-call settings, copied to device memory before each step so captured
// CUDA graphs stay valid across setting changes.  Mirrors the uniform block
// SimParams (src/simulation/gpu/jgs2-shader.ts:141-164).
struct DevParams {
  float dt, invDt, invDt2, maxStep;
  float gravity[3];
  float floorHeight;
  float floorStiffness, regularization, rotationEpsilon, velocityDamping;
  float contactTangentialDamping, contactMargin;
  float residualTolerance, normalizedUpdateTolerance;
  float sceneScale;
  uint32_t objectiveFlags;  // bit0 forces, bit1 targets
  uint32_t stopEnabled;     // convergence latch active (production step)
  uint32_t globalization;   // stable Neo-Hookean path
  uint32_t historyCapacity;
  uint32_t vertexCount, tetCount, cubatureK, bodyCount;
  uint32_t bodyCorrection;  // horizontal body correction in the epilogue
  uint32_t active;          // 0: the scene sits this frame out (no state changes)
  uint32_t cloth;           // the scene has cloth triangles
  // Cloth material (the cloth arena's second global vec4, cloth-layout.ts:45-50).
  float clothLambda, clothMu, clothThickness, clothBending;
  // IPC contact: enabled this frame (candidates, stable path, barrier
  // stiffness > 0, activation above the minimum distance), the per-step
  // activation distance and stiffness (the uniform's contact vec4) and the
  // create-time minimum distance, friction, friction smoothing and step
  // safety (the contact buffer's parameter vec4, jgs2-solver.ts:1096-1105).
  uint32_t ipc;
  float ipcActivation, ipcStiffness, ipcMinDistance, ipcFriction, ipcEpsilon, ipcSafety;
  uint32_t pad2;
};

// One scene of a batch: its slices of the concatenated vertex and tet arrays
// and its slots in the reduction partial arrays.  A single solver is a batch
// of one scene.
struct SceneRange {
  uint32_t vOff, V, tOff, T;
  uint32_t gateBase, gateBlocks;  // prologue / gate partials of this scene
  uint32_t convBase, convBlocks;  // convergence partials of this scene
  uint32_t cOff, C, hOff, H;      // cloth triangles and hinges of this scene
  uint32_t kOff, KC;              // static IPC candidates of this scene
  uint32_t rowOff, rowCount;      // broad-phase rows of this scene (contact surface)
  // Elements one pass of the scene's gate blocks covers (the table's range);
  // broad-phase candidates beyond it stride over the same blocks.
  uint32_t gateSpan, pad[3];
};

// One block of a segmented reduction: elements [begin, end) of `scene`,
// publishing its partial at index `slot`.
struct RedBlock {
  uint32_t scene, begin, end, slot;
};
#ifndef JGS2_GATE_CHUNK
#define JGS2_GATE_CHUNK 2048
#endif
constexpr uint32_t kGateChunk = JGS2_GATE_CHUNK;  // tets / vertices per prologue or gate block
#ifndef JGS2_CONV_CHUNK
#define JGS2_CONV_CHUNK 256
#endif
constexpr uint32_t kConvChunk = JGS2_CONV_CHUNK;  // vertices per convergence block

// Reduction scratch and the GPU-resident control/history records
// (dynamic arena regions globalizationControl/globalizationHistory,
// src/simulation/gpu/layout.ts:418-503).
struct FrameState {
  float4 control[4];
  float4 history[64 * 8];
  // Tickets of the segmented reductions (the last block of the scene folds).
  uint32_t gateTicket, convTicket, prologueTicket;
  // Local diagnostics aggregates of the current sweep (reduceCandidate's
  // vertex loop), accumulated by the solve kernel with order-free atomics.
  uint32_t localFailures, localMaxBacktracks, localSkipped, localEvaluations;
  uint32_t localMaxShift;  // float bits of a non-negative value
  uint32_t localNumericsValid;
  // IPC safe-step reductions (reduceContactStep, jgs2-shader.ts:2870-2907):
  // minimum candidate alpha (float bits) and the all-valid flag of the
  // safe-step pass and of the validation pass, and the resulting contact
  // alpha of the iteration.
  uint32_t stepAlphaBits, stepValid, checkAlphaBits, checkValid;
  float contactAlpha;
  uint32_t pad[2];
};

// All device arrays of one solver.
struct Buffers {
  // dynamic
  float4* pos[2];         // A, B
  float4* predicted;       // inertial target xyz, distributed inertia weight m/(h^2 n) (0 pinned)
  float4* velocity;
  float4* old;
  float4* vertexRot;      // 3 per vertex (columns)
  float4* tetRot;         // 3 per tet (co-rotated only)
  float* finalUpdate;     // per vertex update norm
  float4* local;          // 4 per vertex (local diagnostics)
  // 3 per vertex: the incident-tet part of the local system at the next
  // Jacobi source pose, (g.xyz, Hxx) (Hyy, Hzz, Hxy, Hxz) (Hyz, 0, 0, 0),
  // written by the pass that computes that pose's vertex frames.
  float4* incident;
  FrameState* frames;     // one per scene
  void* gatePartials;     // one GatePartial (32 bytes) per gate / prologue block
  void* convPartials;     // one ConvPartial (80 bytes) per convergence block
  double* bodyAccum;      // 6 per body (mass, solved xz, predicted xz, pinned count)
  // static
  const float4* restMass;     // rest xyz (pin target), mass
  const uint4* vinfo;         // adjacency start, count, pinned, body
  const float4* tets;         // 4 per tet: [g1 vol] [g2 lambda] [g3 mu] [indices as uint]
  const uint32_t* adjacency;  // incident tet * 4 + local slot
  const uint4* cubHead;       // 2 per record: (tet, weight bits, 0, 0), the tet's vertex indices
  const float4* cubBasis;     // 9 float4 per record (36 floats, row-major blocks)
  const float* stiffness;     // 144 per tet (co-rotated only)
  float4* forces;             // external force xyz per vertex
  float4* targets;            // quadratic target xyz, stiffness per vertex
  const uint32_t* colors;     // per vertex colour
  const uint32_t* vertexScene;  // scene of each vertex
  const uint32_t* tetScene;     // scene of each tet (co-rotated engines only)
  const SceneRange* scenes;
  const RedBlock* gateTable;    // prologue / gate blocks
  const RedBlock* convTable;    // convergence blocks
  // Triangle cloth (all null when no scene has cloth): two float4 per
  // triangle (indices as uint + rest area, inverse rest basis), two per hinge
  // (indices as uint, rest angle and edge length), per vertex the incidence
  // ranges (triangle begin, count, hinge begin, count) into `clothIncidence`
  // (element * 4 + local slot).
  const float4* clothTris;
  const float4* clothHinges;
  const uint4* clothRange;
  const uint32_t* clothIncidence;
  // IPC contact (all null without candidates): per candidate its global
  // vertex indices with the type (1 = edge-edge) in bit 31 of the fourth, its
  // scene and 7 float4 of state (jgs2_contact.cuh); per vertex the range
  // (first, count) of its incident candidates in `contactIds` and the count
  // of active ones, listed at the same offsets in `activeIds`.
  uint4* contactIdx;
  uint32_t* contactScene;
  float4* contactState;
  uint2* contactRange;
  const uint32_t* contactIds;
  uint32_t* activeCount;
  uint32_t* activeIds;
  uint32_t* contactFlag;   // per candidate: active this iteration
  float4* contactGrad;     // per vertex: IPC gradient at the accepted pose
  uint32_t gateBlocks, convBlocks, sceneCount, contactCount;
  uint32_t vertexTotal, tetTotal;  // vertices and tets over the scenes (checked builds bound indices by them)
  // IPC broad phase (contact surfaces; all null for static candidates, and
  // contactCount is then the candidate capacity of one iteration).  Rows:
  // one per vertex of a contact scene (vertex-triangle rows) and one per
  // surface edge (edge-edge rows), each (primitive, scene | edge-edge bit 31,
  // first column, end column) over the global surface triangle or edge
  // index; a row's columns are its candidates in the superset's canonical
  // order.  Surface triangles (vertex indices, scene), edges, each vertex's
  // closed surface one-ring; per iteration the primitive and 32-primitive
  // chunk boxes ((lo, motion), (hi, 0)); the current list (row offsets,
  // columns) and the previous iteration's (row offsets, columns, state) for
  // carried caches and lagged friction; per scene its span of the current
  // list; status words (listed candidates, sticky overflow flag, largest
  // count asked for, this iteration's overflow); the sort's key / value
  // ping-pong buffers and tile histograms.
  uint32_t contactDynamic;
  uint32_t bpRowTotal, bpTriTotal, bpEdgeTotal, bpSentinel, bpSortPasses;
  uint32_t bpSuperset;  // candidates of the static superset (clamped to 2^32 - 1)
  // Host-side launch shape: the solve kernel takes its default vertices per
  // block shifted right by this (0-2); scheduling only, never arithmetic.
  uint32_t solveShift;
  const uint4* bpRows;
  const uint4* bpTris;
  const uint2* bpEdges;
  const uint2* bpRing;
  const uint32_t* bpRingIds;
  float4* bpTriBox;
  float4* bpEdgeBox;
  float4* bpTriChunk;
  float4* bpEdgeChunk;
  float4* bpTriSuper;   // 2 per 32 chunks
  float4* bpEdgeSuper;
  uint32_t* bpRowOff;
  const uint32_t* bpPrevRowOff;
  uint32_t* bpCols;
  const uint32_t* bpPrevCols;
  const float4* bpPrevState;
  uint2* bpSpan;
  uint32_t* bpStatus;
  uint32_t* bpKeys[2];
  uint32_t* bpVals[2];
  uint32_t* bpHist;         // 256 digits x tiles, then the 256 digit totals
  uint32_t* bpPinnedMove;   // per vertex: pinned and its snap to rest exceeds maxStep (or is not finite)
  uint32_t* bpPrev;         // per listed candidate: its entry in the previous list, or ~0
};

// Kernel launch entry points (jgs2_kernels.cu).  `p` points at one DevParams
// per scene.  Every launcher returns the number of kernels it launched.
int launchPrologue(const Buffers& b, const DevParams* p, cudaStream_t s);
int launchVertexPolar(const Buffers& b, const DevParams* p, const float4* src, const uint32_t* list,
                      uint32_t count, cudaStream_t s);
// cachedIncident: take the incident-tet gradient and Hessian of each vertex
// from Buffers::incident (valid for a Jacobi source pose) instead of
// gathering them.
int launchSolve(const Buffers& b, const DevParams* p, const float4* src, float4* tgt, const uint32_t* list,
                uint32_t count, uint32_t K, bool cachedIncident, cudaStream_t s);
// The graph-coloured sweep of one iteration as one cooperative persistent
// kernel (per colour: the frames it reads, a grid barrier, its in-place
// solves, a grid barrier), after a memset of the barrier words.  Barriers
// give up after spinLimit polls and set the word the host checks.  Returns
// the kernels launched (memset and sweep), or -1 when the largest colour
// needs more than one wave of resident blocks or the device cannot run the
// grid cooperatively (the caller then launches colour by colour).
int launchColoredSweep(const Buffers& b, const DevParams* p, float4* x, const uint32_t* colorVertices,
                       const uint32_t* colorOffsets, const uint32_t* needVertices, const uint32_t* needOffsets,
                       uint32_t colorCount, uint32_t V, uint32_t K, uint32_t largestColor, uint32_t largestNeed,
                       bool refreshAllFrames, void* barrier, uint32_t spinLimit, cudaStream_t s);
// Bytes of the sweep's barrier words (arrived, generation, error word).
size_t sweepBarrierBytes();
// Co-rotated path: tet frames and the regularised per-vertex solve.
int launchTetPolar(const Buffers& b, const DevParams* p, const float4* src, uint32_t T, cudaStream_t s);
int launchCorotatedSolve(const Buffers& b, const DevParams* p, const float4* src, float4* tgt, const uint32_t* list,
                         uint32_t count, uint32_t K, cudaStream_t s);
int launchCopy(const Buffers& b, const DevParams* p, const float4* src, float4* dst, uint32_t V, cudaStream_t s);
int launchGate(const Buffers& b, const DevParams* p, const float4* src, const float4* tgt, cudaStream_t s);
int launchConvergence(const Buffers& b, const DevParams* p, const float4* src, float4* tgt,
                      bool computeNextRotations, cudaStream_t s);
// IPC contact passes (jgs2-shader.ts:2694-2917): lagContact at the frame
// start; per iteration the active rows before the solve, then the safe-step
// pass, its application, the validation of the scaled pose, its application
// (a failure restores the source), and after the convergence pass the
// promotion of the accepted target contacts.  Each launcher returns the
// number of kernels launched (0 without candidates).
int launchContactLag(const Buffers& b, const DevParams* p, cudaStream_t s);
int launchContactRows(const Buffers& b, const DevParams* p, const float4* src, uint32_t V, cudaStream_t s);
int launchContactStep(const Buffers& b, const DevParams* p, const float4* src, const float4* tgt, cudaStream_t s);
int launchContactApply(const Buffers& b, const DevParams* p, const float4* src, float4* tgt, uint32_t V,
                       bool validated, cudaStream_t s);
int launchContactValidate(const Buffers& b, const DevParams* p, const float4* tgt, cudaStream_t s);
int launchContactPromote(const Buffers& b, const DevParams* p, cudaStream_t s);
// The device broad phase of one iteration (contact surfaces): primitive and
// chunk boxes, row counts, their scan, the rows' candidates with their
// carried or fresh state and activity, and the per-vertex active rows (a
// stable sort of the active candidates' vertex entries).  `first`: the
// frame's first iteration, which also lags the contacts.
int launchBroadPhase(const Buffers& b, const DevParams* p, const float4* src, uint32_t V, bool first,
                     cudaStream_t s);
// Sort passes of launchBroadPhase for `V` vertex keys (the sentinel included).
uint32_t broadPhaseSortPasses(uint32_t V);
// The IPC component of the convergence gradient at the accepted pose, before
// the convergence pass.
int launchContactGradient(const Buffers& b, const DevParams* p, const float4* src, const float4* tgt, uint32_t V,
                          cudaStream_t s);
// Closest features of n caller pairs (12 floats each: four points) by the
// step's device contact routine: 9 floats per pair out and the FP64 flag.
int launchContactFeatures(const float* points, const uint32_t* types, uint32_t n, float* out, uint32_t* wide,
                          cudaStream_t s);
// bodyCorrection: some scene of the batch corrects its bodies this frame.
int launchEpilogue(const Buffers& b, const DevParams* p, const float4* finalPos, uint32_t V, bool bodyCorrection,
                   uint32_t bodies, cudaStream_t s);

// Exact all-element oracle diagnostics of one scene (an opt-in diagnostic,
// not part of the step): at the canonical pose against the last inertial
// target and settings.  invDt2 = 1 / h^2; objectiveFlags bit0 forces, bit1
// targets; corotated selects the co-rotated element energy.
struct OracleParams {
  float invDt2, floorHeight, floorStiffness, rotationEpsilon;
  uint32_t objectiveFlags, vOff, V, tOff, T, corotated, pad[2];
};
// Summary sums (doubles): energies (inertia, elasticity, external force,
// target, floor), squared gradient norms (total, inertia, elasticity,
// external force, target, floor), largest active update, smallest
// determinant, smallest active floor distance, active vertices, active floor
// contacts, all active updates valid, all finite.
constexpr int kOracleSummaryWords = 18;
// Tet records: 3 float4 frame columns + (energy, det, finite, 0); vertex
// records: 9 float4 (gradient + active, Hessian rows with energies, metrics).
int launchOracleDiagnostics(const Buffers& b, const OracleParams& q, float4* tetRot, float4* tetMetric,
                            float4* vertexRecords, double* summary, cudaStream_t s);

// Checked builds (JGS2_BOUNDS_CHECKS=1): the first device index check that
// failed since the last call (a site number, 0 = none); the failing access
// was skipped.  Reading resets it.  Always 0 in a build without checks.
cudaError_t takeBoundsViolation(uint32_t* site);
bool boundsChecked();
// Vertices per solve block for cubature width K (0: K too large to cache).
uint32_t solveGroupsPerBlock(uint32_t K);
// Whether the solve caches records of width K in shared memory (else it
// recomputes them in the line search).
bool solveCachesRecords(uint32_t K);
// Dynamic shared memory available to one solve block.
uint32_t solveSharedBytes();
constexpr size_t kGatePartialBytes = 32;
constexpr size_t kConvPartialBytes = 80;

// Allocation-free gate: static device scratch of a 256-byte header (the block
// ticket) and one partial per block, for at most kGateScratchMaxBlocks blocks
// of one element per thread (gateScratchMaxElements() = max(V, T) limit).
constexpr uint32_t kGateScratchMaxBlocks = 8192;
constexpr size_t kGateScratchHeaderBytes = 256;
constexpr size_t kGateScratchBytes = kGateScratchHeaderBytes + kGateScratchMaxBlocks * kGatePartialBytes;
cudaError_t gateScratchAddress(void** out);
uint32_t gateScratchMaxElements();
// Launches the gate over caller device arrays with `scratch` (the address of
// the static array on the current device); writes 4 float4 to `control`.
// C / H: cloth triangles and hinges.  Returns 0 without launching when
// max(V, T, C, H) is 0 or over the limit.
int launchGateScratch(const Buffers& b, const DevParams& p, const float4* predicted, const float4* src,
                      const float4* tgt, uint32_t V, uint32_t T, uint32_t C, uint32_t H, float4* control,
                      void* scratch, cudaStream_t s);

}  // namespace jgs2
