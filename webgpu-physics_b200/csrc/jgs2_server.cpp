// Continuous-batching request loop (include/jgs2_server.h).
//
// Two threads.  The builder admits queued requests against the memory budget
// into a wave and builds its batch (validation, packing, upload, preflight);
// the stepper launches frames of every wave in flight per round (each wave
// on its own stream, so they overlap), waits for them, and retires requests
// that have run their frames.  The request table, the queue, the ready list
// and the statistics are guarded by one mutex; a wave belongs to the builder
// until it is on the ready list and to the stepper afterwards.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "jgs2.h"
#include "jgs2_server.h"

namespace {

using Clock = std::chrono::steady_clock;

// A deep copy of a jgs2_input: the caller's arrays may go away after submit.
struct OwnedInput {
  jgs2_input view{};
  std::vector<float> positions, velocities, rest, colors, forces, targets, stiff, invDm, meta, restStiffness;
  std::vector<float> cubW, cubBasis;
  std::vector<uint32_t> info, tets, adjacency, cubTet;
  jgs2_cloth_input cloth{};
  std::vector<uint32_t> clothTris, hinges, contacts, surfaceTris;
  jgs2_contact_surface surface{};
  std::vector<float> clothInv, clothAreas, hingeAngles, hingeLengths;

  template <class T>
  static const T* take(std::vector<T>& dst, const T* src, size_t n) {
    if (!src) return nullptr;
    dst.assign(src, src + n);
    return dst.data();
  }

  explicit OwnedInput(const jgs2_input& in) {
    const size_t V = in.vertex_count, T = in.tet_count, K = in.cubature_k;
    view = in;
    view.positions = take(positions, in.positions, 4 * V);
    view.velocities = take(velocities, in.velocities, 4 * V);
    view.vertex_rest = take(rest, in.vertex_rest, 4 * V);
    view.vertex_colors = take(colors, in.vertex_colors, 4 * V);
    view.vertex_info = take(info, in.vertex_info, 4 * V);
    view.external_forces = take(forces, in.external_forces, 3 * V);
    view.target_positions = take(targets, in.target_positions, 3 * V);
    view.target_stiffnesses = take(stiff, in.target_stiffnesses, V);
    view.tet_indices = take(tets, in.tet_indices, 4 * T);
    view.tet_inverse_dm = take(invDm, in.tet_inverse_dm, 12 * T);
    view.tet_meta = take(meta, in.tet_meta, 4 * T);
    view.tet_rest_stiffness = take(restStiffness, in.tet_rest_stiffness, 144 * T);
    view.adjacency = take(adjacency, in.adjacency, in.adjacency_length);
    view.cubature_tet_ids = take(cubTet, in.cubature_tet_ids, V * K);
    view.cubature_weights = take(cubW, in.cubature_weights, V * K);
    view.cubature_basis = take(cubBasis, in.cubature_basis, 36 * V * K);
    if (in.cloth) {
      const jgs2_cloth_input& c = *in.cloth;
      const size_t C = c.triangle_count, H = c.hinge_count;
      cloth = c;
      cloth.triangle_indices = take(clothTris, c.triangle_indices, 3 * C);
      cloth.triangle_inverse_rest_bases = take(clothInv, c.triangle_inverse_rest_bases, 4 * C);
      cloth.triangle_rest_areas = take(clothAreas, c.triangle_rest_areas, C);
      cloth.hinge_indices = take(hinges, c.hinge_indices, 4 * H);
      cloth.hinge_rest_angles = take(hingeAngles, c.hinge_rest_angles, H);
      cloth.hinge_rest_edge_lengths = take(hingeLengths, c.hinge_rest_edge_lengths, H);
      view.cloth = &cloth;
    }
    view.contact_indices = take(contacts, in.contact_indices,
                                4 * (size_t(in.contact_vertex_triangle_count) + in.contact_edge_edge_count));
    if (in.contact_surface) {
      surface = *in.contact_surface;
      surface.triangles = take(surfaceTris, surface.triangles, 3 * size_t(surface.triangle_count));
      view.contact_surface = &surface;
    }
  }
};

struct Request {
  uint64_t id = 0;
  std::unique_ptr<OwnedInput> input;
  jgs2_settings settings{};
  uint32_t mask = 0;
  uint32_t frames = 0, exactIterations = 0;
  uint32_t schedule = 0, iterationsPerFrame = 0;  // the wave key
  uint64_t bytes = 0;
  double submitT = 0, admitT = 0, finishT = 0;
  uint32_t framesDone = 0, waveScenes = 0;
  double sumFrameMs = 0, maxFrameMs = 0;
  std::vector<float> positions, velocities;
  jgs2_status status = JGS2_OK;
  std::string error;
  bool done = false;
};

struct Wave {
  jgs2_batch* batch = nullptr;
  std::vector<Request*> requests;  // scene i = requests[i]
  std::vector<bool> active;
  uint32_t exactIterations = 0;
  uint64_t bytes = 0;
  uint32_t remaining = 0;
  uint32_t roundFrames = 1;  // frames stepped in the current round
  bool started = false;
};

// Frames a wave may step in one round of the stepper.
constexpr uint32_t kRoundFrames = 16;

uint32_t normalizeOdd(uint32_t it) {
  const uint32_t i = it < 1 ? 1 : it;
  return i % 2 == 0 ? i + 1 : i;
}

}  // namespace

struct jgs2_server {
  jgs2_server_options options{};
  std::mutex mutex;
  std::condition_variable builderCv, stepperCv, doneCv;
  std::deque<Request*> queue;
  std::map<uint64_t, std::unique_ptr<Request>> requests;
  std::vector<std::unique_ptr<Wave>> ready;  // built, not yet stepping
  uint32_t wavesOpen = 0;                     // being built, ready or in flight
  uint64_t nextId = 1;
  bool stop = false;
  std::string error;
  Clock::time_point start = Clock::now();
  jgs2_server_stats stats{};
  std::thread builder, stepper;

  double now() const { return std::chrono::duration<double>(Clock::now() - start).count(); }

  // Caller holds the mutex.
  void finishLocked(Request* r, jgs2_status st, const std::string& message) {
    r->status = st;
    r->error = message;
    r->finishT = now();
    r->done = true;
    if (st == JGS2_OK) stats.completed++;
    else stats.failed++;
    doneCv.notify_all();
  }

  void finish(Request* r, jgs2_status st, const std::string& message) {
    std::lock_guard<std::mutex> lock(mutex);
    finishLocked(r, st, message);
  }

  // Caller holds the mutex.  Takes queued requests that share the head's
  // schedule and iteration count while they fit the memory budget (strict
  // FIFO: the head is never passed over).
  std::vector<Request*> admitLocked() {
    std::vector<Request*> taken;
    if (queue.empty()) return taken;
    if (options.max_waves && wavesOpen >= options.max_waves) return taken;
    const Request* head = queue.front();
    for (auto it = queue.begin(); it != queue.end();) {
      Request* r = *it;
      if (options.max_scenes_per_wave && taken.size() >= options.max_scenes_per_wave) break;
      const bool sameKey = r->schedule == head->schedule && r->iterationsPerFrame == head->iterationsPerFrame &&
                           (r->exactIterations == 0) == (head->exactIterations == 0);
      if (!sameKey) { ++it; continue; }
      if (stats.resident_bytes + r->bytes > options.memory_budget_bytes) break;
      stats.resident_bytes += r->bytes;
      if (stats.resident_bytes > stats.peak_resident_bytes) stats.peak_resident_bytes = stats.resident_bytes;
      taken.push_back(r);
      it = queue.erase(it);
    }
    if (!taken.empty()) wavesOpen++;
    stats.queued = static_cast<uint32_t>(queue.size());
    return taken;
  }

  void buildLoop() {
    cudaSetDevice(options.device);
    for (;;) {
      std::vector<Request*> taken;
      {
        std::unique_lock<std::mutex> lock(mutex);
        builderCv.wait(lock, [&] {
          if (stop) return true;
          taken = admitLocked();
          return !taken.empty();
        });
        if (stop) {
          if (!taken.empty()) {
            for (Request* r : taken) {
              stats.resident_bytes -= r->bytes;
              finishLocked(r, JGS2_DESTROYED, "The server was destroyed.");
            }
            wavesOpen--;
          }
          return;
        }
      }
      auto w = std::make_unique<Wave>();
      std::vector<const jgs2_input*> inputs;
      std::vector<jgs2_settings> settings;
      std::vector<uint32_t> masks;
      for (Request* r : taken) {
        inputs.push_back(&r->input->view);
        settings.push_back(r->settings);
        masks.push_back(r->mask);
        w->bytes += r->bytes;
      }
      const jgs2_status st = jgs2_batch_create(inputs.data(), static_cast<uint32_t>(inputs.size()),
                                               settings.data(), masks.data(), options.device, &w->batch);
      std::lock_guard<std::mutex> lock(mutex);
      if (st != JGS2_OK) {
        const std::string msg = jgs2_global_last_error();
        stats.resident_bytes -= w->bytes;
        wavesOpen--;
        for (Request* r : taken) finishLocked(r, st, msg);
        builderCv.notify_all();
        continue;
      }
      for (Request* r : taken) r->waveScenes = static_cast<uint32_t>(taken.size());
      w->requests = taken;
      w->active.assign(taken.size(), true);
      w->remaining = static_cast<uint32_t>(taken.size());
      w->exactIterations = taken[0]->exactIterations;
      stats.waves_created++;
      ready.push_back(std::move(w));
      stepperCv.notify_all();
    }
  }

  // Fails every request still active in a wave.
  void failWave(Wave& w, jgs2_status st) {
    const std::string msg = jgs2_batch_last_error(w.batch);
    for (size_t i = 0; i < w.requests.size(); ++i)
      if (w.active[i]) finish(w.requests[i], st, msg);
    w.remaining = 0;
  }

  void stepLoop() {
    cudaSetDevice(options.device);
    std::vector<std::unique_ptr<Wave>> waves;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(mutex);
        if (waves.empty()) stepperCv.wait(lock, [&] { return stop || !ready.empty(); });
        if (stop) break;
        for (auto& w : ready) waves.push_back(std::move(w));
        ready.clear();
        stats.waves_in_flight = static_cast<uint32_t>(waves.size());
      }
      // One round: every wave in flight steps as many frames as its nearest
      // request still needs (at most kRoundFrames), launched together, so a
      // round's host synchronisation is shared by several frames.
      const auto t0 = Clock::now();
      const double t0s = now();
      for (auto& w : waves) {
        if (!w->started) {
          w->started = true;
          for (Request* r : w->requests) r->admitT = t0s;
        }
        uint32_t n = kRoundFrames;
        for (size_t i = 0; i < w->requests.size(); ++i)
          if (w->active[i]) n = std::min(n, w->requests[i]->frames - w->requests[i]->framesDone);
        w->roundFrames = std::max(1u, n);
        const jgs2_status st =
            jgs2_batch_step_frames(w->batch, w->roundFrames, w->exactIterations, nullptr, nullptr);
        if (st != JGS2_OK) failWave(*w, st);
      }
      for (auto& w : waves) {
        if (w->remaining == 0) continue;
        const jgs2_status st = jgs2_batch_sync(w->batch);
        if (st != JGS2_OK) { failWave(*w, st); continue; }
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count() / w->roundFrames;
        for (size_t i = 0; i < w->requests.size(); ++i) {
          if (!w->active[i]) continue;
          Request* r = w->requests[i];
          r->framesDone += w->roundFrames;
          r->sumFrameMs += ms * w->roundFrames;
          if (ms > r->maxFrameMs) r->maxFrameMs = ms;
          if (r->framesDone < r->frames) continue;
          const size_t n = 4ull * r->input->view.vertex_count;
          r->positions.resize(n);
          r->velocities.resize(n);
          const uint32_t scene = static_cast<uint32_t>(i);
          jgs2_status st2 = jgs2_batch_read_positions(w->batch, scene, r->positions.data(), n);
          if (st2 == JGS2_OK) st2 = jgs2_batch_read_velocities(w->batch, scene, r->velocities.data(), n);
          if (st2 == JGS2_OK) st2 = jgs2_batch_set_scene_active(w->batch, scene, 0);
          w->active[i] = false;
          w->remaining--;
          finish(r, st2, st2 == JGS2_OK ? std::string() : std::string(jgs2_batch_last_error(w->batch)));
        }
      }
      const double roundS = std::chrono::duration<double>(Clock::now() - t0).count();
      uint64_t freed = 0;
      uint32_t closed = 0;
      for (auto it = waves.begin(); it != waves.end();) {
        if ((*it)->remaining == 0) {
          jgs2_batch_destroy((*it)->batch);
          freed += (*it)->bytes;
          closed++;
          it = waves.erase(it);
        } else {
          ++it;
        }
      }
      std::lock_guard<std::mutex> lock(mutex);
      stats.rounds++;
      stats.busy_seconds += roundS;
      stats.resident_bytes -= freed;
      wavesOpen -= closed;
      stats.waves_in_flight = static_cast<uint32_t>(waves.size());
      if (freed) builderCv.notify_all();
    }
    std::lock_guard<std::mutex> lock(mutex);
    for (auto& w : ready) waves.push_back(std::move(w));
    ready.clear();
    for (auto& w : waves) {
      for (size_t i = 0; i < w->requests.size(); ++i)
        if (w->active[i]) finishLocked(w->requests[i], JGS2_DESTROYED, "The server was destroyed.");
      jgs2_batch_destroy(w->batch);
    }
  }
};

extern "C" {

jgs2_status jgs2_server_create(const jgs2_server_options* options, jgs2_server** out) {
  if (!options || !out) return JGS2_INVALID_ARGUMENT;
  *out = nullptr;
  if (options->memory_budget_bytes == 0) return JGS2_INVALID_ARGUMENT;
  std::unique_ptr<jgs2_server> s(new jgs2_server());
  s->options = *options;
  jgs2_server* sp = s.get();
  sp->builder = std::thread([sp] { sp->buildLoop(); });
  sp->stepper = std::thread([sp] { sp->stepLoop(); });
  *out = s.release();
  return JGS2_OK;
}

void jgs2_server_destroy(jgs2_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mutex);
    s->stop = true;
    for (Request* r : s->queue) s->finishLocked(r, JGS2_DESTROYED, "The server was destroyed.");
    s->queue.clear();
  }
  s->builderCv.notify_all();
  s->stepperCv.notify_all();
  if (s->builder.joinable()) s->builder.join();
  if (s->stepper.joinable()) s->stepper.join();
  s->doneCv.notify_all();
  delete s;
}

const char* jgs2_server_last_error(const jgs2_server* s) { return s ? s->error.c_str() : ""; }

jgs2_status jgs2_server_submit(jgs2_server* s, const jgs2_input* input, const jgs2_settings* settings,
                               uint32_t mask, uint32_t frames, uint32_t exactIterations, uint64_t* id) {
  if (!s || !input || !id) return JGS2_INVALID_ARGUMENT;
  jgs2_settings resolved;
  jgs2_status st = jgs2_resolve_settings(nullptr, settings, mask, &resolved);
  if (st == JGS2_OK) st = jgs2_validate_input(input);
  if (st != JGS2_OK) {
    std::lock_guard<std::mutex> lock(s->mutex);
    s->error = jgs2_global_last_error();
    return st;
  }
  if (frames < 1) {
    std::lock_guard<std::mutex> lock(s->mutex);
    s->error = "A request must run at least one frame.";
    return JGS2_INVALID_ARGUMENT;
  }
  const uint64_t bytes = jgs2_estimate_device_bytes(input);
  if (bytes > s->options.memory_budget_bytes) {
    std::lock_guard<std::mutex> lock(s->mutex);
    s->error = "The request needs more device memory than the whole serving budget.";
    return JGS2_OUT_OF_MEMORY;
  }
  auto r = std::make_unique<Request>();
  r->input = std::make_unique<OwnedInput>(*input);
  if (settings) r->settings = *settings;
  r->mask = mask;
  r->frames = frames;
  r->exactIterations = exactIterations;
  r->schedule = resolved.schedule;
  r->iterationsPerFrame = exactIterations ? exactIterations : normalizeOdd(resolved.iterations);
  r->bytes = bytes;
  std::lock_guard<std::mutex> lock(s->mutex);
  if (s->stop) return JGS2_DESTROYED;
  r->id = s->nextId++;
  r->submitT = s->now();
  *id = r->id;
  s->queue.push_back(r.get());
  s->requests.emplace(r->id, std::move(r));
  s->stats.submitted++;
  s->stats.queued = static_cast<uint32_t>(s->queue.size());
  s->builderCv.notify_all();
  return JGS2_OK;
}

jgs2_status jgs2_server_wait(jgs2_server* s, uint64_t id, float* positions, size_t positionFloats,
                             float* velocities, size_t velocityFloats, jgs2_request_result* result) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(s->mutex);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) {
    s->error = "Unknown (or already collected) request id.";
    return JGS2_INVALID_ARGUMENT;
  }
  Request* r = it->second.get();
  s->doneCv.wait(lock, [&] { return r->done; });
  if (r->status == JGS2_OK) {
    const size_t n = r->positions.size();
    if ((positions && positionFloats < n) || (velocities && velocityFloats < n)) {
      s->error = "Output arrays need 4 floats per vertex.";
      return JGS2_INVALID_ARGUMENT;
    }
    if (positions) std::memcpy(positions, r->positions.data(), sizeof(float) * n);
    if (velocities) std::memcpy(velocities, r->velocities.data(), sizeof(float) * n);
  }
  if (result) {
    std::memset(result, 0, sizeof(*result));
    result->id = r->id;
    result->status = r->status;
    result->frames = r->framesDone;
    result->vertex_count = r->input->view.vertex_count;
    result->wave_scenes = r->waveScenes;
    result->submit_seconds = r->submitT;
    result->admit_seconds = r->admitT;
    result->finish_seconds = r->finishT;
    result->mean_frame_ms = r->framesDone ? r->sumFrameMs / r->framesDone : 0.0;
    result->max_frame_ms = r->maxFrameMs;
  }
  const jgs2_status st = r->status;
  if (st != JGS2_OK) s->error = r->error;
  s->requests.erase(it);
  return st;
}

jgs2_status jgs2_server_drain(jgs2_server* s) {
  if (!s) return JGS2_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(s->mutex);
  s->doneCv.wait(lock, [&] { return s->stats.completed + s->stats.failed >= s->stats.submitted || s->stop; });
  return JGS2_OK;
}

jgs2_status jgs2_server_get_stats(jgs2_server* s, jgs2_server_stats* out) {
  if (!s || !out) return JGS2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mutex);
  *out = s->stats;
  out->queued = static_cast<uint32_t>(s->queue.size());
  return JGS2_OK;
}

}  // extern "C"
