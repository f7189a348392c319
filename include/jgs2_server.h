/*
 * jgs2_server.h — continuous-batching request loop over the JGS2 step.
 *
 * The reference steps one scene per JGS2GpuSolver from a browser frame loop
 * and has no serving layer; this is the served form that stands beside the
 * plain per-scene path of jgs2.h.  Requests ("step this scene N frames") are
 * admitted against a device-memory budget and grouped into waves; a wave runs
 * as one batch (jgs2_batch_*).  Every wave in flight advances one frame per
 * round on its own CUDA stream, so waves overlap on the device.  A request
 * that has run its frames is read back and retired at once while its wave
 * keeps stepping the others; its memory returns to the budget when the whole
 * wave has finished.  Waves are built (validation, packing, upload) on a
 * separate thread, so requests that arrive while waves are running are
 * admitted and prepared without stalling the rounds in flight.
 *
 * Results equal what the same scene gives alone through jgs2.h: a batch keeps
 * each scene's gate, convergence and latch to itself.
 */
#ifndef JGS2_SERVER_H_
#define JGS2_SERVER_H_

#include "jgs2.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct jgs2_server jgs2_server;

typedef struct jgs2_server_options {
  int device;
  uint64_t memory_budget_bytes;  /* resident scenes may not exceed this (estimate) */
  uint32_t max_scenes_per_wave;  /* 0: no limit */
  uint32_t max_waves;            /* waves in flight or being built at once; 0: no limit */
} jgs2_server_options;

typedef struct jgs2_request_result {
  uint64_t id;
  jgs2_status status;
  uint32_t frames;           /* frames run */
  uint32_t vertex_count;
  uint32_t wave_scenes;      /* scenes in the wave this request ran in */
  double submit_seconds;     /* server clock: submitted, first frame launched, finished */
  double admit_seconds;
  double finish_seconds;
  double mean_frame_ms;      /* mean round time of the frames this request ran */
  double max_frame_ms;
} jgs2_request_result;

typedef struct jgs2_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t waves_created, rounds;
  uint64_t resident_bytes, peak_resident_bytes;
  uint32_t waves_in_flight, queued;
  double busy_seconds;       /* wall time of the rounds (some wave in flight) */
} jgs2_server_stats;

jgs2_status jgs2_server_create(const jgs2_server_options* options, jgs2_server** out);
/* Stops the loop after the round in flight; pending requests complete with
 * JGS2_DESTROYED. */
void jgs2_server_destroy(jgs2_server* server);
const char* jgs2_server_last_error(const jgs2_server* server);

/* Queue a request: step `input` (copied) `frames` frames.  exact_iterations >
 * 0 runs exactly that many iterations per frame, 0 the production step.
 * Requests that need more memory than the whole budget fail at once. */
jgs2_status jgs2_server_submit(jgs2_server* server, const jgs2_input* input, const jgs2_settings* settings,
                               uint32_t settings_mask, uint32_t frames, uint32_t exact_iterations,
                               uint64_t* request_id);

/* Block until the request has finished; copy its final positions and
 * velocities (4 floats per vertex each; either may be NULL) and its result
 * record.  A request can be waited for once. */
jgs2_status jgs2_server_wait(jgs2_server* server, uint64_t request_id, float* positions, size_t position_floats,
                             float* velocities, size_t velocity_floats, jgs2_request_result* result);

/* Block until every submitted request has finished (results stay waitable). */
jgs2_status jgs2_server_drain(jgs2_server* server);
jgs2_status jgs2_server_get_stats(jgs2_server* server, jgs2_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* JGS2_SERVER_H_ */
