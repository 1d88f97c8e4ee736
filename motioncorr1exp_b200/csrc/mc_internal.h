// Internal interface between the plan (mc_plan.cu) and the batch runner
// (mc_batch.cpp): the pieces of a device-only movie, so that a batch of
// movies can be captured into one CUDA graph and launched once.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "../../include/mc.h"

namespace mc {

int record_error(int code, const char* text);  // sets mc_last_error()

// Bytes of one movie's pinned result block (per-movie copy of the staging
// the device-only movie writes: DC terms, pair results, ki, kept rows,
// per-step shifts, status).
size_t plan_stage_bytes(const mc_plan* pl);
// True when a movie runs device-only on this plan (-itr 0, no refinement).
bool plan_device_only(const mc_plan* pl);
// Re-targets the plan's host state to a movie (frame range, pair list,
// thresholds) without touching the device.
int plan_reframe_host(mc_plan* pl, const mc_params* p, int nz);
// Pair list of the current frame configuration as (i, j) words.
int plan_pair_words(const mc_plan* pl, int* ij, int cap);
// Enqueues one device-only movie on the plan's stream, which must already
// be part of a stream capture: the pair list and the frame base are copied
// from the pinned words `pairs` and `frame_word` (read when the graph runs),
// then forward transforms, pair stage, FP64 solve, sum and C2R, the result
// copies into the pinned block `stage`, and the image into `image` (pinned
// host or device memory, or null).
int plan_enqueue_movie(mc_plan* pl, const void* const* frame_word, const int* pairs, unsigned char* stage,
                       float* image);
// The plan's stream (the capture joins it through an event).
cudaStream_t plan_stream(const mc_plan* pl);
// After the graph ran: one movie's results from its block into the plan's
// host state (the same log lines as a single run).
int plan_finish_movie(mc_plan* pl, const unsigned char* stage, const void* d_frames);

}  // namespace mc
