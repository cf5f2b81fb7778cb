// ww3-gpu_b200/csrc/step.hpp
// Recording of a whole time step on a grid's resident VA (abi_step.cpp): while grid igrid
// records (ww_step_begin .. ww_step_end), its _va entries validate their arguments and copy their
// inputs to device buffers the recording owns, then append their launches here instead of
// running them; ww_step_end captures the launches in one CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <memory>

namespace wwb {

struct StepRecorder;

/// The recorder of grid igrid while it records, else null (the grid's calls run at once).
StepRecorder* step_recorder(int igrid);

/// Keeps obj (the device buffers of a recorded call) alive as long as the recorded step.
void step_keep(StepRecorder* r, std::shared_ptr<void> obj);

/// Appends a recorded call's launches: kernels, memsets and device-to-device work only, no
/// host synchronisation, allocation or host memory, so that a stream capture can record them.
/// A W3SRCE batch also passes its launch as a job (a SrceJob with its layout), so that the
/// batches of several grids' steps can be merged into one launch (ww_steps_fuse).
void step_add(StepRecorder* r, std::function<void(cudaStream_t)> op,
              std::shared_ptr<void> srce_job = nullptr);

/// The stream a recorded call stages its inputs on (synchronise it before returning).
cudaStream_t step_stream(StepRecorder* r);

/// Frees every recorded step (ww_kokkos_finalize).
void release_steps();

/// Frees a device table of a grid's configuration (DIA, ST4, W3SRCE arrays) that a new
/// registration replaces: at once when no recorded step exists, else when the last recorded step
/// is freed, since a recorded step keeps the table addresses it was recorded with.
void free_table(void* p);

}  // namespace wwb
