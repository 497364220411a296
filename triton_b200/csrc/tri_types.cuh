// tri_types.cuh -- device-resident structures shared by the host code and
// the step kernels.
#pragma once

#include <stdint.h>

#include "tri_common.cuh"

namespace tri {

// Volume accounting terms of the FP32 form: inflow through boundary faces,
// point sources, runoff, external-boundary depth resets, negative-depth clipping.
constexpr int kAccTerms = 5;
enum { kAccBoundary = 0, kAccSources = 1, kAccRunoff = 2, kAccExtbc = 3, kAccClip = 4 };

// Device-resident loop state.  Host mirror: tri_clock plus the bookkeeping
// fields below.
struct DevClock {
  double simtime, sim_duration, print_interval, print_observation, last_obs_time;
  double init_dt, time_step, average_dt, global_dt;
  double t_step;  // simtime at the start of the running step
  double rdt;     // RN(1/global_dt)
  int32_t print_id, it_count, it_print, time_series, time_increment_fixed;
  int32_t runoff_row, src_idx_low, src_idx_high;
  int32_t active, halt, events, steps;
  int32_t cur, src, dst, rd, wr;  // ping-pong state buffers and dt slots
  int32_t nroff, roff_rows, nsrc, hyg_rows;
  int32_t status;  // nonzero: a device-side check failed (value = reason)
  uint32_t tile_next;  // work counter of the flux kernel's dynamic tiles, reset every step
  uint32_t pad0;
  unsigned long long dt_key[2];
  const double* roff_t;
  const double* hyg_t;
  // FP32 form: FP64 volume accounting in depth units (multiply by dx^2).
  // acc_step collects the running step (atomics), the wet-dry kernel folds it
  // into the Kahan-compensated totals acc_sum/acc_comp.
  double acc_step[kAccTerms];
  double acc_sum[kAccTerms];
  double acc_comp[kAccTerms];
};

template <typename T>
struct StateBufs {
  T* h[2];
  T* qx[2];
  T* qy[2];
};

}  // namespace tri
