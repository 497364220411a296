// tri_domain_impl.h -- the domain object behind the C ABI handle, shared by
// the domain and batch translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "tri_step_launch.h"
#include "tri_types.cuh"
#include "triton_b200.h"

using tri::DevClock;

struct tri_domain {
  tri_grid_desc desc{};
  int prec = TRI_FP64;
  size_t esize = 8;
  int64_t ncells = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // state (ping-pong) and static fields; element type double or float
  void* h[2] = {nullptr, nullptr};
  void* qx[2] = {nullptr, nullptr};
  void* qy[2] = {nullptr, nullptr};
  void* z = nullptr;
  void* n2 = nullptr;
  void* maxh = nullptr;
  double* stage = nullptr;  // FP64 staging field for FP32 uploads/downloads
  double* zbase = nullptr;  // FP32 form: FP64 bed base level per 32x32 tile
  int ntc = 0, ntr = 0;     // tiles per row / per column
  float* arrival = nullptr; // optional first time h exceeds arrival_depth
  float arrival_depth = 0.1f;
  // runoff
  int32_t nroff = 0, roff_rows = 0;
  int32_t* zone = nullptr;
  void* rates = nullptr;
  double* roff_t = nullptr;
  // sources
  int32_t nsrc = 0, hyg_rows = 0;
  int32_t* src_cells = nullptr;
  int32_t* src_order = nullptr;
  std::vector<int32_t> src_waves, src_order_host, src_cells_host;
  double* hyg_t = nullptr;
  void* hyg_v = nullptr;
  // external boundary cells
  int32_t nbc = 0;
  int32_t *bc_cells = nullptr, *bc_types = nullptr, *bc_start = nullptr, *bc_nrows = nullptr, *bc_order = nullptr;
  std::vector<int32_t> bc_waves, bc_order_host, bc_cells_host;
  void *bc_v1 = nullptr, *bc_v2 = nullptr;
  // observations
  int32_t nobs = 0;
  int32_t* obs_cells = nullptr;
  double* obs_out = nullptr;
  double* obs_host = nullptr;
  // clock
  DevClock* clk = nullptr;  // device
  DevClock* mirror = nullptr;  // pinned host mirror
  int32_t* halt_host = nullptr;  // pinned, one per chunk slot
  bool dt_valid = false;
  // volume reduction scratch
  double* vol_part = nullptr;
  double* vol_out = nullptr;
  int vol_blocks = 0;
  // launch shape of the flux kernel (tile height, register variant, grid)
  int rb = 16, flux_blocks = 1, flux_variant = 1;
  // dry-tile flags of the flux kernel for the current tile shape: [2][tiles]
  // (tile holds only +0 in buffer 0 / 1) then [tiles] pinned.  Any change of
  // state, forcing or shape outside the step kernels marks them dirty; they
  // are reset (nothing known zero) before the next steps.
  uint8_t* tzero = nullptr;
  int64_t tz_cap = 0, tz_tiles = 0;
  bool tz_on = false, tz_dirty = true;
  int32_t* maxh_neg = nullptr;  // device flag: an uploaded max depth is negative (or NaN)
  int64_t work_steps = 0;       // steps advance() ran since tri_domain_set_timing
  std::vector<uint8_t> tz_pin_host;
  double tuned_ms = 0;
  // graphs of 'graph_steps' steps
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  bool use_graphs = true;
  // timing: CUDA event pairs around every flux and wet-dry launch, read once
  // the timed region is over so the stream is never stalled
  bool timing = false;
  std::vector<cudaEvent_t> tev;
  size_t tev_used = 0;
  cudaEvent_t chunk_ev[2] = {nullptr, nullptr};
};


namespace tri {
// helpers implemented in tri_domain.cu
int domain_push_clock(tri_domain* d);
int domain_pull_clock(tri_domain* d);
int domain_launch_dt(tri_domain* d);
StepArgs domain_step_args(tri_domain* d);
}  // namespace tri
