// tri_step_launch.h -- host side of the step kernels: what one domain's
// step needs (device pointers and sizes) and the launch functions.  The
// kernels are instantiated in two translation units: tri_step_f64.cu (IEEE,
// no contraction: bit-exact with the reference) and tri_step_f32.cu (FP32
// precision form, contraction and fast division/sqrt allowed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tri_types.cuh"

namespace tri {

constexpr int kStripCols = 30;   // interior columns per warp tile of the flux kernel
constexpr int kFluxVariants = 5; // register budgets (FluxBudget)
constexpr int kWetCols = 128;    // columns per block of the wet-dry/dt kernel
constexpr int kWetBand = 16;     // rows per block of the initial-dt kernel
// Blocks of 128 threads per SM that the flux kernel's register-budget
// variants are compiled for (__launch_bounds__ minimum).  FP64: 122, 96, 80,
// 72 and 64 registers a thread (from 96 down they spill to L1, 8 to 300
// bytes); FP32: 88, 80, 64, 48 and 40.  The kernel is latency bound, so
// occupancy can pay for some spilling; the autotuner picks per domain.
template <typename T>
struct FluxBudget;
template <>
struct FluxBudget<double> {
  static constexpr int v0 = 4, v1 = 5, v2 = 6, v3 = 7, v4 = 8;
};
template <>
struct FluxBudget<float> {
  static constexpr int v0 = 5, v1 = 6, v2 = 8, v3 = 10, v4 = 12;
};
// the variant untuned domains and batches start from
constexpr int kFluxDefaultVariant = 1;
// rows per block of the staged wet-dry/dt kernel (its shared-memory tile),
// and output rows per group of its copies (each group on its own mbarrier)
template <typename T>
constexpr int kStageBand = sizeof(T) == 8 ? 4 : 8;
template <typename T>
constexpr int kStageGroupRows = 2;

struct StepArgs {
  DevClock* clk;
  void* h[2];
  void* qx[2];
  void* qy[2];
  void* z;             // FP64 form: DEM; FP32 form: offsets from the tile bases
  const double* zbase; // FP32 form: FP64 base level per 32x32 tile
  int ntc;             // tiles per row
  void* n2;
  void* maxh;
  const int32_t* zone;
  const void* rates;
  int rows, cols;
  int rb, flux_blocks, flux_variant;
  double dx, courant, hextra;
  int open_boundaries;
  int nsrc;
  const int32_t* src_cells;
  const int32_t* src_order;
  const double* hyg_t;
  const void* hyg_v;
  const int32_t* src_waves;  // host array, n_src_waves + 1 offsets
  int n_src_waves;
  int nbc;
  const int32_t *bc_cells, *bc_types, *bc_start, *bc_nrows, *bc_order;
  const void *bc_v1, *bc_v2;
  const int32_t* bc_waves;  // host array, n_bc_waves + 1 offsets
  int n_bc_waves;
  float* arrival;
  float arrival_depth;
  // dry-tile flags of the flux kernel ([2][tiles] by buffer + [tiles]
  // pinned), or null to compute every tile; the same for the wet-dry kernel
  // (null also while the arrival depth is negative), which skips bands only
  // while *maxh_neg (an uploaded max depth is negative) is 0
  uint8_t* tzero;
  const uint8_t* tzero_wet;
  const int32_t* maxh_neg;
};

// One time step (clock, flux/update, sources, open ghosts, boundary cells,
// wet-dry/dt).  ev: optional 4 events around the flux and wet-dry launches.
template <typename T>
int launch_step(const StepArgs& a, cudaStream_t s, cudaEvent_t* ev);
// CFL dt of the current state into the slot the next step reads.
template <typename T>
int launch_initial_dt(const StepArgs& a, cudaStream_t s);
template <typename T>
void flux_occupancy(int variant, int* per_sm);

// A batch of member domains advanced together (one step of each member per
// batched step).  Device pointers; wave offsets are host arrays.
struct BatchArgs {
  const void* mem;  // MemberDev<T>[nm] in device memory
  int nm;
  const int32_t* tile_member;  // member of every flux tile
  const int32_t* wet_member;   // member of every wet-dry block
  BatchCtl* ctl;
  uint32_t ntiles, nwet_blocks;
  int flux_blocks, flux_variant;
  const int2* src_items;
  const int32_t* src_waves;
  int n_src_waves;
  const int2* bc_items;
  const int32_t* bc_waves;
  int n_bc_waves;
  const int32_t* open_members;  // members with open edges (device), their count and largest max(rows, cols)
  int n_open, open_dim;
};
template <typename T>
int launch_batch_step(const BatchArgs& a, cudaStream_t s);
// Single-launch mode: nsteps batched steps in one launch of k_batch_steps
// (the control block's ticket and status and the progress counters must be
// zero); grid: the blocks resident at once (batch_steps_grid).  Register
// budget: variant 0 or (any other) 1 of FluxBudget.
template <typename T>
int launch_batch_steps(const BatchArgs& a, MemberProgress* prog, int nsteps, int grid, cudaStream_t s);
template <typename T>
int batch_steps_grid(int variant);
template <typename T>
void batch_flux_occupancy(int variant, int* per_sm);

// Kernel attributes (shared-memory sizes) on the current device; call before
// the first launch on a device.
template <typename T>
int prepare_kernels();

extern template int prepare_kernels<double>();
extern template int prepare_kernels<float>();
extern template int launch_step<double>(const StepArgs&, cudaStream_t, cudaEvent_t*);
extern template int launch_step<float>(const StepArgs&, cudaStream_t, cudaEvent_t*);
extern template int launch_initial_dt<double>(const StepArgs&, cudaStream_t);
extern template int launch_initial_dt<float>(const StepArgs&, cudaStream_t);
extern template void flux_occupancy<double>(int, int*);
extern template void flux_occupancy<float>(int, int*);
extern template int launch_batch_step<double>(const BatchArgs&, cudaStream_t);
extern template int launch_batch_step<float>(const BatchArgs&, cudaStream_t);
extern template int launch_batch_steps<double>(const BatchArgs&, MemberProgress*, int, int, cudaStream_t);
extern template int launch_batch_steps<float>(const BatchArgs&, MemberProgress*, int, int, cudaStream_t);
extern template int batch_steps_grid<double>(int);
extern template int batch_steps_grid<float>(int);
extern template void batch_flux_occupancy<double>(int, int*);
extern template void batch_flux_occupancy<float>(int, int*);

}  // namespace tri
