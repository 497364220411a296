// tri_types.cuh -- device-resident structures shared by the host code and
// the step kernels.
#pragma once

#include <stdint.h>

#include "tri_common.cuh"

namespace tri {

// Every field allocation has this many bytes past its last element: bulk row
// copies round their end up to a 16-byte boundary and may read into it.
constexpr size_t kFieldPad = 256;

// Volume accounting terms of the FP32 form: inflow through boundary faces,
// point sources, runoff, external-boundary depth resets, negative-depth clipping.
constexpr int kAccTerms = 5;
enum { kAccBoundary = 0, kAccSources = 1, kAccRunoff = 2, kAccExtbc = 3, kAccClip = 4 };

// Slots of the skipped-cell counters in DevClock.
constexpr int kSkipSlots = 32;

// Device-resident loop state.  Host mirror: tri_clock plus the bookkeeping
// fields below.
struct DevClock {
  double simtime, sim_duration, print_interval, print_observation, last_obs_time;
  double init_dt, time_step, average_dt, global_dt;
  double t_step;  // simtime at the start of the running step
  double rdt;     // RN(1/global_dt)
  double cfl_a;   // RN(courant * dx): the CFL dt is cfl_a / (largest wave speed)
  int32_t print_id, it_count, it_print, time_series, time_increment_fixed;
  int32_t runoff_row, src_idx_low, src_idx_high;
  int32_t active, halt, events, steps;
  int32_t cur, src, dst, rd, wr;  // ping-pong state buffers and dt slots
  int32_t nroff, roff_rows, nsrc, hyg_rows;
  int32_t status;  // nonzero: a device-side check failed (value = reason)
  uint32_t tile_next;  // work counter of the flux kernel's dynamic tiles, reset every step
  uint32_t wait_test;  // test hook: nonzero = polls of a wait nothing completes (tri_domain_set_wait_test)
  unsigned long long dt_key[2];
  const double* roff_t;
  const double* hyg_t;
  // FP64 volume accounting in depth units (multiply by dx^2), both forms.
  // acc_step collects the running step (atomics), the wet-dry kernel folds it
  // into the Kahan-compensated totals acc_sum/acc_comp.
  double acc_step[kAccTerms];
  double acc_sum[kAccTerms];
  double acc_comp[kAccTerms];
  // interior cells of the flux tiles [0] and wet-dry bands [1] that dry-tile
  // skipping left out, summed over slots (one address would serialize the
  // atomics of a launch)
  unsigned long long skipped[2][kSkipSlots];
};

template <typename T>
struct StateBufs {
  T* h[2];
  T* qx[2];
  T* qy[2];
  // buffer i (0 or 1) by selection: indexing a kernel parameter's array with a
  // runtime index would copy the whole struct to local memory
  __device__ __forceinline__ T* H(int i) const { return i ? h[1] : h[0]; }
  __device__ __forceinline__ T* QX(int i) const { return i ? qx[1] : qx[0]; }
  __device__ __forceinline__ T* QY(int i) const { return i ? qy[1] : qy[0]; }
};

// The bed.  FP64 form: the DEM itself.  FP32 form: per 32x32 tile an FP64
// base level and per cell an FP32 offset from it; kernels work with bed
// levels relative to a nearby base ('ref'), so the differences that drive the
// flux (bed steps, water level against a neighbour's bed) keep FP32 accuracy
// on terrain hundreds of metres high.
template <typename T>
struct BedMap;
template <>
struct BedMap<double> {
  const double* z;
  const double* base;  // unused
  int ntc;
  __device__ __forceinline__ double ref_of(int, int) const { return 0.0; }
  __device__ __forceinline__ double local(size_t id, int, int, double) const { return z[id]; }
  __device__ __forceinline__ double local_v(double zv, int, int, double) const { return zv; }
  __device__ __forceinline__ double base_at(int, int) const { return 0.0; }
  __device__ __forceinline__ double absolute(size_t id, int, int) const { return z[id]; }
};
template <>
struct BedMap<float> {
  const float* z;      // offset from the tile base
  const double* base;  // FP64 base level of each 32x32 tile
  int ntc;             // tiles per row
  __device__ __forceinline__ double ref_of(int r, int c) const { return base[(r >> 5) * ntc + (c >> 5)]; }
  __device__ __forceinline__ float local(size_t id, int r, int c, double ref) const {
    const double b = base[(r >> 5) * ntc + (c >> 5)];
    return b == ref ? z[id] : z[id] + (float)(b - ref);
  }
  __device__ __forceinline__ double base_at(int r, int c) const { return base[(r >> 5) * ntc + (c >> 5)]; }
  // the same for an offset already read (from shared memory)
  __device__ __forceinline__ float local_v(float zv, int r, int c, double ref) const {
    const double b = base[(r >> 5) * ntc + (c >> 5)];
    return b == ref ? zv : zv + (float)(b - ref);
  }
  __device__ __forceinline__ double absolute(size_t id, int r, int c) const {
    return base[(r >> 5) * ntc + (c >> 5)] + (double)z[id];
  }
};

template <typename T>
struct MemberDev {
  DevClock* clk;
  StateBufs<T> sb;
  BedMap<T> bed;
  const T* n2;
  const int32_t* zone;
  const T* rates;
  T* maxh;
  float* arrival;
  float arrival_depth;
  int rows, cols, rb;
  T dx, rdx, hextra;
  double dxd, courant;
  uint32_t tile_begin, tile_end;  // this member's tiles in the flux queue
  uint32_t wet_begin, wet_nbx;    // first wet-dry block, blocks per band row
  // sparse forcing (device arrays of the member)
  int nsrc;
  const int32_t* src_cells;
  const double* hyg_t;
  const T* hyg_v;
  const int32_t *bc_cells, *bc_types, *bc_start, *bc_nrows;
  const T *bc_v1, *bc_v2;
  // single-launch mode (k_batch_steps): the member's wet-dry block count and
  // its forcing as conflict-free waves of its own items (order: device item
  // indices wave after wave, woff: nw+1 wave offsets), open edges
  uint32_t wet_count;
  const int32_t *src_order, *src_woff, *bc_order, *bc_woff;
  int src_nw, bc_nw, open;
};

struct BatchCtl {
  uint32_t tile_next;  // flux tile queue, reset every batched step
  int32_t halted;      // members that raised an event during this advance call
  uint32_t ticket;     // single-launch mode: next work item, reset by every launch
  int32_t status;      // single-launch mode: nonzero if a bounded wait gave up
  uint32_t wait_test;  // single-launch mode test hook: polls of a wait that never ends (0: off)
};

// Single-launch mode: per member, cumulative counts of finished work items
// within one launch (zeroed before it): clock steps, flux tiles, forcing
// passes, wet-dry blocks.
struct MemberProgress {
  uint32_t clock, flux, forcing, wet;
};

}  // namespace tri
