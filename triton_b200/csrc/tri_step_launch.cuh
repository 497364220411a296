// tri_step_launch.cuh -- definitions of the launch functions declared in
// tri_step_launch.h; included by the two instantiation units only.
#pragma once

#include <algorithm>

#include "tri_internal.h"
#include "tri_step_kernels.cuh"
#include "tri_step_launch.h"

namespace tri {

template <typename T>
BedMap<T> bed_of(const StepArgs& a) {
  BedMap<T> b;
  b.z = (const T*)a.z;
  b.base = a.zbase;
  b.ntc = a.ntc;
  return b;
}

template <typename T>
StateBufs<T> bufs_of(const StepArgs& a) {
  StateBufs<T> s;
  for (int i = 0; i < 2; i++) {
    s.h[i] = (T*)a.h[i];
    s.qx[i] = (T*)a.qx[i];
    s.qy[i] = (T*)a.qy[i];
  }
  return s;
}

// The flux kernel instance of a register-budget variant.
template <typename T, bool SKIP>
auto flux_kernel(int variant) -> decltype(&k_flux_update<T, FluxBudget<T>::v0, SKIP>) {
  switch (variant) {
    case 0: return &k_flux_update<T, FluxBudget<T>::v0, SKIP>;
    case 1: return &k_flux_update<T, FluxBudget<T>::v1, SKIP>;
    case 2: return &k_flux_update<T, FluxBudget<T>::v2, SKIP>;
    case 3: return &k_flux_update<T, FluxBudget<T>::v3, SKIP>;
    default: return &k_flux_update<T, FluxBudget<T>::v4, SKIP>;
  }
}
template <typename T>
auto batch_flux_kernel(int variant) -> decltype(&k_batch_flux<T, FluxBudget<T>::v0>) {
  switch (variant) {
    case 0: return &k_batch_flux<T, FluxBudget<T>::v0>;
    case 1: return &k_batch_flux<T, FluxBudget<T>::v1>;
    case 2: return &k_batch_flux<T, FluxBudget<T>::v2>;
    case 3: return &k_batch_flux<T, FluxBudget<T>::v3>;
    default: return &k_batch_flux<T, FluxBudget<T>::v4>;
  }
}

template <typename T>
void flux_occupancy(int variant, int* per_sm) {
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, flux_kernel<T, false>(variant), 128, 0);
}

// Launches kernel k after the previous work on stream s with programmatic
// stream serialization: its blocks may be scheduled while the previous
// kernel drains; the kernel waits for it (pdl_wait) before touching memory.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

template <typename T>
int launch_step(const StepArgs& a, cudaStream_t s, cudaEvent_t* ev) {
  const int rows = a.rows, cols = a.cols;
  const T dx = (T)a.dx, hx = (T)a.hextra, rdx = (T)(1.0 / a.dx);
  StateBufs<T> sb = bufs_of<T>(a);
  const BedMap<T> bed = bed_of<T>(a);
  TRI_CUDA_TRY(launch_pdl(k_clock, 1, 32, 0, s, a.clk));
  if (ev) cudaEventRecord(ev[0], s);
  if (a.tzero != nullptr)  // dry-tile skipping
    TRI_CUDA_TRY(launch_pdl(flux_kernel<T, true>(a.flux_variant), a.flux_blocks, 128, 0, s, a.clk, sb, bed,
                            (const T*)a.n2, a.zone, (const T*)a.rates, rows, cols, a.rb, dx, rdx, hx, a.tzero));
  else
    TRI_CUDA_TRY(launch_pdl(flux_kernel<T, false>(a.flux_variant), a.flux_blocks, 128, 0, s, a.clk, sb, bed,
                            (const T*)a.n2, a.zone, (const T*)a.rates, rows, cols, a.rb, dx, rdx, hx, a.tzero));
  if (ev) cudaEventRecord(ev[1], s);
  for (int w = 0; a.nsrc > 0 && w < a.n_src_waves; w++) {
    const int off = a.src_waves[w], cnt = a.src_waves[w + 1] - off;
    TRI_CUDA_TRY(launch_pdl(k_sources<T>, (cnt + 127) / 128, 128, 0, s, a.clk, sb, a.src_order + off, cnt, a.nsrc,
                            a.src_cells, a.hyg_t, (const T*)a.hyg_v, dx));
  }
  if (a.open_boundaries) {
    const int n = std::max(rows, cols);
    TRI_CUDA_TRY(launch_pdl(k_open_bc<T>, (n + 255) / 256, 256, 0, s, a.clk, sb, rows, cols));
  }
  for (int w = 0; a.nbc > 0 && w < a.n_bc_waves; w++) {
    const int off = a.bc_waves[w], cnt = a.bc_waves[w + 1] - off;
    TRI_CUDA_TRY(launch_pdl(k_extbc<T>, (cnt + 127) / 128, 128, 0, s, a.clk, sb, bed, (const T*)a.n2,
                            a.bc_order + off, cnt, a.bc_cells, a.bc_types, a.bc_start, a.bc_nrows, (const T*)a.bc_v1,
                            (const T*)a.bc_v2, rows, cols));
  }
  dim3 g2((cols + kWetCols - 1) / kWetCols, (rows + WetStage<T>::kBand - 1) / WetStage<T>::kBand);
  if (ev) cudaEventRecord(ev[2], s);
  TRI_CUDA_TRY(launch_pdl(k_wetdry_staged<T>, g2, kWetCols, WetStage<T>::kBytes, s, a.clk, sb, bed, (T*)a.maxh,
                          rows, cols, hx, a.arrival, a.arrival_depth, a.tzero_wet, a.rb, a.maxh_neg));
  if (ev) cudaEventRecord(ev[3], s);
  TRI_CUDA_TRY(cudaGetLastError());
  return TRI_OK;
}

template <typename T>
int launch_initial_dt(const StepArgs& a, cudaStream_t s) {
  dim3 g2((a.cols + kWetCols - 1) / kWetCols, (a.rows + kWetBand - 1) / kWetBand);
  k_wetdry_dt<T, false><<<g2, kWetCols, 0, s>>>(a.clk, bufs_of<T>(a), bed_of<T>(a), (T*)a.maxh, a.rows, a.cols,
                                                kWetBand, a.dx, a.courant, (T)a.hextra, nullptr, 0.0f);
  TRI_CUDA_TRY(cudaGetLastError());
  return TRI_OK;
}

template <typename T>
void batch_flux_occupancy(int variant, int* per_sm) {
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_flux_kernel<T>(variant), 128, 0);
}

template <typename T>
int launch_batch_step(const BatchArgs& a, cudaStream_t s) {
  const MemberDev<T>* mem = (const MemberDev<T>*)a.mem;
  k_batch_clock<T><<<(a.nm + 127) / 128, 128, 0, s>>>(mem, a.nm, a.ctl);
  batch_flux_kernel<T>(a.flux_variant)<<<a.flux_blocks, 128, 0, s>>>(mem, a.tile_member, a.ctl, a.ntiles);
  for (int w = 0; w < a.n_src_waves; w++) {
    const int off = a.src_waves[w], cnt = a.src_waves[w + 1] - off;
    k_batch_sources<T><<<(cnt + 127) / 128, 128, 0, s>>>(mem, a.src_items + off, cnt);
  }
  if (a.n_open > 0)
    k_batch_open_bc<T><<<dim3((unsigned)((a.open_dim + 255) / 256), (unsigned)a.n_open), 256, 0, s>>>(
        mem, a.open_members);
  for (int w = 0; w < a.n_bc_waves; w++) {
    const int off = a.bc_waves[w], cnt = a.bc_waves[w + 1] - off;
    k_batch_extbc<T><<<(cnt + 127) / 128, 128, 0, s>>>(mem, a.bc_items + off, cnt);
  }
  k_batch_wetdry<T><<<a.nwet_blocks, kWetCols, WetStage<T>::kBytes, s>>>(mem, a.wet_member);
  TRI_CUDA_TRY(cudaGetLastError());
  return TRI_OK;
}

// Single-launch kernel of a register-budget variant (the first two budgets).
template <typename T>
auto steps_kernel(int variant) -> decltype(&k_batch_steps<T, FluxBudget<T>::v0>) {
  return variant == 0 ? &k_batch_steps<T, FluxBudget<T>::v0> : &k_batch_steps<T, FluxBudget<T>::v1>;
}

template <typename T>
int batch_steps_grid(int variant) {
  int sms = 148, dev = 0, per_sm = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, steps_kernel<T>(variant), 128, WetStage<T>::kBytes);
  return sms * std::max(per_sm, 1);
}

template <typename T>
int launch_batch_steps(const BatchArgs& a, MemberProgress* prog, int nsteps, int grid, cudaStream_t s) {
  const MemberDev<T>* mem = (const MemberDev<T>*)a.mem;
  steps_kernel<T>(a.flux_variant)<<<grid, 128, WetStage<T>::kBytes, s>>>(
      mem, a.nm, a.tile_member, a.ntiles, a.wet_member, a.nwet_blocks, nsteps, a.ctl, prog);
  TRI_CUDA_TRY(cudaGetLastError());
  return TRI_OK;
}

template <typename T>
int prepare_kernels() {
  for (int v = 0; v < 2; v++)
    TRI_CUDA_TRY(cudaFuncSetAttribute(steps_kernel<T>(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)WetStage<T>::kBytes));
  TRI_CUDA_TRY(cudaFuncSetAttribute(k_wetdry_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)WetStage<T>::kBytes));
  TRI_CUDA_TRY(cudaFuncSetAttribute(k_batch_wetdry<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)WetStage<T>::kBytes));
  return TRI_OK;
}

}  // namespace tri
