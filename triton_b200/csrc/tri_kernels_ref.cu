// tri_kernels_ref.cu -- tri_kernel_*_f64: one entry point per reference
// device kernel (src/kernels*.h), same arguments over raw device pointers plus
// the stream.  They keep the reference's one-pass-per-kernel structure so a
// maintainer can swap them into triton_simulate.h call by call; the fused
// domain path (tri_domain.cu) is the fast path.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "tri_face.cuh"
#include "tri_internal.h"

using namespace tri;

namespace {

constexpr int kThreads = 128;  // the reference's raw launcher width (kokkos_utils.h:23)

inline unsigned nblocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__global__ void kr_compute_dt_and_sqrt(int size, double dx, const double* __restrict__ qx,
                                       const double* __restrict__ qy, const double* __restrict__ h,
                                       double* __restrict__ sqrth, double* __restrict__ out, double cn,
                                       double hextra) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  out[id] = kMaxValue;
  const double hij = h[id];
  const double s = fmax(sqrt(hij), 0.0);
  sqrth[id] = s;
  if (hij > hextra) {
    const double maxu = fmax(fabs(qx[id]), fabs(qy[id])) / hij;
    out[id] = cn * dx / (maxu + kSqrtG * s);
  }
}

// Minimum of a double array straight into a device scalar: warp/block
// reduction of order-preserving keys and one atomicMin per block.  The first
// block seeds the result with +inf before any block folds into it (a flag word
// next to the result is not available, so the seed is a separate launch).
// Keys of this path order every double (negatives included): positive values
// get the sign bit set, negative ones are complemented.  The empty key is the
// largest one.
constexpr unsigned long long kEmptyKey = 0xFFFFFFFFFFFFFFFFull;

__global__ void kr_seed_min(unsigned long long* out) { *out = kEmptyKey; }

__global__ void kr_min_keys(int size, const double* __restrict__ v, unsigned long long* __restrict__ out) {
  unsigned long long key = kEmptyKey;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
    const double x = v[i];
    // The reference folds with "a < m ? a : m" from the largest double, so
    // negative values are legal minima; map them so the unsigned order still
    // matches the numeric one.
    unsigned long long k;
    if (x != x) {
      k = kEmptyKey;
    } else {
      const unsigned long long b = (unsigned long long)__double_as_longlong(x);
      k = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    }
    key = k < key ? k : key;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  __shared__ unsigned long long s[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s[warp] = key;
  __syncthreads();
  if (warp == 0) {
    key = lane < (int)(blockDim.x >> 5) ? s[lane] : kEmptyKey;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
      key = other < key ? other : key;
    }
    if (lane == 0) atomicMin(out, key);
  }
}

__global__ void kr_decode_min(unsigned long long* slot) {
  // in place: key -> double (the identity of an empty or all-NaN array is the
  // largest double, as Kokkos::Min starts from it)
  const unsigned long long k = *slot;
  double v;
  if (k == kEmptyKey) {
    v = 1.7976931348623157e308;
  } else {
    const unsigned long long b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    v = __longlong_as_double((long long)b);
  }
  *reinterpret_cast<double*>(slot) = v;
}

template <bool XFACE>
__global__ void kr_flux(int size, int nrows, int ncols, double dx, double dt, const double* __restrict__ h,
                        const double* __restrict__ qx, const double* __restrict__ qy, const double* __restrict__ dem,
                        const double* __restrict__ sqrth, double* rhsh0, double* rhsh1, double* rhsqx0,
                        double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  const int ix = id / ncols, iy = id % ncols;
  int id2;
  if (XFACE) {
    if (ix <= 0 || ix >= nrows - 1 || iy >= ncols - 1) return;  // kernels_flux.h:62-71
    id2 = id + 1;
  } else {
    if (ix <= 0 || ix >= nrows || iy <= 0 || iy >= ncols - 1) return;  // kernels_flux.h:342-354
    id2 = id - ncols;
  }
  CellQ<double> a = make_cell<double>(h[id], qx[id], qy[id], dem[id], hextra);
  CellQ<double> b = make_cell<double>(h[id2], qx[id2], qy[id2], dem[id2], hextra);
  a.sq = sqrth[id];  // the kernels read the SQRTH array, not sqrt(h)
  b.sq = sqrth[id2];
  const bool wet = (a.h > 0.0 || b.h > 0.0);
  const StepK<double> K = step_k<double>(dx, dt, 1.0 / dx, 1.0 / dt, hextra);
  const FaceOut<double> f = face_flux<double, XFACE>(a, b, K);
  if (XFACE) {
    rhsh0[id] = f.a0;
    rhsqx0[id] = f.a1;
    rhsqy0[id] = f.a2;
    rhsh1[id2] = f.b0;
    rhsqx1[id2] = f.b1;
    rhsqy1[id2] = f.b2;
  } else if (wet) {
    rhsh0[id] += f.a0;
    rhsqx0[id] += f.a1;
    rhsqy0[id] += f.a2;
    rhsh1[id2] += f.b0;
    rhsqx1[id2] += f.b1;
    rhsqy1[id2] += f.b2;
  }
}

__global__ void kr_update_cells(int size, int nrows, int ncols, double dt, double* h, double* qx, double* qy,
                                const double* __restrict__ n, const double* rhsh0, const double* rhsh1,
                                const double* rhsqx0, const double* rhsqx1, const double* rhsqy0,
                                const double* rhsqy1, double hextra) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  const int ix = id / ncols, iy = id % ncols;
  if (ix <= 0 || ix >= nrows - 1 || iy <= 0 || iy >= ncols - 1) return;
  const double hn = h[id];
  double hij = hn - rhsh0[id] - rhsh1[id];
  double qxij, qyij;
  if (hij < 0.0) hij = 0.0;
  if (hij < hextra) {
    qxij = 0.0;
    qyij = 0.0;
  } else {
    const double mx = qx[id] - rhsqx0[id] - rhsqx1[id];
    const double my = qy[id] - rhsqy0[id] - rhsqy1[id];
    const double modM = sqrt(mx * mx + my * my);
    if (n[id] > 1e-12 && hn >= hextra && modM > 1e-12) {
      const double tt = dt * kGravity * n[id] * modM / (hn * hn * cbrt(hn));
      const double s = sqrt(1.0 + 4.0 * tt);
      qxij = -0.5 * (mx - mx * s) / tt;
      qyij = -0.5 * (my - my * s) / tt;
    } else {
      qxij = mx;
      qyij = my;
    }
  }
  h[id] = hij;
  qx[id] = qxij;
  qy[id] = qyij;
}

__global__ void kr_update_runoff(int size, int nrows, int ncols, double dt, const int32_t* __restrict__ rid,
                                 int row, int nrows_runoff, const double* __restrict__ rate, double* h, double* qx,
                                 double* qy, double hextra) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  const int ix = id / ncols, iy = id % ncols;
  if (ix <= 0 || ix >= nrows - 1 || iy <= 0 || iy >= ncols - 1) return;
  double hij = h[id];
  const double net = rate[(size_t)rid[id] * nrows_runoff + row];
  hij += net * dt;
  if (hij < hextra) {
    if (hij < 0.0) hij = 0.0;
    qx[id] = 0.0;
    qy[id] = 0.0;
  }
  h[id] = hij;
}

// Point inflows in source order (one thread), so sources sharing a cell add
// up as in the reference's serial build.
__global__ void kr_compute_flow(int size, const double* __restrict__ ht, const double* __restrict__ hv, double dx,
                                double dt, double simtime, int lo, int hi, double* h, const int32_t* __restrict__ pos) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int id = 0; id < size; id++) {
    const double flo = hv[(size_t)lo * size + id], fhi = hv[(size_t)hi * size + id];
    const double tlo = ht[lo], thi = ht[hi];
    double flow;
    if (lo == hi) {
      flow = flo;
    } else {
      const double td = simtime - tlo, td2 = thi - tlo;
      flow = flo + (((fhi - flo) * td) / td2);
    }
    const int sid = pos[id];
    double hij = h[sid];
    hij += (flow * dt) / (dx * dx);
    h[sid] = hij;
  }
}

__global__ void kr_open_we(int size, int nrows, int ncols, double* h, double* qx, double* qy) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  int g, i;
  if (id < nrows) {
    g = (id % nrows) * ncols + id / nrows;
    i = (id % nrows) * ncols + 1;
  } else {
    g = (id % nrows) * ncols + id / nrows + ncols - 2;
    i = (id % nrows) * ncols + ncols - 2;
  }
  h[g] = h[i];
  qx[g] = qx[i];
  qy[g] = qy[i];
}

__global__ void kr_open_ns(int size, int nrows, int ncols, double* h, double* qx, double* qy, int rank, int nproc) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  if (rank > 0 && rank < nproc - 1) return;
  if (rank == 0) {
    const int g = id, i = (id % ncols) + ncols;
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
  }
  if (rank == nproc - 1) {
    const int g = id + (nrows - 1) * ncols, i = (id % ncols) + (nrows - 2) * ncols;
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
  }
}

__global__ void kr_wet_dry(int size, int nrows, int ncols, const double* __restrict__ h, double* qx, double* qy,
                           const double* __restrict__ dem, double* maxh, double hextra, int mpi_tasks) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  const int ix = id / ncols, iy = id % ncols;
  if (ix <= 0 || ix >= nrows - 1 || iy <= 0 || iy >= ncols - 1) return;
  const int rx = ix * ncols;
  const double hij = h[id], zij = dem[id];
  if (hij > hextra) {
    if ((hij + zij < dem[rx + iy + 1] && h[rx + iy + 1] < 1e-12) ||
        (hij + zij < dem[rx + iy - 1] && h[rx + iy - 1] < 1e-12))
      qx[id] = 0.0;
    if (ix == 1 && mpi_tasks > 1) {
      if (hij + zij < dem[rx + ncols + iy] && h[rx + ncols + iy] < 1e-12) qy[id] = 0.0;
    } else if (ix == nrows - 2 && mpi_tasks > 1) {
      if (hij + zij < dem[rx - ncols + iy] && h[rx - ncols + iy] < 1e-12) qy[id] = 0.0;
    } else if ((hij + zij < dem[rx - ncols + iy] && h[rx - ncols + iy] < 1e-12) ||
               (hij + zij < dem[rx + ncols + iy] && h[rx + ncols + iy] < 1e-12)) {
      qy[id] = 0.0;
    }
  }
  if (hij > maxh[id]) maxh[id] = hij;
}

__global__ void kr_extbc(const int32_t* __restrict__ order, int count, int nrows, int ncols, double dt, double* h,
                         double* qx, double* qy, const double* __restrict__ dem, const double* __restrict__ n,
                         const int32_t* __restrict__ rel, const int32_t* __restrict__ types,
                         const int32_t* __restrict__ start, const int32_t* __restrict__ nvars,
                         const double* __restrict__ v1, const double* __restrict__ v2, double simtime, int rank,
                         int nproc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int id = order[k];
  const int ii = rel[id], bt = types[id], s0 = start[id];
  const int ix = ii / ncols, iy = ii % ncols;
  const bool top = ix == 1, btm = ix == nrows - 2, lt = iy == 1, rt = iy == ncols - 2;
  if (!((rank == 0 && top) || lt || rt || (rank == nproc - 1 && btm))) return;
  bool corner = false;
  int ib = ii, ibc = ii;
  double f0 = 1.0, f1 = 0.0, f2 = 0.0;
  if (lt) { ib = ii - 1; f1 = -1.0; f2 = 0.0; }
  if (rt) { ib = ii + 1; f1 = 1.0; f2 = 0.0; }
  if (rank == 0 && top) {
    ib = ii - ncols; f1 = 0.0; f2 = 1.0;
    if (lt) { corner = true; ibc = ii - 1; f2 = 0.0; }
    if (rt) { corner = true; ibc = ii + 1; f2 = 0.0; }
  }
  if (rank == nproc - 1 && btm) {
    ib = ii + ncols; f1 = 0.0; f2 = -1.0;
    if (lt) { corner = true; ibc = ii - 1; f2 = 0.0; }
    if (rt) { corner = true; ibc = ii + 1; f2 = 0.0; }
  }
  double hij = h[ii], qxij = qx[ii], qyij = qy[ii];
  if (bt == 0) {
    h[ib] = hij; qx[ib] = qxij; qy[ib] = qyij;
    if (corner) { h[ibc] = hij; qx[ibc] = qxij; qy[ibc] = qyij; }
    return;
  }
  if (bt == 1) {
    const double lvar = 0.5 * (simtime + simtime + dt);
    int lo = 0, hi = nvars[id] - 1;
    if (lvar < v1[s0]) {
      lo = 0; hi = 0;
    } else if (lvar > v1[hi + s0]) {
      lo = hi;
    } else {
      for (int i = 0; i < hi; i++)
        if (v1[i + s0] <= lvar && v1[i + 1 + s0] > lvar) { lo = i; hi = i + 1; break; }
    }
    double aux;
    if (lo == hi) {
      aux = v2[lo + s0];
    } else {
      const double td = lvar - v1[lo + s0], td2 = v1[hi + s0] - v1[lo + s0];
      aux = v2[lo + s0] + (((v2[hi + s0] - v2[lo + s0]) * td) / td2);
    }
    hij = fmax(aux - dem[ii], 0.0);
  } else {
    const double aux = v1[s0];
    double vel = 0.0;
    if (bt == 2) vel = sqrt(aux * hij * cbrt(hij) / fmax(n[ii], 1e-6));
    if (bt == 3) vel = aux * sqrt(kGravity * hij);
    qxij = hij * vel;
    qyij = hij * vel;
  }
  h[ib] = hij * f0; qx[ib] = qxij * f1; qy[ib] = qyij * f2;
  h[ii] = hij * f0; qx[ii] = qxij * f1; qy[ii] = qyij * f2;
  if (corner) { h[ibc] = hij * f0; qx[ibc] = qxij * f1; qy[ibc] = qyij * f2; }
}

__global__ void kr_copy_obs(int size, const double* __restrict__ arr, double* __restrict__ out,
                            const int32_t* __restrict__ idx) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id < size) out[id] = arr[idx[id]];
}

int launched() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(TRI_E_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  return TRI_OK;
}

// Application order of tri_kernel_compute_extbc_values_f64 for one host
// thread on one device: the cell list it was built for, its waves, and its
// device copy (allocated on that device, grown when a longer list comes).
struct ExtbcOrderCache {
  std::vector<int32_t> cells, order, waves;
  int32_t* d_order = nullptr;
  size_t cap = 0;
};

// Per host thread (each thread's calls are ordered on its own streams), per
// device.  At thread exit the device copies are freed; a failure there (the
// runtime may be shutting down at process exit) is ignored.
struct ExtbcOrderCaches {
  std::vector<std::pair<int, ExtbcOrderCache>> by_device;
  ~ExtbcOrderCaches() {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return;
    for (auto& e : by_device) {
      if (!e.second.d_order) continue;
      if (cudaSetDevice(e.first) == cudaSuccess) cudaFree(e.second.d_order);
    }
    cudaSetDevice(cur);
  }
};

ExtbcOrderCache& extbc_cache_of(int dev) {
  static thread_local ExtbcOrderCaches caches;
  for (auto& e : caches.by_device)
    if (e.first == dev) return e.second;
  caches.by_device.emplace_back(dev, ExtbcOrderCache());
  return caches.by_device.back().second;
}

}  // namespace

extern "C" {

int tri_kernel_compute_dt_and_sqrt_f64(int size, double dx, const double* qx, const double* qy, const double* h,
                                       double* sqrth, double* dt_out, double cn, double hextra, void* stream) {
  if (size <= 0) return TRI_OK;
  TRI_CHECK_ARG(qx && qy && h && sqrth && dt_out, "null device pointer");
  kr_compute_dt_and_sqrt<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, dx, qx, qy, h, sqrth, dt_out, cn,
                                                                          hextra);
  return launched();
}

int tri_kernel_find_min_dt_f64(int size, const double* dt, double* min_out, void* stream) {
  TRI_CHECK_ARG(dt && min_out, "null device pointer");
  TRI_CHECK_ARG(((uintptr_t)min_out & 7) == 0, "min_out must be 8-byte aligned");
  cudaStream_t s = as_stream(stream);
  unsigned long long* slot = reinterpret_cast<unsigned long long*>(min_out);
  kr_seed_min<<<1, 1, 0, s>>>(slot);
  if (size > 0) {
    const unsigned nb = std::min<unsigned>(nblocks(size), 148u * 8u);
    kr_min_keys<<<nb, 256, 0, s>>>(size, dt, slot);
  }
  kr_decode_min<<<1, 1, 0, s>>>(slot);
  return launched();
}

int tri_kernel_flux_x_f64(int size, int nrows, int ncols, double dx, double dt, const double* h, const double* qx,
                          const double* qy, const double* dem, const double* sqrth, double* rhsh0, double* rhsh1,
                          double* rhsqx0, double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra,
                          void* stream) {
  if (size <= 0) return TRI_OK;
  TRI_CHECK_ARG(size == nrows * ncols, "size must be nrows*ncols");
  kr_flux<true><<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, dx, dt, h, qx, qy, dem, sqrth,
                                                                   rhsh0, rhsh1, rhsqx0, rhsqx1, rhsqy0, rhsqy1,
                                                                   hextra);
  return launched();
}

int tri_kernel_flux_y_f64(int size, int nrows, int ncols, double dx, double dt, const double* h, const double* qx,
                          const double* qy, const double* dem, const double* sqrth, double* rhsh0, double* rhsh1,
                          double* rhsqx0, double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra,
                          void* stream) {
  if (size <= 0) return TRI_OK;
  TRI_CHECK_ARG(size == nrows * ncols, "size must be nrows*ncols");
  kr_flux<false><<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, dx, dt, h, qx, qy, dem,
                                                                    sqrth, rhsh0, rhsh1, rhsqx0, rhsqx1, rhsqy0,
                                                                    rhsqy1, hextra);
  return launched();
}

int tri_kernel_update_cells_f64(int size, int nrows, int ncols, double dt, double* h, double* qx, double* qy,
                                const double* dem, const double* n, double* rhsh0, double* rhsh1, double* rhsqx0,
                                double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra, void* stream) {
  (void)dem;
  if (size <= 0) return TRI_OK;
  kr_update_cells<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, dt, h, qx, qy, n, rhsh0,
                                                                    rhsh1, rhsqx0, rhsqx1, rhsqy0, rhsqy1, hextra);
  return launched();
}

int tri_kernel_update_runoff_f64(int size, int nrows, int ncols, double dt, const int32_t* runoff_id,
                                 int index_row_runoff, int n_rows_runoff, const double* runoff_intensity, double* h,
                                 double* qx, double* qy, double hextra, void* stream) {
  if (size <= 0) return TRI_OK;
  kr_update_runoff<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, dt, runoff_id,
                                                                     index_row_runoff, n_rows_runoff,
                                                                     runoff_intensity, h, qx, qy, hextra);
  return launched();
}

int tri_kernel_compute_flow_f64(int size, const double* hyd_time, const double* hyd_val, double dx, double dt,
                                double simtime, int idx_low, int idx_high, double* h, const int32_t* pos,
                                void* stream) {
  if (size <= 0) return TRI_OK;
  kr_compute_flow<<<1, 32, 0, as_stream(stream)>>>(size, hyd_time, hyd_val, dx, dt, simtime, idx_low, idx_high, h,
                                                   pos);
  return launched();
}

int tri_kernel_copy_info_to_exterior_boundaries_west_east_f64(int size, int nrows, int ncols, double* h, double* qx,
                                                              double* qy, void* stream) {
  if (size <= 0) return TRI_OK;
  kr_open_we<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, h, qx, qy);
  return launched();
}

int tri_kernel_copy_info_to_exterior_boundaries_north_south_f64(int size, int nrows, int ncols, double* h,
                                                                double* qx, double* qy, int rank,
                                                                int total_process, void* stream) {
  if (size <= 0) return TRI_OK;
  kr_open_ns<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, h, qx, qy, rank, total_process);
  return launched();
}

int tri_kernel_compute_extbc_values_f64(int size, int nrows, int ncols, double dt, double* h, double* qx, double* qy,
                                        const double* dem, const double* n, const int32_t* relative_index,
                                        const int32_t* extbctype, const int32_t* start_index,
                                        const int32_t* nrows_vars, const double* extbcvar1, const double* extbcvar2,
                                        double simtime, int rank, int total_process, void* stream) {
  if (size <= 0) return TRI_OK;
  TRI_CHECK_ARG(relative_index && extbctype && start_index && nrows_vars, "null device pointer");
  // The cell list decides the application order: cells that touch the same
  // cell run in index order (the reference's serial semantics), the rest in
  // parallel.  The list is small (boundary cells); its waves are cached per
  // host thread and device (a device pointer is only valid on the device it
  // was allocated on), keyed by the list's contents.
  cudaStream_t s = as_stream(stream);
  int dev = 0;
  TRI_CUDA_TRY(cudaGetDevice(&dev));
  ExtbcOrderCache& cache = extbc_cache_of(dev);
  std::vector<int32_t> cells((size_t)size);
  TRI_CUDA_TRY(cudaMemcpyAsync(cells.data(), relative_index, size * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TRI_CUDA_TRY(cudaStreamSynchronize(s));
  if (cells != cache.cells) {
    std::vector<std::vector<int64_t>> touch((size_t)size);
    for (int i = 0; i < size; i++) {
      const int64_t ii = cells[i];
      touch[i] = extbc_touches(ii, nrows, ncols);
    }
    cache.cells.clear();  // stays invalid if an allocation or copy below fails
    build_waves(touch, cache.order, cache.waves);
    if (cache.cap < cache.order.size()) {
      if (cache.d_order) cudaFree(cache.d_order);
      cache.d_order = nullptr;
      cache.cap = 0;
      TRI_CUDA_TRY(cudaMalloc((void**)&cache.d_order, cache.order.size() * sizeof(int32_t)));
      cache.cap = cache.order.size();
    }
    TRI_CUDA_TRY(cudaMemcpy(cache.d_order, cache.order.data(), cache.order.size() * sizeof(int32_t),
                            cudaMemcpyHostToDevice));
    cache.cells = std::move(cells);
  }
  for (size_t w = 0; w + 1 < cache.waves.size(); w++) {
    const int off = cache.waves[w], cnt = cache.waves[w + 1] - off;
    kr_extbc<<<nblocks(cnt), kThreads, 0, s>>>(cache.d_order + off, cnt, nrows, ncols, dt, h, qx, qy, dem, n,
                                                relative_index, extbctype, start_index, nrows_vars, extbcvar1,
                                                extbcvar2, simtime, rank, total_process);
  }
  return launched();
}

int tri_kernel_wet_dry_f64(int size, int nrows, int ncols, double dt, const double* h, double* qx, double* qy,
                           const double* dem, double* max_h, double hextra, int mpi_tasks, void* stream) {
  (void)dt;
  if (size <= 0) return TRI_OK;
  kr_wet_dry<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, nrows, ncols, h, qx, qy, dem, max_h, hextra,
                                                               mpi_tasks);
  return launched();
}

int tri_kernel_copy_observation_points_f64(int size, const double* arr, double* obs_arr,
                                           const int32_t* relative_index, void* stream) {
  if (size <= 0) return TRI_OK;
  kr_copy_obs<<<nblocks(size), kThreads, 0, as_stream(stream)>>>(size, arr, obs_arr, relative_index);
  return launched();
}

}  // extern "C"

// ---- no-alloc variant of compute_extbc_values ------------------------------
// tri_kernel_compute_extbc_values_f64 keeps its application order in device
// memory it allocates (and grows) on first use.  Callers that cannot allocate
// device memory inside their time loop use the variant below, whose order
// lives in a fixed array in the library's own device image: a host that
// claimed the GPU's free memory before the loop (the reference creates every
// device array up front, triton_init.h:1452-1591; a memory pool or caching
// allocator in the same process may hold the rest) would see cudaMalloc fail
// mid-run, and cudaMalloc/cudaFree synchronize the whole device, stalling the
// other streams of the step.
namespace {

// 65536 boundary cells (the four edges of a 16384 x 16384 interior), 256 KiB.
constexpr int kNoAllocExtbcMaxCells = TRI_NOALLOC_EXTBC_MAX_CELLS;
// Application order: indices into the cell list, wave after wave.  Nothing in
// it has to start at zero: a call launches the boundary kernel only after the
// order of its own cell list has been written here (by this call, or by the
// previous call on this device with the same list).
static __device__ __align__(256) int32_t g_extbc_order[kNoAllocExtbcMaxCells];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocSlot {
  int32_t* order = nullptr;    // device address of g_extbc_order on this device
  std::vector<int32_t> cells;  // cell list whose order g_extbc_order holds
  std::vector<int32_t> order_host, waves;
};
std::mutex g_noalloc_mu;  // guards the host-side slots only
NoAllocSlot g_noalloc[kNoAllocMaxDevices];

}  // namespace

extern "C" int tri_kernel_compute_extbc_values_noalloc_f64(
    int size, int nrows, int ncols, double dt, double* h, double* qx, double* qy, const double* dem, const double* n,
    const int32_t* relative_index, const int32_t* extbctype, const int32_t* start_index, const int32_t* nrows_vars,
    const double* extbcvar1, const double* extbcvar2, double simtime, int rank, int total_process, void* stream) {
  if (size <= 0) return TRI_OK;
  TRI_CHECK_ARG(size <= kNoAllocExtbcMaxCells,
                "compute_extbc_values_noalloc: %d boundary cells exceed its fixed limit of %d; use "
                "tri_kernel_compute_extbc_values_f64 for longer lists",
                size, kNoAllocExtbcMaxCells);
  TRI_CHECK_ARG(relative_index && extbctype && start_index && nrows_vars, "null device pointer");
  int dev = 0;
  TRI_CUDA_TRY(cudaGetDevice(&dev));
  TRI_CHECK_ARG(dev >= 0 && dev < kNoAllocMaxDevices, "device %d beyond the %d devices the no-alloc entry serves",
                dev, kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot& slot = g_noalloc[dev];
  if (!slot.order) {
    // once per device, with that device current; may load the module
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_extbc_order);
    if (e != cudaSuccess || !p)
      return set_error(TRI_E_CUDA, "compute_extbc_values_noalloc: address of the order array on device %d: %s",
                       dev, cudaGetErrorString(e));
    slot.order = (int32_t*)p;
  }
  cudaStream_t s = as_stream(stream);
  std::vector<int32_t> cells((size_t)size);
  TRI_CUDA_TRY(cudaMemcpyAsync(cells.data(), relative_index, size * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TRI_CUDA_TRY(cudaStreamSynchronize(s));
  if (cells != slot.cells) {
    std::vector<std::vector<int64_t>> touch((size_t)size);
    for (int i = 0; i < size; i++) {
      const int64_t ii = cells[i];
      touch[i] = extbc_touches(ii, nrows, ncols);
    }
    slot.cells.clear();  // stays invalid if the copy below fails
    build_waves(touch, slot.order_host, slot.waves);
    TRI_CUDA_TRY(cudaMemcpyAsync(slot.order, slot.order_host.data(), slot.order_host.size() * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, s));
    // The order is marked valid only once it has landed: a later call with
    // the same list on another stream launches without copying it again.
    TRI_CUDA_TRY(cudaStreamSynchronize(s));
    slot.cells = std::move(cells);
  }
  for (size_t w = 0; w + 1 < slot.waves.size(); w++) {
    const int off = slot.waves[w], cnt = slot.waves[w + 1] - off;
    kr_extbc<<<nblocks(cnt), kThreads, 0, s>>>(slot.order + off, cnt, nrows, ncols, dt, h, qx, qy, dem, n,
                                                relative_index, extbctype, start_index, nrows_vars, extbcvar1,
                                                extbcvar2, simtime, rank, total_process);
  }
  return launched();
}
