// tri_domain.cu -- the domain entry points of the C ABI (include/triton_b200.h).
//
// A domain owns the device arrays of one simulation (the reference allocates
// them in create_device_vectors, triton_init.h:1452-1591) and runs whole time
// steps with the fused kernels of tri_step_kernels.cuh.  The CFL dt is reduced
// on the device and the reference's dt policy runs there too, so the steps of
// an advance() call need no host round trip; steps are launched in chunks
// captured as CUDA graphs and stop at the first event the reference loop
// reacts to (triton_simulate.h:69-134).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "tri_internal.h"
#include "tri_domain_impl.h"
#include "tri_step_launch.h"
#include "tri_types.cuh"

namespace tri {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void build_waves(const std::vector<std::vector<int64_t>>& touches, std::vector<int32_t>& order,
                        std::vector<int32_t>& wave_start) {
  const int n = (int)touches.size();
  std::map<int64_t, int> last;
  std::vector<int> wave(n, 0);
  int nw = 0;
  for (int k = 0; k < n; k++) {
    int w = 0;
    for (int64_t cidx : touches[k]) {
      auto it = last.find(cidx);
      if (it != last.end()) w = std::max(w, it->second + 1);
    }
    wave[k] = w;
    for (int64_t cidx : touches[k]) last[cidx] = w;
    nw = std::max(nw, w + 1);
  }
  order.clear();
  wave_start.assign(1, 0);
  for (int w = 0; w < nw; w++) {
    for (int k = 0; k < n; k++)
      if (wave[k] == w) order.push_back(k);
    wave_start.push_back((int32_t)order.size());
  }
}

}  // namespace tri

using namespace tri;

namespace {

template <typename T>
StateBufs<T> bufs(tri_domain* d) {
  StateBufs<T> s;
  for (int i = 0; i < 2; i++) {
    s.h[i] = (T*)d->h[i];
    s.qx[i] = (T*)d->qx[i];
    s.qy[i] = (T*)d->qy[i];
  }
  return s;
}

void free_dev(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <typename P>
void free_devp(P*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void drop_graph(tri_domain* d) {
  if (d->graph) cudaGraphExecDestroy(d->graph);
  d->graph = nullptr;
  d->graph_steps = 0;
}

int64_t footprint_bytes(const tri_grid_desc* g) {
  const int64_t n = (int64_t)g->rows * g->cols;
  const int64_t es = g->precision == TRI_FP32 ? 4 : 8;
  // 6 state buffers + z + n2 + maxh, one FP64 staging field, runoff zone ids
  return n * es * 9 + 9 * (int64_t)kFieldPad + n * 8 + n * 4 + (1 << 20);
}

template <typename T>
__global__ void k_from_f64(const double* __restrict__ src, T* __restrict__ dst, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (T)src[i];
}
template <typename T>
__global__ void k_to_f64(const T* __restrict__ src, double* __restrict__ dst, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}

// FP32 form: offsets of the bed from each 32x32 tile's FP64 base level.
// Base level of each 32x32 tile (one block of 256 threads per tile): the
// lowest interior cell of the tile (ghost cells hold walls or copies and must
// not pull the base away from the terrain), 0 for a tile without interior
// cells; NaN levels are passed over; a zero base is +0.
__global__ void k_tile_base(const double* __restrict__ z, double* __restrict__ base, int rows, int cols, int ntc) {
  const int tr = blockIdx.y, tc = blockIdx.x;
  double m = 1e300;
  for (int k = threadIdx.x; k < 32 * 32; k += blockDim.x) {
    const int r = tr * 32 + (k >> 5), c = tc * 32 + (k & 31);
    if (r >= 1 && r <= rows - 2 && c >= 1 && c <= cols - 2) m = fmin(m, z[(size_t)r * cols + c]);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmin(m, wm[w]);
    base[(size_t)tr * ntc + tc] = (m == 1e300 || m == 0.0) ? 0.0 : m;
  }
}

__global__ void k_bed_offsets(const double* __restrict__ z, const double* __restrict__ base, float* __restrict__ off,
                              int rows, int cols, int ntc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)rows * cols) return;
  const int r = (int)(i / cols), c = (int)(i % cols);
  off[i] = (float)(z[i] - base[(r >> 5) * ntc + (c >> 5)]);
}
__global__ void k_bed_levels(const float* __restrict__ off, const double* __restrict__ base, double* __restrict__ z,
                             int rows, int cols, int ntc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)rows * cols) return;
  const int r = (int)(i / cols), c = (int)(i % cols);
  z[i] = base[(r >> 5) * ntc + (c >> 5)] + (double)off[i];
}

template <typename T>
__global__ void k_observe(const DevClock* __restrict__ clk, StateBufs<T> sb, const int32_t* __restrict__ cells,
                          int nobs, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nobs) return;
  const int b = clk->cur;
  const int id = cells[k];
  out[k] = (double)sb.H(b)[id];
  out[nobs + k] = (double)sb.QX(b)[id];
  out[2 * nobs + k] = (double)sb.QY(b)[id];
}

// Interior volume: each block sums a fixed set of rows in a fixed order, then
// one block adds the partials in block order, so the result is reproducible.
template <typename T>
__global__ void __launch_bounds__(256) k_volume_part(const DevClock* __restrict__ clk, StateBufs<T> sb, int rows,
                                                     int cols, double* __restrict__ part) {
  const T* h = sb.H(clk->cur);
  double acc = 0.0;
  for (int r = 1 + blockIdx.x; r <= rows - 2; r += gridDim.x)
    for (int c = 1 + threadIdx.x; c <= cols - 2; c += blockDim.x) acc += (double)h[(size_t)r * cols + c];
  __shared__ double s[256];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
__global__ void k_volume_sum(const double* __restrict__ part, int n, double scale, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double acc = 0.0;
  for (int i = 0; i < n; i++) acc += part[i];
  *out = acc * scale;
}

// *flag = 1 if any of the n values is negative or NaN (a zero of either sign is not).
template <typename T>
__global__ void k_flag_negative(const T* __restrict__ v, int64_t n, int32_t* __restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool neg = i < n && !(v[i] >= T(0));
  if (__syncthreads_or(neg) && threadIdx.x == 0) atomicExch(flag, 1);
}

StepArgs step_args(tri_domain* d) {
  StepArgs a{};
  a.clk = d->clk;
  for (int i = 0; i < 2; i++) {
    a.h[i] = d->h[i];
    a.qx[i] = d->qx[i];
    a.qy[i] = d->qy[i];
  }
  a.z = d->z;
  a.zbase = d->zbase;
  a.ntc = d->ntc;
  a.n2 = d->n2;
  a.maxh = d->maxh;
  a.zone = d->zone;
  a.rates = d->rates;
  a.rows = d->desc.rows;
  a.cols = d->desc.cols;
  a.rb = d->rb;
  a.flux_blocks = d->flux_blocks;
  a.flux_variant = d->flux_variant;
  a.dx = d->desc.cell_size;
  a.courant = d->desc.courant;
  a.hextra = d->desc.hextra;
  a.open_boundaries = d->desc.open_boundaries;
  a.nsrc = d->nsrc;
  a.src_cells = d->src_cells;
  a.src_order = d->src_order;
  a.hyg_t = d->hyg_t;
  a.hyg_v = d->hyg_v;
  a.src_waves = d->src_waves.data();
  a.n_src_waves = d->src_waves.empty() ? 0 : (int)d->src_waves.size() - 1;
  a.nbc = d->nbc;
  a.bc_cells = d->bc_cells;
  a.bc_types = d->bc_types;
  a.bc_start = d->bc_start;
  a.bc_nrows = d->bc_nrows;
  a.bc_order = d->bc_order;
  a.bc_v1 = d->bc_v1;
  a.bc_v2 = d->bc_v2;
  a.bc_waves = d->bc_waves.data();
  a.n_bc_waves = d->bc_waves.empty() ? 0 : (int)d->bc_waves.size() - 1;
  a.arrival = d->arrival;
  a.arrival_depth = d->arrival_depth;
  a.tzero = d->tz_on ? d->tzero : nullptr;
  a.tzero_wet = (d->arrival == nullptr || d->arrival_depth >= 0.0f) ? a.tzero : nullptr;
  a.maxh_neg = d->maxh_neg;
  return a;
}

// Resets the dry-tile flags of the flux kernel for the current tile shape
// (nothing is known to be zero, so the next two steps compute every tile)
// and marks the tiles that must never be skipped: those holding a source or
// an external boundary cell, and the edge tiles when the open boundaries
// rewrite the ghost ring.  Runoff reaches every cell, so a domain with runoff
// computes every tile.  Called outside graph capture, before steps.
int reset_tiles(tri_domain* d) {
  const int rows = d->desc.rows, cols = d->desc.cols;
  const int64_t ns = (cols - 2 + kStripCols - 1) / kStripCols, nty = (rows - 2 + d->rb - 1) / d->rb;
  const int64_t nt = ns * nty;
  d->tz_dirty = false;
  d->tz_on = d->nroff == 0;
  if (!d->tz_on) return TRI_OK;
  if (nt > d->tz_cap) {
    drop_graph(d);  // the graphs hold the old flag pointer
    free_devp(d->tzero);
    d->tz_cap = 0;
    if (cudaMalloc((void**)&d->tzero, 3 * (size_t)nt) != cudaSuccess) {
      d->tz_on = false;
      return set_error(TRI_E_NOMEM, "cudaMalloc of %lld tile flags failed", (long long)(3 * nt));
    }
    d->tz_cap = nt;
  }
  if (nt != d->tz_tiles) drop_graph(d);  // the pinned table moved
  d->tz_tiles = nt;
  std::vector<uint8_t>& pin = d->tz_pin_host;
  pin.assign((size_t)nt, 0);
  auto pin_cell = [&](int64_t id) {
    const int r = (int)(id / cols), c = (int)(id % cols);
    const int64_t ry = std::min<int64_t>(std::max(r - 1, 0) / d->rb, nty - 1);
    const int64_t sx = std::min<int64_t>(std::max(c - 1, 0) / kStripCols, ns - 1);
    pin[(size_t)(ry * ns + sx)] = 1;
  };
  if (d->nsrc > 0)
    for (int32_t id : d->src_cells_host) pin_cell(id);
  if (d->nbc > 0)
    for (int32_t id : d->bc_cells_host) pin_cell(id);
  if (d->desc.open_boundaries)
    for (int64_t ry = 0; ry < nty; ry++)
      for (int64_t sx = 0; sx < ns; sx++)
        if (ry == 0 || ry == nty - 1 || sx == 0 || sx == ns - 1) pin[(size_t)(ry * ns + sx)] = 1;
  TRI_CUDA_TRY(cudaMemsetAsync(d->tzero, 0, 2 * (size_t)nt, d->stream));
  TRI_CUDA_TRY(cudaMemcpyAsync(d->tzero + 2 * nt, pin.data(), (size_t)nt, cudaMemcpyHostToDevice, d->stream));
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));  // 'pin' may be reassigned before the copy ran
  return TRI_OK;
}

// Grid of the flux kernel for the domain's variant and tile height: one
// resident wave of blocks, each warp fetching tiles until none are left.
void size_flux_grid(tri_domain* d) {
  const int rows = d->desc.rows - 2, cols = d->desc.cols - 2;
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = 0;
  if (d->prec == TRI_FP64)
    flux_occupancy<double>(d->flux_variant, &per_sm);
  else
    flux_occupancy<float>(d->flux_variant, &per_sm);
  if (per_sm < 1) per_sm = 1;
  const int64_t strips = (cols + kStripCols - 1) / kStripCols;
  const int64_t tiles = strips * ((rows + d->rb - 1) / d->rb);
  d->flux_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, (tiles + 3) / 4));
}

// Default shape before any tuning: the register budget of 5 blocks per SM
// in FP64 and 8 in FP32 (the fastest on watersheds of 1024^2 to 8192^2) and
// the largest tile height, 32 down to 8, that still gives every warp of a
// full wave about eight tiles.
void choose_shape(tri_domain* d) {
  const int rows = d->desc.rows - 2, cols = d->desc.cols - 2;
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t strips = (cols + kStripCols - 1) / kStripCols;
  const int64_t warps = (int64_t)sms * 12;
  int rb = 32;
  while (rb > 8 && strips * ((rows + rb - 1) / rb) < 8 * warps) rb /= 2;
  d->flux_variant = d->prec == TRI_FP64 ? 1 : 2;
  d->rb = rb;
  size_flux_grid(d);
}

int launch_one_step(tri_domain* d) {
  cudaEvent_t* ev = nullptr;
  if (d->timing) {
    while (d->tev.size() < d->tev_used + 4) {
      cudaEvent_t e;
      TRI_CUDA_TRY(cudaEventCreate(&e));
      d->tev.push_back(e);
    }
    ev = &d->tev[d->tev_used];
    d->tev_used += 4;
  }
  const StepArgs a = step_args(d);
  return d->prec == TRI_FP64 ? launch_step<double>(a, d->stream, ev) : launch_step<float>(a, d->stream, ev);
}

int launch_dt(tri_domain* d) {
  const StepArgs a = step_args(d);
  return d->prec == TRI_FP64 ? launch_initial_dt<double>(a, d->stream) : launch_initial_dt<float>(a, d->stream);
}

int launch_steps(tri_domain* d, int n) {
  if (d->use_graphs && !d->timing) {
    const int G = 8;
    if (!d->graph) {
      cudaGraph_t g = nullptr;
      TRI_CUDA_TRY(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal));
      int rc = TRI_OK;
      for (int i = 0; i < G && rc == TRI_OK; i++)
        rc = launch_one_step(d);
      cudaError_t e = cudaStreamEndCapture(d->stream, &g);
      if (rc != TRI_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return set_error(TRI_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&d->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return set_error(TRI_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
      d->graph_steps = G;
    }
    while (n >= d->graph_steps) {
      TRI_CUDA_TRY(cudaGraphLaunch(d->graph, d->stream));
      n -= d->graph_steps;
    }
  }
  for (int i = 0; i < n; i++) {
    int rc = launch_one_step(d);
    if (rc != TRI_OK) return rc;
  }
  return TRI_OK;
}

int field_ptr(tri_domain* d, int field, void** p) {
  switch (field) {
    case TRI_FIELD_H: *p = d->h[d->mirror->cur]; return TRI_OK;
    case TRI_FIELD_QX: *p = d->qx[d->mirror->cur]; return TRI_OK;
    case TRI_FIELD_QY: *p = d->qy[d->mirror->cur]; return TRI_OK;
    case TRI_FIELD_NMAN2: *p = d->n2; return TRI_OK;
    case TRI_FIELD_DEM: *p = d->z; return TRI_OK;
    case TRI_FIELD_MAXH: *p = d->maxh; return TRI_OK;
  }
  return set_error(TRI_E_INVALID, "unknown field id %d", field);
}

template <typename T>
int upload_table(tri_domain* d, const double* host, int64_t n, void** dst) {
  free_dev(*dst);
  const int64_t m = std::max<int64_t>(n, 1);
  TRI_CUDA_TRY(cudaMalloc(dst, m * sizeof(T)));
  if (n == 0) return TRI_OK;
  if (sizeof(T) == 8) {
    TRI_CUDA_TRY(cudaMemcpyAsync(*dst, host, n * 8, cudaMemcpyHostToDevice, d->stream));
  } else {
    std::vector<float> tmp(host, host + n);
    TRI_CUDA_TRY(cudaMemcpyAsync(*dst, tmp.data(), n * 4, cudaMemcpyHostToDevice, d->stream));
    TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  }
  return TRI_OK;
}

int upload_raw(tri_domain* d, const void* host, size_t bytes, void** dst) {
  free_dev(*dst);
  TRI_CUDA_TRY(cudaMalloc(dst, std::max<size_t>(bytes, 8)));
  if (bytes) TRI_CUDA_TRY(cudaMemcpyAsync(*dst, host, bytes, cudaMemcpyHostToDevice, d->stream));
  return TRI_OK;
}

int push_clock(tri_domain* d) {
  TRI_CUDA_TRY(cudaMemcpyAsync(d->clk, d->mirror, sizeof(DevClock), cudaMemcpyHostToDevice, d->stream));
  return TRI_OK;
}
int pull_clock(tri_domain* d) {
  TRI_CUDA_TRY(cudaMemcpyAsync(d->mirror, d->clk, sizeof(DevClock), cudaMemcpyDeviceToHost, d->stream));
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  return TRI_OK;
}

}  // namespace

namespace tri {
int domain_push_clock(tri_domain* d) { return push_clock(d); }
int domain_pull_clock(tri_domain* d) { return pull_clock(d); }
int domain_launch_dt(tri_domain* d) { return launch_dt(d); }
StepArgs domain_step_args(tri_domain* d) { return step_args(d); }
}  // namespace tri

extern "C" {

int tri_abi_version(void) { return TRI_ABI_VERSION; }

const char* tri_last_error(void) { return g_last_error.c_str(); }

int tri_domain_footprint(const tri_grid_desc* desc, int64_t* bytes) {
  TRI_CHECK_ARG(desc && bytes, "null argument");
  *bytes = footprint_bytes(desc);
  return TRI_OK;
}

int tri_domain_create(const tri_grid_desc* desc, void* stream, tri_domain** out) {
  TRI_CHECK_ARG(desc && out, "null argument");
  TRI_CHECK_ARG(desc->rows >= 3 && desc->cols >= 3, "grid must have at least one interior cell (rows=%d cols=%d)",
                desc->rows, desc->cols);
  TRI_CHECK_ARG((int64_t)desc->rows * desc->cols < (int64_t)1 << 31, "grid too large for 32-bit cell indices");
  TRI_CHECK_ARG(desc->cell_size > 0, "cell_size must be positive");
  TRI_CHECK_ARG(desc->precision == TRI_FP64 || desc->precision == TRI_FP32, "unknown precision %d", desc->precision);
  *out = nullptr;
  tri_domain* d = new tri_domain();
  d->desc = *desc;
  d->prec = desc->precision;
  d->esize = d->prec == TRI_FP64 ? 8 : 4;
  d->ncells = (int64_t)desc->rows * desc->cols;
  int rc = TRI_OK;
  auto fail = [&](int code) {
    tri_domain_destroy(d);
    return code;
  };
  if (stream) {
    d->stream = as_stream(stream);
  } else {
    if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(set_error(TRI_E_CUDA, "cannot create a CUDA stream (is a GPU visible?)"));
    d->own_stream = true;
  }
  const size_t fb = d->ncells * d->esize;
  void** fields[] = {&d->h[0], &d->h[1], &d->qx[0], &d->qx[1], &d->qy[0], &d->qy[1], &d->z, &d->n2, &d->maxh};
  for (void** f : fields) {
    cudaError_t e = cudaMalloc(f, fb + kFieldPad);
    if (e != cudaSuccess)
      return fail(set_error(e == cudaErrorMemoryAllocation ? TRI_E_NOMEM : TRI_E_CUDA, "cudaMalloc(%zu): %s", fb,
                            cudaGetErrorString(e)));
    cudaMemsetAsync(*f, 0, fb, d->stream);
  }
  d->ntr = (desc->rows + 31) / 32;
  d->ntc = (desc->cols + 31) / 32;
  if (d->prec == TRI_FP32) {
    if (cudaMalloc((void**)&d->stage, d->ncells * 8) != cudaSuccess ||
        cudaMalloc((void**)&d->zbase, (size_t)d->ntr * d->ntc * 8) != cudaSuccess)
      return fail(set_error(TRI_E_NOMEM, "cudaMalloc staging field failed"));
    cudaMemsetAsync(d->zbase, 0, (size_t)d->ntr * d->ntc * 8, d->stream);
  }
  if (cudaMalloc((void**)&d->clk, sizeof(DevClock)) != cudaSuccess ||
      cudaMallocHost((void**)&d->mirror, sizeof(DevClock)) != cudaSuccess ||
      cudaMallocHost((void**)&d->halt_host, 2 * sizeof(int32_t)) != cudaSuccess)
    return fail(set_error(TRI_E_CUDA, "clock allocation failed"));
  memset(d->mirror, 0, sizeof(DevClock));
  d->mirror->dt_key[0] = d->mirror->dt_key[1] = kDtKeyInf;
  d->mirror->cfl_a = desc->courant * desc->cell_size;
  d->mirror->sim_duration = 0;
  d->mirror->print_interval = 1e300;
  d->mirror->print_observation = 1e300;
  d->mirror->init_dt = 0.01;
  if (cudaMalloc((void**)&d->maxh_neg, sizeof(int32_t)) != cudaSuccess)
    return fail(set_error(TRI_E_CUDA, "flag allocation failed"));
  cudaMemsetAsync(d->maxh_neg, 0, sizeof(int32_t), d->stream);
  d->vol_blocks = 296;
  if (cudaMalloc((void**)&d->vol_part, d->vol_blocks * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&d->vol_out, sizeof(double)) != cudaSuccess)
    return fail(set_error(TRI_E_CUDA, "volume scratch allocation failed"));
  for (int i = 0; i < 2; i++) cudaEventCreateWithFlags(&d->chunk_ev[i], cudaEventDisableTiming);
  rc = d->prec == TRI_FP64 ? prepare_kernels<double>() : prepare_kernels<float>();
  if (rc != TRI_OK) return fail(rc);
  choose_shape(d);
  rc = push_clock(d);
  if (rc != TRI_OK) return fail(rc);
  cudaError_t e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return fail(set_error(TRI_E_CUDA, "domain init: %s", cudaGetErrorString(e)));
  *out = d;
  return TRI_OK;
}

int tri_domain_destroy(tri_domain* d) {
  if (!d) return TRI_OK;
  if (d->stream) cudaStreamSynchronize(d->stream);
  drop_graph(d);
  free_devp(d->tzero);
  free_devp(d->maxh_neg);
  for (int i = 0; i < 2; i++) {
    free_dev(d->h[i]);
    free_dev(d->qx[i]);
    free_dev(d->qy[i]);
  }
  free_dev(d->z);
  free_dev(d->n2);
  free_dev(d->maxh);
  free_devp(d->stage);
  free_devp(d->zbase);
  free_devp(d->arrival);
  free_devp(d->zone);
  free_dev(d->rates);
  free_devp(d->roff_t);
  free_devp(d->src_cells);
  free_devp(d->src_order);
  free_devp(d->hyg_t);
  free_dev(d->hyg_v);
  free_devp(d->bc_cells);
  free_devp(d->bc_types);
  free_devp(d->bc_start);
  free_devp(d->bc_nrows);
  free_devp(d->bc_order);
  free_dev(d->bc_v1);
  free_dev(d->bc_v2);
  free_devp(d->obs_cells);
  free_devp(d->obs_out);
  free_devp(d->vol_part);
  free_devp(d->vol_out);
  free_devp(d->clk);
  if (d->obs_host) cudaFreeHost(d->obs_host);
  if (d->mirror) cudaFreeHost(d->mirror);
  if (d->halt_host) cudaFreeHost(d->halt_host);
  for (cudaEvent_t e : d->tev) cudaEventDestroy(e);
  for (int i = 0; i < 2; i++)
    if (d->chunk_ev[i]) cudaEventDestroy(d->chunk_ev[i]);
  if (d->own_stream && d->stream) cudaStreamDestroy(d->stream);
  delete d;
  return TRI_OK;
}

int tri_domain_upload(tri_domain* d, int32_t field, const double* host, int64_t n) {
  TRI_CHECK_ARG(d && host, "null argument");
  TRI_CHECK_ARG(n == d->ncells, "field size %lld != rows*cols %lld", (long long)n, (long long)d->ncells);
  void* p = nullptr;
  int rc = field_ptr(d, field, &p);
  if (rc != TRI_OK) return rc;
  if (d->prec == TRI_FP64) {
    TRI_CUDA_TRY(cudaMemcpyAsync(p, host, n * 8, cudaMemcpyHostToDevice, d->stream));
  } else if (field == TRI_FIELD_DEM) {
    // base level of each 32x32 tile = its lowest interior cell
    const int R = d->desc.rows, Cc = d->desc.cols;
    TRI_CUDA_TRY(cudaMemcpyAsync(d->stage, host, n * 8, cudaMemcpyHostToDevice, d->stream));
    k_tile_base<<<dim3((unsigned)d->ntc, (unsigned)d->ntr), 256, 0, d->stream>>>(d->stage, d->zbase, R, Cc, d->ntc);
    k_bed_offsets<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(d->stage, d->zbase, (float*)p, R, Cc, d->ntc);
    TRI_CUDA_TRY(cudaGetLastError());
  } else {
    TRI_CUDA_TRY(cudaMemcpyAsync(d->stage, host, n * 8, cudaMemcpyHostToDevice, d->stream));
    k_from_f64<float><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(d->stage, (float*)p, n);
    TRI_CUDA_TRY(cudaGetLastError());
  }
  if (field == TRI_FIELD_MAXH) {  // dry bands skip the wet-dry kernel only while no max depth is negative
    TRI_CUDA_TRY(cudaMemsetAsync(d->maxh_neg, 0, sizeof(int32_t), d->stream));
    if (d->prec == TRI_FP64)
      k_flag_negative<double><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>((const double*)p, n, d->maxh_neg);
    else
      k_flag_negative<float><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>((const float*)p, n, d->maxh_neg);
    TRI_CUDA_TRY(cudaGetLastError());
  }
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (field != TRI_FIELD_MAXH && field != TRI_FIELD_NMAN2) d->dt_valid = false;
  d->tz_dirty = true;
  if (field == TRI_FIELD_H) {  // a new state restarts the volume accounts
    memset(d->mirror->acc_step, 0, sizeof(d->mirror->acc_step));
    memset(d->mirror->acc_sum, 0, sizeof(d->mirror->acc_sum));
    memset(d->mirror->acc_comp, 0, sizeof(d->mirror->acc_comp));
    int rc2 = push_clock(d);
    if (rc2 != TRI_OK) return rc2;
  }
  return TRI_OK;
}

int tri_domain_init_max_depth(tri_domain* d) {
  TRI_CHECK_ARG(d, "null domain");
  const size_t es = d->prec == TRI_FP64 ? 8 : 4;
  const int64_t n = d->ncells;
  void* h = d->h[d->mirror->cur];
  TRI_CUDA_TRY(cudaMemcpyAsync(d->maxh, h, (size_t)n * es, cudaMemcpyDeviceToDevice, d->stream));
  // dry bands skip the wet-dry kernel only while no max depth is negative
  TRI_CUDA_TRY(cudaMemsetAsync(d->maxh_neg, 0, sizeof(int32_t), d->stream));
  if (d->prec == TRI_FP64)
    k_flag_negative<double><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>((const double*)d->maxh, n,
                                                                                 d->maxh_neg);
  else
    k_flag_negative<float><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>((const float*)d->maxh, n,
                                                                               d->maxh_neg);
  TRI_CUDA_TRY(cudaGetLastError());
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->tz_dirty = true;
  return TRI_OK;
}

int tri_domain_download(tri_domain* d, int32_t field, double* host, int64_t n) {
  TRI_CHECK_ARG(d && host, "null argument");
  TRI_CHECK_ARG(n == d->ncells, "field size %lld != rows*cols %lld", (long long)n, (long long)d->ncells);
  void* p = nullptr;
  int rc = field_ptr(d, field, &p);
  if (rc != TRI_OK) return rc;
  if (d->prec == TRI_FP64) {
    TRI_CUDA_TRY(cudaMemcpyAsync(host, p, n * 8, cudaMemcpyDeviceToHost, d->stream));
  } else if (field == TRI_FIELD_DEM) {
    k_bed_levels<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>((const float*)p, d->zbase, d->stage,
                                                                     d->desc.rows, d->desc.cols, d->ntc);
    TRI_CUDA_TRY(cudaGetLastError());
    TRI_CUDA_TRY(cudaMemcpyAsync(host, d->stage, n * 8, cudaMemcpyDeviceToHost, d->stream));
  } else {
    k_to_f64<float><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>((const float*)p, d->stage, n);
    TRI_CUDA_TRY(cudaGetLastError());
    TRI_CUDA_TRY(cudaMemcpyAsync(host, d->stage, n * 8, cudaMemcpyDeviceToHost, d->stream));
  }
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  return TRI_OK;
}

int tri_domain_set_runoff(tri_domain* d, int32_t nzones, int32_t nrows, const double* times, const double* rates,
                          const int32_t* zone_of_cell, int64_t ncells) {
  TRI_CHECK_ARG(d, "null domain");
  drop_graph(d);
  d->tz_dirty = true;
  if (nzones <= 0) {
    d->nroff = 0;
    d->mirror->nroff = 0;
    return TRI_OK;
  }
  TRI_CHECK_ARG(times && rates && zone_of_cell, "null runoff table");
  TRI_CHECK_ARG(nrows >= 2, "runoff table needs at least two rows (got %d)", nrows);
  TRI_CHECK_ARG(ncells == d->ncells, "runoff map size %lld != rows*cols", (long long)ncells);
  const int R = d->desc.rows, Cc = d->desc.cols;
  for (int r = 1; r <= R - 2; r++)
    for (int c = 1; c <= Cc - 2; c++) {
      const int32_t zid = zone_of_cell[(size_t)r * Cc + c];
      TRI_CHECK_ARG(zid >= 0 && zid < nzones, "runoff zone %d at cell (%d,%d) outside [0,%d)", zid, r, c, nzones);
    }
  int rc;
  if ((rc = upload_raw(d, zone_of_cell, ncells * 4, (void**)&d->zone)) != TRI_OK) return rc;
  if ((rc = upload_raw(d, times, nrows * 8, (void**)&d->roff_t)) != TRI_OK) return rc;
  rc = d->prec == TRI_FP64 ? upload_table<double>(d, rates, (int64_t)nzones * nrows, &d->rates)
                           : upload_table<float>(d, rates, (int64_t)nzones * nrows, &d->rates);
  if (rc != TRI_OK) return rc;
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->nroff = nzones;
  d->roff_rows = nrows;
  d->mirror->nroff = nzones;
  d->mirror->roff_rows = nrows;
  d->mirror->roff_t = d->roff_t;
  return TRI_OK;
}

int tri_domain_set_sources(tri_domain* d, int32_t nsrc, const int32_t* cells, int32_t nrows, const double* times,
                           const double* flows) {
  TRI_CHECK_ARG(d, "null domain");
  drop_graph(d);
  d->tz_dirty = true;
  if (nsrc <= 0) {
    d->nsrc = 0;
    d->mirror->nsrc = 0;
    return TRI_OK;
  }
  TRI_CHECK_ARG(cells && times && flows, "null source table");
  TRI_CHECK_ARG(nrows >= 2, "hydrograph needs at least two rows (got %d)", nrows);
  const int R = d->desc.rows, Cc = d->desc.cols;
  std::vector<std::vector<int64_t>> touch(nsrc);
  for (int i = 0; i < nsrc; i++) {
    const int r = cells[i] / Cc, c = cells[i] % Cc;
    TRI_CHECK_ARG(cells[i] >= 0 && r >= 1 && r <= R - 2 && c >= 1 && c <= Cc - 2,
                  "source %d cell index %d is not an interior cell", i + 1, cells[i]);
    touch[i].push_back(cells[i]);
  }
  std::vector<int32_t> order;
  build_waves(touch, order, d->src_waves);
  d->src_order_host = order;
  int rc;
  if ((rc = upload_raw(d, cells, nsrc * 4, (void**)&d->src_cells)) != TRI_OK) return rc;
  d->src_cells_host.assign(cells, cells + nsrc);
  if ((rc = upload_raw(d, order.data(), order.size() * 4, (void**)&d->src_order)) != TRI_OK) return rc;
  if ((rc = upload_raw(d, times, nrows * 8, (void**)&d->hyg_t)) != TRI_OK) return rc;
  rc = d->prec == TRI_FP64 ? upload_table<double>(d, flows, (int64_t)nsrc * nrows, &d->hyg_v)
                           : upload_table<float>(d, flows, (int64_t)nsrc * nrows, &d->hyg_v);
  if (rc != TRI_OK) return rc;
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->nsrc = nsrc;
  d->hyg_rows = nrows;
  d->mirror->nsrc = nsrc;
  d->mirror->hyg_rows = nrows;
  d->mirror->hyg_t = d->hyg_t;
  return TRI_OK;
}

int tri_domain_set_extbc(tri_domain* d, int32_t ncells, const int32_t* cells, const int32_t* types,
                         const int32_t* start, const int32_t* nrows, int32_t nvars, const double* var1,
                         const double* var2) {
  TRI_CHECK_ARG(d, "null domain");
  drop_graph(d);
  d->tz_dirty = true;
  if (ncells <= 0) {
    d->nbc = 0;
    return TRI_OK;
  }
  TRI_CHECK_ARG(cells && types && start && nrows && var1 && var2, "null extbc table");
  const int R = d->desc.rows, Cc = d->desc.cols;
  std::vector<std::vector<int64_t>> touch(ncells);
  for (int i = 0; i < ncells; i++) {
    const int ii = cells[i];
    TRI_CHECK_ARG(ii >= 0 && ii < R * Cc, "extbc cell %d index %d outside the grid", i, ii);
    TRI_CHECK_ARG(types[i] >= 0 && types[i] <= 3, "extbc cell %d has unknown type %d", i, types[i]);
    TRI_CHECK_ARG(nrows[i] >= 1 && start[i] >= 0 && start[i] + nrows[i] <= nvars,
                  "extbc cell %d table rows [%d,%d) outside [0,%d)", i, start[i], start[i] + nrows[i], nvars);
    const int ix = ii / Cc, iy = ii % Cc;
    TRI_CHECK_ARG(ix >= 1 && ix <= R - 2 && iy >= 1 && iy <= Cc - 2, "extbc cell %d is not an interior cell", i);
    touch[i] = extbc_touches(ii, R, Cc);
  }
  std::vector<int32_t> order;
  build_waves(touch, order, d->bc_waves);
  d->bc_order_host = order;
  int rc;
  if ((rc = upload_raw(d, cells, ncells * 4, (void**)&d->bc_cells)) != TRI_OK) return rc;
  d->bc_cells_host.assign(cells, cells + ncells);
  if ((rc = upload_raw(d, types, ncells * 4, (void**)&d->bc_types)) != TRI_OK) return rc;
  if ((rc = upload_raw(d, start, ncells * 4, (void**)&d->bc_start)) != TRI_OK) return rc;
  if ((rc = upload_raw(d, nrows, ncells * 4, (void**)&d->bc_nrows)) != TRI_OK) return rc;
  if ((rc = upload_raw(d, order.data(), order.size() * 4, (void**)&d->bc_order)) != TRI_OK) return rc;
  rc = d->prec == TRI_FP64 ? upload_table<double>(d, var1, nvars, &d->bc_v1) : upload_table<float>(d, var1, nvars, &d->bc_v1);
  if (rc != TRI_OK) return rc;
  rc = d->prec == TRI_FP64 ? upload_table<double>(d, var2, nvars, &d->bc_v2) : upload_table<float>(d, var2, nvars, &d->bc_v2);
  if (rc != TRI_OK) return rc;
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->nbc = ncells;
  return TRI_OK;
}

int tri_domain_set_observations(tri_domain* d, int32_t nobs, const int32_t* cells) {
  TRI_CHECK_ARG(d, "null domain");
  free_devp(d->obs_cells);
  free_devp(d->obs_out);
  if (d->obs_host) cudaFreeHost(d->obs_host);
  d->obs_host = nullptr;
  d->nobs = 0;
  if (nobs <= 0) return TRI_OK;
  TRI_CHECK_ARG(cells, "null observation cells");
  for (int i = 0; i < nobs; i++)
    TRI_CHECK_ARG(cells[i] >= 0 && cells[i] < d->ncells, "observation %d cell index %d outside the grid", i + 1,
                  cells[i]);
  int rc = upload_raw(d, cells, nobs * 4, (void**)&d->obs_cells);
  if (rc != TRI_OK) return rc;
  TRI_CUDA_TRY(cudaMalloc((void**)&d->obs_out, 3 * nobs * sizeof(double)));
  TRI_CUDA_TRY(cudaMallocHost((void**)&d->obs_host, 3 * nobs * sizeof(double)));
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->nobs = nobs;
  return TRI_OK;
}

int tri_domain_set_clock(tri_domain* d, const tri_clock* c) {
  TRI_CHECK_ARG(d && c, "null argument");
  DevClock* m = d->mirror;
  m->simtime = c->simtime;
  m->sim_duration = c->sim_duration;
  m->print_interval = c->print_interval;
  m->print_observation = c->print_observation;
  m->last_obs_time = c->last_obs_time;
  m->init_dt = c->init_dt;
  m->time_step = c->time_step;
  m->average_dt = c->average_dt;
  m->global_dt = c->global_dt;
  m->print_id = c->print_id;
  m->it_count = c->it_count;
  m->it_print = c->it_print;
  m->time_series = c->time_series;
  m->time_increment_fixed = c->time_increment_fixed;
  m->runoff_row = c->runoff_row;
  m->src_idx_low = c->src_idx_low;
  return TRI_OK;
}

int tri_domain_get_clock(tri_domain* d, tri_clock* c) {
  TRI_CHECK_ARG(d && c, "null argument");
  const DevClock* m = d->mirror;
  c->simtime = m->simtime;
  c->sim_duration = m->sim_duration;
  c->print_interval = m->print_interval;
  c->print_observation = m->print_observation;
  c->last_obs_time = m->last_obs_time;
  c->init_dt = m->init_dt;
  c->time_step = m->time_step;
  c->average_dt = m->average_dt;
  c->global_dt = m->global_dt;
  c->print_id = m->print_id;
  c->it_count = m->it_count;
  c->it_print = m->it_print;
  c->time_series = m->time_series;
  c->time_increment_fixed = m->time_increment_fixed;
  c->runoff_row = m->runoff_row;
  c->src_idx_low = m->src_idx_low;
  c->last_events = m->events;
  return TRI_OK;
}

int tri_domain_advance(tri_domain* d, int32_t max_steps, tri_progress* p) {
  TRI_CHECK_ARG(d && p, "null argument");
  TRI_CHECK_ARG(max_steps >= 0, "max_steps must be >= 0");
  p->steps = 0;
  p->events = 0;
  DevClock* m = d->mirror;
  if (!(m->simtime < m->sim_duration)) {
    p->events = TRI_EV_END;
    return TRI_OK;
  }
  if (max_steps == 0) return TRI_OK;
  TRI_CHECK_ARG(d->nroff == 0 || (m->runoff_row >= 0 && m->runoff_row < d->roff_rows),
                "runoff_row %d outside the runoff table [0,%d)", m->runoff_row, d->roff_rows);
  TRI_CHECK_ARG(d->nsrc == 0 || (m->src_idx_low >= 0 && m->src_idx_low < d->hyg_rows),
                "src_idx_low %d outside the hydrograph [0,%d)", m->src_idx_low, d->hyg_rows);
  TRI_CHECK_ARG(m->print_interval > 0, "print_interval must be positive");
  m->halt = 0;
  m->events = 0;
  m->steps = 0;
  m->status = 0;
  const bool need_dt = !d->dt_valid && !m->time_increment_fixed;
  if (need_dt) m->dt_key[m->rd] = kDtKeyInf;
  int rc = push_clock(d);
  if (rc != TRI_OK) return rc;
  if (need_dt) {
    rc = launch_dt(d);
    if (rc != TRI_OK) return rc;
  }
  d->dt_valid = true;
  if (d->tz_dirty) {
    rc = reset_tiles(d);
    if (rc != TRI_OK) return rc;
  }
  // Chunks of steps, two in flight: after launching chunk k the host waits
  // for chunk k-1 and stops launching once a step has raised an event.
  const int chunk = 8;
  int left = max_steps, k = 0;
  bool halted = false;
  while (left > 0 && !halted) {
    const int n = std::min(chunk, left);
    rc = launch_steps(d, n);
    if (rc != TRI_OK) return rc;
    TRI_CUDA_TRY(cudaMemcpyAsync(&d->halt_host[k & 1], &d->clk->halt, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                 d->stream));
    TRI_CUDA_TRY(cudaEventRecord(d->chunk_ev[k & 1], d->stream));
    left -= n;
    if (k > 0) {
      TRI_CUDA_TRY(cudaEventSynchronize(d->chunk_ev[(k - 1) & 1]));
      if (d->halt_host[(k - 1) & 1]) halted = true;
    }
    k++;
  }
  rc = pull_clock(d);
  if (rc != TRI_OK) return rc;
  p->steps = m->steps;
  p->events = m->events;
  d->work_steps += m->steps;
  if (m->status != 0)
    return set_error(TRI_E_TIMEOUT, "a device-side wait gave up during the last advance (status %d); the state "
                     "of this domain is not valid", m->status);
  return TRI_OK;
}

int tri_domain_compute_dt(tri_domain* d, double* local_dt) {
  TRI_CHECK_ARG(d && local_dt, "null argument");
  DevClock* m = d->mirror;
  m->dt_key[m->rd] = kDtKeyInf;
  int rc = push_clock(d);
  if (rc != TRI_OK) return rc;
  rc = launch_dt(d);
  if (rc != TRI_OK) return rc;
  rc = pull_clock(d);
  if (rc != TRI_OK) return rc;
  d->dt_valid = true;
  *local_dt = dt_of_key(m->dt_key[m->rd], m->cfl_a);
  return TRI_OK;
}

int tri_domain_observe(tri_domain* d, double* h, double* qx, double* qy) {
  TRI_CHECK_ARG(d, "null domain");
  if (d->nobs == 0) return TRI_OK;
  if (d->prec == TRI_FP64)
    k_observe<double><<<(d->nobs + 127) / 128, 128, 0, d->stream>>>(d->clk, bufs<double>(d), d->obs_cells, d->nobs,
                                                                     d->obs_out);
  else
    k_observe<float><<<(d->nobs + 127) / 128, 128, 0, d->stream>>>(d->clk, bufs<float>(d), d->obs_cells, d->nobs,
                                                                   d->obs_out);
  TRI_CUDA_TRY(cudaGetLastError());
  TRI_CUDA_TRY(cudaMemcpyAsync(d->obs_host, d->obs_out, 3 * d->nobs * sizeof(double), cudaMemcpyDeviceToHost,
                               d->stream));
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (h) memcpy(h, d->obs_host, d->nobs * sizeof(double));
  if (qx) memcpy(qx, d->obs_host + d->nobs, d->nobs * sizeof(double));
  if (qy) memcpy(qy, d->obs_host + 2 * d->nobs, d->nobs * sizeof(double));
  return TRI_OK;
}

int tri_domain_volume(tri_domain* d, double* volume) {
  TRI_CHECK_ARG(d && volume, "null argument");
  const double dx = d->desc.cell_size;
  if (d->prec == TRI_FP64)
    k_volume_part<double><<<d->vol_blocks, 256, 0, d->stream>>>(d->clk, bufs<double>(d), d->desc.rows, d->desc.cols,
                                                                d->vol_part);
  else
    k_volume_part<float><<<d->vol_blocks, 256, 0, d->stream>>>(d->clk, bufs<float>(d), d->desc.rows, d->desc.cols,
                                                               d->vol_part);
  k_volume_sum<<<1, 32, 0, d->stream>>>(d->vol_part, d->vol_blocks, dx * dx, d->vol_out);
  TRI_CUDA_TRY(cudaGetLastError());
  TRI_CUDA_TRY(cudaMemcpyAsync(volume, d->vol_out, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  return TRI_OK;
}

int tri_domain_autotune(tri_domain* d, int32_t trial_steps, tri_tuning* out) {
  TRI_CHECK_ARG(d && out, "null argument");
  TRI_CHECK_ARG(trial_steps >= 1, "trial_steps must be >= 1");
  DevClock* m = d->mirror;
  const DevClock saved = *m;
  const bool saved_valid = d->dt_valid;
  const int cur = m->cur;
  const size_t fb = d->ncells * d->esize;
  // back up the current state and max depth
  void* bak = nullptr;
  TRI_CUDA_TRY(cudaMalloc(&bak, 4 * fb));
  char* b = (char*)bak;
  auto save_restore = [&](bool save) -> int {
    void* f[4] = {d->h[cur], d->qx[cur], d->qy[cur], d->maxh};
    for (int i = 0; i < 4; i++) {
      if (save)
        TRI_CUDA_TRY(cudaMemcpyAsync(b + i * fb, f[i], fb, cudaMemcpyDeviceToDevice, d->stream));
      else
        TRI_CUDA_TRY(cudaMemcpyAsync(f[i], b + i * fb, fb, cudaMemcpyDeviceToDevice, d->stream));
    }
    return TRI_OK;
  };
  int rc = save_restore(true);
  const int heights[3] = {8, 16, 32};
  double best = 1e300;
  int best_v = d->flux_variant, best_rb = d->rb, ncand = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const bool timing = d->timing;
  d->timing = false;
  for (int v = 0; v < kFluxVariants && rc == TRI_OK; v++) {
    for (int hi = 0; hi < 3 && rc == TRI_OK; hi++) {
      if (heights[hi] > std::max(8, d->desc.rows - 2)) continue;
      d->flux_variant = v;
      d->rb = heights[hi];
      size_flux_grid(d);
      drop_graph(d);
      rc = save_restore(false);
      if (rc == TRI_OK) rc = reset_tiles(d);  // the other buffer holds the last trial's state
      if (rc != TRI_OK) break;
      *m = saved;
      m->sim_duration = m->print_interval = m->print_observation = 1e300;
      m->it_print = 0;
      m->time_series = 0;
      m->halt = 0;
      m->dt_key[m->rd] = kDtKeyInf;
      rc = push_clock(d);
      if (rc == TRI_OK) rc = launch_dt(d);
      if (rc == TRI_OK) rc = launch_steps(d, 2);  // warm-up (also builds the graph)
      cudaEventRecord(e0, d->stream);
      if (rc == TRI_OK) rc = launch_steps(d, trial_steps);
      cudaEventRecord(e1, d->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = set_error(TRI_E_CUDA, "autotune trial failed");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      ncand++;
      if (rc == TRI_OK && ms / trial_steps < best) {
        best = ms / trial_steps;
        best_v = v;
        best_rb = heights[hi];
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  d->timing = timing;
  d->flux_variant = best_v;
  d->rb = best_rb;
  size_flux_grid(d);
  drop_graph(d);
  int rc2 = save_restore(false);
  *m = saved;
  d->dt_valid = saved_valid;
  d->tz_dirty = true;
  if (rc2 == TRI_OK) rc2 = push_clock(d);
  cudaStreamSynchronize(d->stream);
  cudaFree(bak);
  if (rc != TRI_OK) return rc;
  if (rc2 != TRI_OK) return rc2;
  d->tuned_ms = best;
  return tri_domain_get_tuning(d, out);
}

int tri_domain_get_tuning(tri_domain* d, tri_tuning* out) {
  TRI_CHECK_ARG(d && out, "null argument");
  out->variant = d->flux_variant;
  out->rows_per_tile = d->rb;
  out->candidates = kFluxVariants * 3;
  out->flux_blocks = d->flux_blocks;
  out->ms_per_step = d->tuned_ms;
  return TRI_OK;
}

int tri_domain_set_tuning(tri_domain* d, int32_t variant, int32_t rows_per_tile) {
  TRI_CHECK_ARG(d, "null domain");
  TRI_CHECK_ARG(variant >= 0 && variant < kFluxVariants, "variant %d outside [0,%d)", variant, kFluxVariants);
  TRI_CHECK_ARG(rows_per_tile >= 1, "rows_per_tile must be >= 1");
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->flux_variant = variant;
  d->rb = rows_per_tile;
  size_flux_grid(d);
  drop_graph(d);
  d->tz_dirty = true;
  return TRI_OK;
}

int tri_domain_mass_balance(tri_domain* d, double* out) {
  TRI_CHECK_ARG(d && out, "null argument");
  int rc = pull_clock(d);
  if (rc != TRI_OK) return rc;
  double vol = 0;
  rc = tri_domain_volume(d, &vol);
  if (rc != TRI_OK) return rc;
  const double a = d->desc.cell_size * d->desc.cell_size;
  out[0] = vol;
  for (int k = 0; k < kAccTerms; k++) out[1 + k] = d->mirror->acc_sum[k] * a;
  return TRI_OK;
}

int tri_domain_set_wait_test(tri_domain* d, uint32_t polls) {
  TRI_CHECK_ARG(d, "null domain");
  d->mirror->wait_test = polls;  // reaches the device with the clock at the next advance
  return TRI_OK;
}

int tri_domain_track_arrival(tri_domain* d, double depth) {
  TRI_CHECK_ARG(d, "null domain");
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (!d->arrival) TRI_CUDA_TRY(cudaMalloc((void**)&d->arrival, d->ncells * sizeof(float)));
  std::vector<float> inf((size_t)d->ncells, 3.402823466e38f);
  TRI_CUDA_TRY(cudaMemcpy(d->arrival, inf.data(), d->ncells * sizeof(float), cudaMemcpyHostToDevice));
  d->arrival_depth = (float)depth;
  drop_graph(d);
  return TRI_OK;
}

int tri_domain_download_arrival(tri_domain* d, double* host, int64_t n) {
  TRI_CHECK_ARG(d && host, "null argument");
  TRI_CHECK_ARG(d->arrival, "arrival tracking is not enabled");
  TRI_CHECK_ARG(n == d->ncells, "size %lld != rows*cols", (long long)n);
  std::vector<float> tmp((size_t)n);
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  TRI_CUDA_TRY(cudaMemcpy(tmp.data(), d->arrival, n * sizeof(float), cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < n; i++) host[i] = tmp[i] >= 3.0e38f ? -1.0 : (double)tmp[i];
  return TRI_OK;
}

int tri_domain_synchronize(tri_domain* d) {
  TRI_CHECK_ARG(d, "null domain");
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  return TRI_OK;
}

int tri_domain_set_timing(tri_domain* d, int32_t enabled) {
  TRI_CHECK_ARG(d, "null domain");
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->timing = enabled != 0;
  d->tev_used = 0;
  memset(d->mirror->skipped, 0, sizeof(d->mirror->skipped));  // sent with the clock at the next advance
  d->work_steps = 0;
  return TRI_OK;
}

int tri_domain_get_work(tri_domain* d, int64_t* flux_cells, int64_t* wetdry_cells) {
  TRI_CHECK_ARG(d, "null domain");
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  const int64_t all = d->work_steps * (int64_t)(d->desc.rows - 2) * (d->desc.cols - 2);
  int64_t sk[2] = {0, 0};
  for (int k = 0; k < 2; k++)
    for (int i = 0; i < kSkipSlots; i++) sk[k] += (int64_t)d->mirror->skipped[k][i];
  if (flux_cells) *flux_cells = all - sk[0];
  if (wetdry_cells) *wetdry_cells = all - sk[1];
  return TRI_OK;
}

int tri_domain_get_timing(tri_domain* d, double* flux_ms, int32_t* flux_launches, double* wetdry_ms,
                          int32_t* wetdry_launches) {
  TRI_CHECK_ARG(d, "null domain");
  TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  double fa = 0, wa = 0;
  for (size_t i = 0; i + 3 < d->tev_used; i += 4) {
    float a = 0, b = 0;
    TRI_CUDA_TRY(cudaEventElapsedTime(&a, d->tev[i], d->tev[i + 1]));
    TRI_CUDA_TRY(cudaEventElapsedTime(&b, d->tev[i + 2], d->tev[i + 3]));
    fa += a;
    wa += b;
  }
  if (flux_ms) *flux_ms = fa;
  if (flux_launches) *flux_launches = (int32_t)(d->tev_used / 4);
  if (wetdry_ms) *wetdry_ms = wa;
  if (wetdry_launches) *wetdry_launches = (int32_t)(d->tev_used / 4);
  return TRI_OK;
}

}  // extern "C"
