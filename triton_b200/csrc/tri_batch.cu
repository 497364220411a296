// tri_batch.cu -- tri_batch_*: ensembles of member domains advanced together.
//
// The reference runs ensemble members as separate MPI rank groups (Ensify,
// src/Ensify.h:43-72), one process group per member.  Here every member is a
// tri_domain on one GPU and a batched step advances each member by one of its
// own time steps with one launch per kernel type: a clock kernel over the
// member table (per-member dt policy and events), one flux kernel whose warps
// take tiles from a single queue over all members' tiles (uneven sizes pack
// without idle SMs), the sparse forcing in conflict-free waves of (member,
// item) pairs, and one wet-dry/dt kernel over all members' bands, each member
// folding its own dt minimum.  Steps are launched as CUDA graphs of 8 batched
// steps; the host checks after each graph how many members have halted.  In
// single-launch mode (tri_batch_set_mode) one persistent launch of
// k_batch_steps runs a chunk of 32 batched steps instead: its blocks take the
// same work items from a ticket counter and wait, bounded, only for their own
// member's earlier items.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "tri_domain_impl.h"
#include "tri_internal.h"
#include "tri_step_launch.h"

using namespace tri;

struct tri_batch {
  int prec = TRI_FP64;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<tri_domain*> members;
  void* d_mem = nullptr;
  int32_t* d_tile_mem = nullptr;  // member of every flux tile
  int32_t* d_wet_mem = nullptr;   // member of every wet-dry block
  BatchCtl* d_ctl = nullptr;
  BatchCtl* h_ctl = nullptr;  // pinned
  int32_t* h_seen = nullptr;  // pinned, one per chunk slot
  uint32_t ntiles = 0, nwet = 0;
  int rb = 8, variant = 1, flux_blocks = 1;
  int2* d_src_items = nullptr;
  std::vector<int32_t> src_waves;
  int2* d_bc_items = nullptr;
  std::vector<int32_t> bc_waves;
  int32_t* d_open = nullptr;  // members with open edges
  int n_open = 0, open_dim = 0;
  // single-launch mode (TRI_BATCH_SINGLE_LAUNCH): progress counters per
  // member, the members' forcing wave offsets, resident grid
  int mode = TRI_BATCH_GRAPHS;
  MemberProgress* d_prog = nullptr;
  int32_t* d_woff = nullptr;
  int steps_grid = 0;
  uint32_t wait_test = 0;  // tri_batch_set_wait_test
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  double tuned_ms = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool launched = false;  // tri_batch_launch without its tri_batch_wait yet
};

namespace {

template <typename T>
MemberDev<T> member_dev(tri_domain* d, int rb, uint32_t& tiles, uint32_t& wet) {
  const StepArgs a = domain_step_args(d);
  MemberDev<T> m{};
  m.clk = d->clk;
  for (int i = 0; i < 2; i++) {
    m.sb.h[i] = (T*)a.h[i];
    m.sb.qx[i] = (T*)a.qx[i];
    m.sb.qy[i] = (T*)a.qy[i];
  }
  m.bed.z = (const T*)a.z;
  m.bed.base = a.zbase;
  m.bed.ntc = a.ntc;
  m.n2 = (const T*)a.n2;
  m.zone = a.zone;
  m.rates = (const T*)a.rates;
  m.maxh = (T*)a.maxh;
  m.arrival = a.arrival;
  m.arrival_depth = a.arrival_depth;
  m.rows = a.rows;
  m.cols = a.cols;
  m.rb = rb;
  m.dx = (T)a.dx;
  m.rdx = (T)(1.0 / a.dx);
  m.hextra = (T)a.hextra;
  m.dxd = a.dx;
  m.courant = a.courant;
  const uint32_t strips = (uint32_t)((a.cols - 2 + kStripCols - 1) / kStripCols);
  const uint32_t rowb = (uint32_t)((a.rows - 2 + rb - 1) / rb);
  m.tile_begin = tiles;
  tiles += strips * rowb;
  m.tile_end = tiles;
  m.wet_nbx = (uint32_t)((a.cols + kWetCols - 1) / kWetCols);
  m.wet_begin = wet;
  wet += m.wet_nbx * (uint32_t)((a.rows + kStageBand<T> - 1) / kStageBand<T>);
  m.nsrc = a.nsrc;
  m.src_cells = a.src_cells;
  m.hyg_t = a.hyg_t;
  m.hyg_v = (const T*)a.hyg_v;
  m.bc_cells = a.bc_cells;
  m.bc_types = a.bc_types;
  m.bc_start = a.bc_start;
  m.bc_nrows = a.bc_nrows;
  m.bc_v1 = (const T*)a.bc_v1;
  m.bc_v2 = (const T*)a.bc_v2;
  m.wet_count = wet - m.wet_begin;
  m.src_order = d->nsrc > 0 ? d->src_order : nullptr;
  m.src_nw = d->nsrc > 0 ? (int)d->src_waves.size() - 1 : 0;
  m.bc_order = d->nbc > 0 ? d->bc_order : nullptr;
  m.bc_nw = d->nbc > 0 ? (int)d->bc_waves.size() - 1 : 0;
  m.open = d->desc.open_boundaries ? 1 : 0;
  m.src_woff = m.bc_woff = nullptr;  // set once the offsets are on the device
  return m;
}

void drop_graph(tri_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_steps = 0;
}

// Member table, tile and block counts, grid of the flux kernel.
template <typename T>
int build_table(tri_batch* b) {
  std::vector<MemberDev<T>> tab;
  uint32_t tiles = 0, wet = 0;
  for (tri_domain* d : b->members) tab.push_back(member_dev<T>(d, b->rb, tiles, wet));
  b->ntiles = tiles;
  b->nwet = wet;
  for (void** p : {&b->d_mem, (void**)&b->d_tile_mem, (void**)&b->d_wet_mem, (void**)&b->d_prog,
                   (void**)&b->d_woff}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  drop_graph(b);
  if (tab.empty()) return TRI_OK;
  // single-launch mode: every member's wave offsets in one buffer, progress counters
  std::vector<int32_t> woff;
  std::vector<std::pair<size_t, size_t>> at(tab.size());
  for (size_t m = 0; m < tab.size(); m++) {
    const tri_domain* d = b->members[m];
    at[m].first = woff.size();
    if (tab[m].src_nw > 0) woff.insert(woff.end(), d->src_waves.begin(), d->src_waves.end());
    at[m].second = woff.size();
    if (tab[m].bc_nw > 0) woff.insert(woff.end(), d->bc_waves.begin(), d->bc_waves.end());
  }
  TRI_CUDA_TRY(cudaMalloc((void**)&b->d_woff, std::max<size_t>(woff.size(), 1) * sizeof(int32_t)));
  if (!woff.empty())
    TRI_CUDA_TRY(cudaMemcpy(b->d_woff, woff.data(), woff.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  for (size_t m = 0; m < tab.size(); m++) {
    tab[m].src_woff = b->d_woff + at[m].first;
    tab[m].bc_woff = b->d_woff + at[m].second;
  }
  TRI_CUDA_TRY(cudaMalloc((void**)&b->d_prog, tab.size() * sizeof(MemberProgress)));
  b->steps_grid = batch_steps_grid<T>(b->variant);
  std::vector<int32_t> tm(tiles), wm(wet);
  for (size_t m = 0; m < tab.size(); m++) {
    std::fill(tm.begin() + tab[m].tile_begin, tm.begin() + tab[m].tile_end, (int32_t)m);
    const uint32_t w1 = m + 1 < tab.size() ? tab[m + 1].wet_begin : wet;
    std::fill(wm.begin() + tab[m].wet_begin, wm.begin() + w1, (int32_t)m);
  }
  TRI_CUDA_TRY(cudaMalloc(&b->d_mem, tab.size() * sizeof(MemberDev<T>)));
  TRI_CUDA_TRY(cudaMemcpy(b->d_mem, tab.data(), tab.size() * sizeof(MemberDev<T>), cudaMemcpyHostToDevice));
  TRI_CUDA_TRY(cudaMalloc(&b->d_tile_mem, std::max<size_t>(tm.size(), 1) * sizeof(int32_t)));
  TRI_CUDA_TRY(cudaMemcpy(b->d_tile_mem, tm.data(), tm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  TRI_CUDA_TRY(cudaMalloc(&b->d_wet_mem, std::max<size_t>(wm.size(), 1) * sizeof(int32_t)));
  TRI_CUDA_TRY(cudaMemcpy(b->d_wet_mem, wm.data(), wm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  int sms = 148, dev = 0, per_sm = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  batch_flux_occupancy<T>(b->variant, &per_sm);
  if (per_sm < 1) per_sm = 1;
  b->flux_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, (tiles + 3) / 4));
  drop_graph(b);
  return TRI_OK;
}

int rebuild(tri_batch* b) { return b->prec == TRI_FP64 ? build_table<double>(b) : build_table<float>(b); }

// (member, item) pairs of every member's conflict-free waves, wave by wave.
int build_items(tri_batch* b) {
  auto gather = [&](bool src, int2** dptr, std::vector<int32_t>& waves) -> int {
    std::vector<std::vector<int2>> per;
    for (size_t m = 0; m < b->members.size(); m++) {
      tri_domain* d = b->members[m];
      const std::vector<int32_t>& w = src ? d->src_waves : d->bc_waves;
      const std::vector<int32_t>& o = src ? d->src_order_host : d->bc_order_host;
      const int n = src ? d->nsrc : d->nbc;
      if (n <= 0 || w.size() < 2) continue;
      for (size_t k = 0; k + 1 < w.size(); k++) {
        if (per.size() <= k) per.resize(k + 1);
        for (int j = w[k]; j < w[k + 1]; j++) per[k].push_back(make_int2((int)m, o[j]));
      }
    }
    std::vector<int2> flat;
    waves.assign(1, 0);
    for (auto& v : per) {
      flat.insert(flat.end(), v.begin(), v.end());
      waves.push_back((int32_t)flat.size());
    }
    if (*dptr) cudaFree(*dptr);
    *dptr = nullptr;
    if (!flat.empty()) {
      TRI_CUDA_TRY(cudaMalloc((void**)dptr, flat.size() * sizeof(int2)));
      TRI_CUDA_TRY(cudaMemcpy(*dptr, flat.data(), flat.size() * sizeof(int2), cudaMemcpyHostToDevice));
    }
    return TRI_OK;
  };
  int rc = gather(true, &b->d_src_items, b->src_waves);
  if (rc == TRI_OK) rc = gather(false, &b->d_bc_items, b->bc_waves);
  if (rc != TRI_OK) return rc;
  // open-boundary members: ghost copies after the sources, before the
  // external-boundary cells, as in the single-domain step
  std::vector<int32_t> open;
  b->open_dim = 0;
  for (size_t m = 0; m < b->members.size(); m++) {
    const tri_grid_desc& g = b->members[m]->desc;
    if (!g.open_boundaries) continue;
    open.push_back((int32_t)m);
    b->open_dim = std::max(b->open_dim, std::max(g.rows, g.cols));
  }
  if (b->d_open) cudaFree(b->d_open);
  b->d_open = nullptr;
  b->n_open = (int)open.size();
  if (!open.empty()) {
    TRI_CUDA_TRY(cudaMalloc((void**)&b->d_open, open.size() * sizeof(int32_t)));
    TRI_CUDA_TRY(cudaMemcpy(b->d_open, open.data(), open.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  return TRI_OK;
}

BatchArgs batch_args(tri_batch* b) {
  BatchArgs a{};
  a.mem = b->d_mem;
  a.nm = (int)b->members.size();
  a.tile_member = b->d_tile_mem;
  a.wet_member = b->d_wet_mem;
  a.ctl = b->d_ctl;
  a.ntiles = b->ntiles;
  a.nwet_blocks = b->nwet;
  a.flux_blocks = b->flux_blocks;
  a.flux_variant = b->variant;
  a.src_items = b->d_src_items;
  a.src_waves = b->src_waves.data();
  a.n_src_waves = (int)b->src_waves.size() - 1;
  a.bc_items = b->d_bc_items;
  a.bc_waves = b->bc_waves.data();
  a.n_bc_waves = (int)b->bc_waves.size() - 1;
  a.open_members = b->d_open;
  a.n_open = b->n_open;
  a.open_dim = b->open_dim;
  return a;
}

// Single-launch mode: n batched steps in launches of k_batch_steps, each
// with fresh progress counters and ticket (tickets of one launch stay below
// 2^31); the status word is cleared once, so a timeout in any launch of the
// chunk reaches the host.
int launch_batch_single(tri_batch* b, int n) {
  const BatchArgs a = batch_args(b);
  const uint64_t per_step = 2ull * (uint64_t)a.nm + (a.ntiles + 3) / 4 + a.nwet_blocks;
  const int max_steps = (int)std::max<uint64_t>(1, std::min<uint64_t>(1u << 20, (1ull << 31) / per_step));
  TRI_CUDA_TRY(cudaMemsetAsync(&b->d_ctl->status, 0, sizeof(int32_t), b->stream));
  while (n > 0) {
    const int k = std::min(n, max_steps);
    TRI_CUDA_TRY(cudaMemsetAsync(b->d_prog, 0, b->members.size() * sizeof(MemberProgress), b->stream));
    TRI_CUDA_TRY(cudaMemsetAsync(&b->d_ctl->ticket, 0, sizeof(uint32_t), b->stream));
    const int rc = b->prec == TRI_FP64 ? launch_batch_steps<double>(a, b->d_prog, k, b->steps_grid, b->stream)
                                       : launch_batch_steps<float>(a, b->d_prog, k, b->steps_grid, b->stream);
    if (rc != TRI_OK) return rc;
    n -= k;
  }
  return TRI_OK;
}

int launch_batch(tri_batch* b, int n) {
  if (b->mode == TRI_BATCH_SINGLE_LAUNCH) return launch_batch_single(b, n);
  const BatchArgs a = batch_args(b);
  auto one = [&]() {
    return b->prec == TRI_FP64 ? launch_batch_step<double>(a, b->stream) : launch_batch_step<float>(a, b->stream);
  };
  const int G = 8;
  if (!b->graph) {
    cudaGraph_t g = nullptr;
    TRI_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = TRI_OK;
    for (int i = 0; i < G && rc == TRI_OK; i++) rc = one();
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc != TRI_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return set_error(TRI_E_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_error(TRI_E_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
    b->graph_steps = G;
  }
  while (n >= b->graph_steps) {
    TRI_CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
    n -= b->graph_steps;
  }
  for (int i = 0; i < n; i++) {
    int rc = one();
    if (rc != TRI_OK) return rc;
  }
  return TRI_OK;
}

// Prepares every member's clock for a batched advance (members at or past
// their end stay halted for the whole call); counts the members that step.
// Clocks go to the device on the batch stream, ahead of the batched launches;
// a member without a valid CFL dt (new, or state uploaded) gets it first on
// its own stream.
int prepare_members(tri_batch* b, int* runnable) {
  *runnable = 0;
  for (tri_domain* d : b->members) {
    DevClock* m = d->mirror;
    d->tz_dirty = true;  // batched steps keep no dry-tile flags
    const bool live = m->simtime < m->sim_duration;
    m->halt = live ? 0 : 1;
    m->events = 0;
    m->steps = 0;
    m->status = 0;
    const bool need_dt = live && !d->dt_valid && !m->time_increment_fixed;
    if (need_dt) {
      m->dt_key[m->rd] = kDtKeyInf;
      int rc = domain_push_clock(d);
      if (rc == TRI_OK) rc = domain_launch_dt(d);
      if (rc != TRI_OK) return rc;
      TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
      d->dt_valid = true;
    } else {
      TRI_CUDA_TRY(cudaMemcpyAsync(d->clk, d->mirror, sizeof(DevClock), cudaMemcpyHostToDevice, b->stream));
    }
    if (live) (*runnable)++;
  }
  return TRI_OK;
}

// Reads every member's clock back (one stream synchronization) and sums the
// progress of the advance.
int pull_members(tri_batch* b, tri_batch_progress* p) {
  memset(p, 0, sizeof(*p));
  for (tri_domain* d : b->members)
    TRI_CUDA_TRY(cudaMemcpyAsync(d->mirror, d->clk, sizeof(DevClock), cudaMemcpyDeviceToHost, b->stream));
  b->h_ctl->status = 0;
  TRI_CUDA_TRY(cudaMemcpyAsync(&b->h_ctl->status, &b->d_ctl->status, sizeof(int32_t), cudaMemcpyDeviceToHost,
                               b->stream));
  TRI_CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (b->h_ctl->status != 0)
    return set_error(TRI_E_TIMEOUT, "a dependency wait of the single-launch batch kernel gave up (status %d); the "
                     "members' states are not valid", b->h_ctl->status);
  int64_t updates = 0;
  for (tri_domain* d : b->members) {
    const DevClock* m = d->mirror;
    p->steps = std::max(p->steps, m->steps);
    if (m->events) p->members_with_events++;
    if (!(m->simtime < m->sim_duration)) p->members_ended++;
    updates += (int64_t)m->steps * (int64_t)(d->desc.rows - 2) * (int64_t)(d->desc.cols - 2);
  }
  p->cell_updates = updates;
  for (tri_domain* d : b->members)
    if (d->mirror->status != 0)
      return set_error(TRI_E_TIMEOUT, "a device-side wait gave up during the last batched advance (status %d)",
                       d->mirror->status);
  return TRI_OK;
}

int reset_ctl(tri_batch* b) {
  b->h_ctl->halted = 0;
  b->h_ctl->tile_next = 0;
  b->h_ctl->ticket = 0;
  b->h_ctl->status = 0;
  b->h_ctl->wait_test = b->wait_test;
  TRI_CUDA_TRY(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, b->stream));
  return TRI_OK;
}

// Members of one batch: existing, distinct, one precision.
int check_members(int prec, int32_t n, tri_domain* const* members, std::vector<tri_domain*>& out) {
  out.clear();
  for (int i = 0; i < n; i++) {
    tri_domain* d = members[i];
    if (!d || d->prec != prec)
      return set_error(TRI_E_INVALID, "batch member %d: members must exist and share one precision", i);
    for (int j = 0; j < i; j++)
      if (members[j] == d) return set_error(TRI_E_INVALID, "batch member %d repeats member %d", i, j);
    out.push_back(d);
  }
  return TRI_OK;
}

}  // namespace

extern "C" {

int tri_batch_create(int32_t nmembers, tri_domain* const* members, void* stream, tri_batch** out) {
  TRI_CHECK_ARG(out && members && nmembers >= 1 && members[0], "need at least one member");
  *out = nullptr;
  tri_batch* b = new tri_batch();
  b->prec = members[0]->prec;
  {
    const int rc0 = check_members(b->prec, nmembers, members, b->members);
    if (rc0 != TRI_OK) {
      delete b;
      return rc0;
    }
  }
  int rc = TRI_OK;
  auto fail = [&](int code) {
    tri_batch_destroy(b);
    return code;
  };
  if (stream) {
    b->stream = as_stream(stream);
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(set_error(TRI_E_CUDA, "cannot create a CUDA stream"));
    b->own_stream = true;
  }
  if (cudaMalloc((void**)&b->d_ctl, sizeof(BatchCtl)) != cudaSuccess ||
      cudaMallocHost((void**)&b->h_ctl, sizeof(BatchCtl)) != cudaSuccess ||
      cudaMallocHost((void**)&b->h_seen, 2 * sizeof(int32_t)) != cudaSuccess)
    return fail(set_error(TRI_E_CUDA, "batch control allocation failed"));
  cudaEventCreateWithFlags(&b->ev[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&b->ev[1], cudaEventDisableTiming);
  // the members' own streams must be idle before the batch uses their memory
  for (tri_domain* d : b->members) cudaStreamSynchronize(d->stream);
  if ((rc = rebuild(b)) != TRI_OK) return fail(rc);
  if ((rc = build_items(b)) != TRI_OK) return fail(rc);
  *out = b;
  return TRI_OK;
}

int tri_batch_destroy(tri_batch* b) {
  if (!b) return TRI_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  if (b->d_mem) cudaFree(b->d_mem);
  if (b->d_tile_mem) cudaFree(b->d_tile_mem);
  if (b->d_wet_mem) cudaFree(b->d_wet_mem);
  if (b->d_ctl) cudaFree(b->d_ctl);
  if (b->h_ctl) cudaFreeHost(b->h_ctl);
  if (b->h_seen) cudaFreeHost(b->h_seen);
  if (b->d_src_items) cudaFree(b->d_src_items);
  if (b->d_bc_items) cudaFree(b->d_bc_items);
  if (b->d_open) cudaFree(b->d_open);
  if (b->d_prog) cudaFree(b->d_prog);
  if (b->d_woff) cudaFree(b->d_woff);
  for (int i = 0; i < 2; i++)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return TRI_OK;
}

int tri_batch_set_members(tri_batch* b, int32_t nmembers, tri_domain* const* members) {
  TRI_CHECK_ARG(b && nmembers >= 0 && (nmembers == 0 || members), "null argument");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  std::vector<tri_domain*> next;
  int rc = check_members(b->prec, nmembers, members, next);
  if (rc != TRI_OK) return rc;
  TRI_CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (tri_domain* d : next) TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
  b->members = std::move(next);
  if ((rc = rebuild(b)) != TRI_OK) return rc;
  return build_items(b);
}

int tri_batch_advance(tri_batch* b, int32_t max_steps, tri_batch_progress* p) {
  TRI_CHECK_ARG(b && p, "null argument");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  TRI_CHECK_ARG(max_steps >= 0, "max_steps must be >= 0");
  int runnable = 0;
  int rc = prepare_members(b, &runnable);
  if (rc != TRI_OK) return rc;
  if (runnable > 0 && max_steps > 0) {
    if ((rc = reset_ctl(b)) != TRI_OK) return rc;
    // chunks of 8 batched steps (32 in single-launch mode), two in flight;
    // stop once every runnable member has raised an event
    const int chunk = b->mode == TRI_BATCH_SINGLE_LAUNCH ? 32 : 8;
    int left = max_steps, k = 0;
    bool done = false;
    while (left > 0 && !done) {
      const int n = std::min(chunk, left);
      rc = launch_batch(b, n);
      if (rc != TRI_OK) return rc;
      TRI_CUDA_TRY(cudaMemcpyAsync(&b->h_seen[k & 1], &b->d_ctl->halted, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   b->stream));
      TRI_CUDA_TRY(cudaEventRecord(b->ev[k & 1], b->stream));
      left -= n;
      if (k > 0) {
        TRI_CUDA_TRY(cudaEventSynchronize(b->ev[(k - 1) & 1]));
        if (b->h_seen[(k - 1) & 1] >= runnable) done = true;
      }
      k++;
    }
  }
  return pull_members(b, p);
}

int tri_batch_launch(tri_batch* b, int32_t steps) {
  TRI_CHECK_ARG(b, "null batch");
  TRI_CHECK_ARG(steps >= 0, "steps must be >= 0");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  int runnable = 0;
  int rc = prepare_members(b, &runnable);
  if (rc != TRI_OK) return rc;
  if (runnable > 0 && steps > 0) {
    if ((rc = reset_ctl(b)) != TRI_OK) return rc;
    if ((rc = launch_batch(b, steps)) != TRI_OK) return rc;
  }
  b->launched = true;
  return TRI_OK;
}

int tri_batch_wait(tri_batch* b, tri_batch_progress* p) {
  TRI_CHECK_ARG(b && p, "null argument");
  b->launched = false;
  return pull_members(b, p);
}

int tri_batch_set_mode(tri_batch* b, int32_t mode) {
  TRI_CHECK_ARG(b, "null batch");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  TRI_CHECK_ARG(mode == TRI_BATCH_GRAPHS || mode == TRI_BATCH_SINGLE_LAUNCH, "unknown batch mode %d", mode);
  b->mode = mode;
  return TRI_OK;
}

int tri_batch_set_wait_test(tri_batch* b, uint32_t polls) {
  TRI_CHECK_ARG(b, "null batch");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  b->wait_test = polls;
  return TRI_OK;
}

int tri_batch_set_tuning(tri_batch* b, int32_t variant, int32_t rows_per_tile) {
  TRI_CHECK_ARG(b, "null batch");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  TRI_CHECK_ARG(variant >= 0 && variant < kFluxVariants, "variant %d outside [0,%d)", variant, kFluxVariants);
  TRI_CHECK_ARG(rows_per_tile >= 1, "rows_per_tile must be >= 1");
  TRI_CUDA_TRY(cudaStreamSynchronize(b->stream));
  b->variant = variant;
  b->rb = rows_per_tile;
  return rebuild(b);
}

int tri_batch_autotune(tri_batch* b, int32_t trial_steps, tri_tuning* out) {
  TRI_CHECK_ARG(b && out, "null argument");
  if (b->launched) return set_error(TRI_E_STATE, "batch has launched steps; call tri_batch_wait first");
  TRI_CHECK_ARG(!b->members.empty(), "autotune needs at least one member");
  TRI_CHECK_ARG(trial_steps >= 1, "trial_steps must be >= 1");
  // snapshot every member: current state, max depth and clock
  struct Snap {
    void* buf = nullptr;
    DevClock clk;
    bool valid = false;
  };
  std::vector<Snap> snaps(b->members.size());
  int rc = TRI_OK;
  for (size_t i = 0; i < b->members.size() && rc == TRI_OK; i++) {
    tri_domain* d = b->members[i];
    const size_t fb = d->ncells * d->esize;
    if (cudaMalloc(&snaps[i].buf, 4 * fb) != cudaSuccess) {
      rc = set_error(TRI_E_NOMEM, "autotune snapshot allocation failed");
      break;
    }
    const int cur = d->mirror->cur;
    void* f[4] = {d->h[cur], d->qx[cur], d->qy[cur], d->maxh};
    for (int k = 0; k < 4; k++) cudaMemcpy((char*)snaps[i].buf + k * fb, f[k], fb, cudaMemcpyDeviceToDevice);
    snaps[i].clk = *d->mirror;
    snaps[i].valid = d->dt_valid;
  }
  auto restore = [&]() -> int {
    for (size_t i = 0; i < b->members.size(); i++) {
      tri_domain* d = b->members[i];
      const size_t fb = d->ncells * d->esize;
      *d->mirror = snaps[i].clk;
      d->dt_valid = snaps[i].valid;
      const int cur = d->mirror->cur;
      void* f[4] = {d->h[cur], d->qx[cur], d->qy[cur], d->maxh};
      for (int k = 0; k < 4; k++)
        TRI_CUDA_TRY(cudaMemcpy(f[k], (char*)snaps[i].buf + k * fb, fb, cudaMemcpyDeviceToDevice));
      int r = domain_push_clock(d);
      if (r != TRI_OK) return r;
      TRI_CUDA_TRY(cudaStreamSynchronize(d->stream));
    }
    return TRI_OK;
  };
  const int heights[3] = {4, 8, 16};
  double best = 1e300;
  int best_v = b->variant, best_rb = b->rb, ncand = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int v = 0; v < kFluxVariants && rc == TRI_OK; v++) {
    for (int hi = 0; hi < 3 && rc == TRI_OK; hi++) {
      b->variant = v;
      b->rb = heights[hi];
      rc = rebuild(b);
      if (rc == TRI_OK) rc = restore();
      for (tri_domain* d : b->members) {  // trials run without events
        d->mirror->sim_duration = d->mirror->print_interval = d->mirror->print_observation = 1e300;
        d->mirror->it_print = 0;
        d->mirror->time_series = 0;
      }
      int runnable = 0;
      if (rc == TRI_OK) rc = prepare_members(b, &runnable);
      if (rc == TRI_OK) rc = reset_ctl(b);
      if (rc == TRI_OK) rc = launch_batch(b, 2);  // warm-up, also builds the graph
      cudaEventRecord(e0, b->stream);
      if (rc == TRI_OK) rc = launch_batch(b, trial_steps);
      cudaEventRecord(e1, b->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess && rc == TRI_OK)
        rc = set_error(TRI_E_CUDA, "batch autotune trial failed");
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
  b->variant = best_v;
  b->rb = best_rb;
  int rc2 = rebuild(b);
  if (rc2 == TRI_OK && snaps.size() && snaps.back().buf) rc2 = restore();
  for (Snap& s : snaps)
    if (s.buf) cudaFree(s.buf);
  if (rc != TRI_OK) return rc;
  if (rc2 != TRI_OK) return rc2;
  b->tuned_ms = best;
  out->variant = b->variant;
  out->rows_per_tile = b->rb;
  out->candidates = ncand;
  out->flux_blocks = b->flux_blocks;
  out->ms_per_step = best;
  return TRI_OK;
}

}  // extern "C"
