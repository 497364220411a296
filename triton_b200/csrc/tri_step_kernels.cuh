// tri_step_kernels.cuh -- the fused time-step kernels of the domain path.
//
// One time step of the reference (triton_simulate.h:191-346) becomes, on the
// domain's stream:
//   k_clock         1 thread: dt policy (compute_global_dt :202-226), runoff
//                   row and hydrograph bracket (:246-285), step events
//   k_flux_update   fluxes + conserved update + Manning friction + runoff
//                   (kernels_flux.h, kernels_state.h, kernels.h:103-152)
//   k_sources       point inflows (kernels.h:51-84), only with sources
//   k_open_bc       open-boundary ghosts (kernels.h:437-512), only if open
//   k_extbc         external boundary cells (kernels.h:237-424), only with extbc
//   k_wetdry_dt     wet/dry masks + max depth (kernels_wetdry.h:25-93) fused
//                   with the NEXT step's CFL dt and its min reduction
//                   (kernels.h:167-212)
// Every kernel reads the step's parameters from the device clock, so a
// sequence of steps needs no host round trip and can be captured in a graph.
#pragma once

#include "tri_common.cuh"
#include "tri_bulk.cuh"
#include "tri_face.cuh"
#include "tri_step_launch.h"
#include "tri_types.cuh"

namespace tri {

template <typename T>
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// k_clock: the per-step scalar work of the reference host loop.
// ---------------------------------------------------------------------------
// Returns true when this step raised an event (the domain halts after it).
__device__ __forceinline__ bool clock_step(DevClock* __restrict__ c) {
  if (c->halt) {
    c->active = 0;
    return false;
  }
  const double t0 = c->simtime;
  double dt;
  if (!c->time_increment_fixed) {
    // compute_global_dt: dry fallback, then clamp to the next print time
    dt = dt_of_key(c->dt_key[c->rd], c->cfl_a);
    if (dt >= kMaxValue - 1.0) dt = c->init_dt;
    const double tp = c->print_interval * (c->print_id + 1);
    if (t0 + dt > tp) dt = tp - t0;
  } else {
    dt = c->time_step;
  }
  c->global_dt = dt;
  c->rdt = 1.0 / dt;
  c->t_step = t0;
  c->it_count++;
  if (c->nroff > 0) {
    const int last = c->roff_rows - 1;
    if (t0 > c->roff_t[last]) {
      c->runoff_row = last;
    } else if (c->runoff_row + 1 <= last && t0 > c->roff_t[c->runoff_row + 1]) {
      c->runoff_row++;
    }
  }
  if (c->nsrc > 0) {
    int lo = c->src_idx_low, hi = c->hyg_rows - 1;
    bool found = false;
    for (int i = lo; i < hi; i++) {
      if (c->hyg_t[i + 1] > t0) {
        lo = i;
        hi = i + 1;
        found = true;
        break;
      }
    }
    if (!found) lo = hi;
    c->src_idx_low = lo;
    c->src_idx_high = hi;
  }
  c->tile_next = 0;
  c->src = c->cur;
  c->dst = c->cur ^ 1;
  c->cur = c->dst;
  c->wr = c->rd ^ 1;
  c->dt_key[c->wr] = kDtKeyInf;
  c->rd = c->wr;
  const double t1 = t0 + dt;
  c->simtime = t1;
  c->average_dt += dt;
  c->steps++;
  int ev = 0;
  if (c->it_print > 0 && c->it_count % c->it_print == 0) ev |= TRI_EV_LOG;
  if (c->time_series && t1 - c->last_obs_time >= c->print_observation) ev |= TRI_EV_OBS;
  if (t1 >= c->print_interval * (c->print_id + 1)) ev |= TRI_EV_PRINT;
  if (!(t1 < c->sim_duration)) ev |= TRI_EV_END;
  c->active = 1;
  if (ev) {
    c->halt = 1;
    c->events = ev;
    return true;
  }
  return false;
}

static __global__ void k_clock(DevClock* __restrict__ c) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x == 0) clock_step(c);
}

// ---------------------------------------------------------------------------
// k_flux_update: fluxes + conserved update + friction + runoff.
//
// Work unit: a tile of one warp = a strip of 30 interior columns and rb rows.
// Lane l holds column c = c0-1+l: lanes 1..30 own interior columns, lanes 0
// and 31 are the west/east halo columns.  The warp marches down its rows
// keeping the previous row in registers, so every x face and y face of the
// strip is evaluated once (plus one halo y row per tile and one halo x face
// per row); neighbours are exchanged with shuffles, there is no block-level
// synchronisation.  Warps fetch tiles from a per-step counter (the dry part of
// a domain costs far less than the wet part, so static tiling leaves SMs idle).
//   y face (r, r-1): owner row r, north neighbour row r-1 (kernels_flux.h:359-360)
//   x face (c-1, c): owner column c-1, east neighbour c   (kernels_flux.h:76-77)
// A row's update runs once its south face (computed with the next row) is
// known: h = hn - (xE+yN) - (xW+yS), i.e. hn - rhsh0 - rhsh1 with the
// reference's rhs0 = flux_x part + flux_y part (kernels_state.h:65).
// Ghost cells are copied from the source to the destination buffer so both
// ping-pong buffers keep the boundary state the reference keeps in place.
// ---------------------------------------------------------------------------
// rhs contributions collected for one cell before its south face is known.
// The owner parts of its east and north faces are summed at once, in the
// reference's order (flux_x writes rhs*0, flux_y adds to it):
// r = e + n; the west face's neighbour part w waits for the south face's s
// (rhs*1 = w + s).  Six values carried per lane instead of nine.
template <typename T>
struct RowParts {
  T r0, r1, r2;  // east + north owner parts
  T w0, w1, w2;  // west face, neighbour part (flux_x rhs*1)
  T an;          // FP32 form: |e0| + |n0|, for the noise test of the depth update
};

template <typename T>
__device__ __forceinline__ void update_cell(const CellQ<T>& c, const RowParts<T>& p, T s0, T s1, T s2, T n2v, T dt,
                                            T hextra, T& ho, T& qxo, T& qyo, double& clip, uint32_t rnd) {
  const T E12 = eps12<T>();
  const T G = T(kGravity);
  const T hn = c.h;
  T hij;
  if (sizeof(T) == 8) {
    const T rh1 = p.w0 + s0;
    hij = hn - p.r0 - rh1;
    clip = hij < T(0) ? -(double)hij : 0.0;
  } else {
    // FP32 form: the depth change is summed in FP64 and rounded
    // stochastically (unbiased).  Rounded to nearest, a deep cell drops every
    // inflow below half its ulp while the thin cell it came from loses it
    // exactly, so runoff draining from films into channels would vanish
    // (1.4e-5 of the volume over 2 h of rain on a 2048^2 watershed).  A
    // result within the rounding noise of its terms is zero, as FP32
    // arithmetic would give it: noise must not leave water on a cell that
    // drained, or the cell counts as wet.
    const float parts = p.r0 + (p.w0 + s0);
    float lo;
    const float hs = sr_add(hn, -parts, rnd, &lo);
    const float noise = float(kNoise32) * (hn + p.an + dev_fabs(p.w0) + dev_fabs(s0));
    if (__fadd_rn(hn, -parts) <= noise) {
      clip = -((double)__fadd_rn(hn, -parts) + (double)lo);  // removed (noise) or clipped to zero: accounted
      hij = T(0);
    } else {
      clip = 0.0;
      hij = hs;
    }
  }
  T qxij, qyij;
  if (hij < T(0)) hij = T(0);
  if (hij < hextra) {
    qxij = T(0);
    qyij = T(0);
  } else {
    const T rx1 = p.w1 + s1;
    const T ry1 = p.w2 + s2;
    const T mx = c.qx - p.r1 - rx1;
    const T my = c.qy - p.r2 - ry1;
    const T modM = dev_sqrt(mx * mx + my * my);
    if (n2v > E12 && hn >= hextra && modM > E12) {
      const T tt = fdiv(dt * G * n2v * modM, hn * hn * dev_cbrt(hn));
      const T sq = dev_sqrt(T(1) + T(4) * tt);
      if (sizeof(T) == 8) {  // the reference's expression (kernels_state.h:86-96), bit for bit
        const T rtt = recip(tt);
        qxij = div_shared(T(-0.5) * (mx - mx * sq), tt, rtt);
        qyij = div_shared(T(-0.5) * (my - my * sq), tt, rtt);
      } else {
        // FP32 form: -(m - m*s)/(2t) with s = sqrt(1 + 4t) equals
        // 2m/(1 + s), without the cancellation of 1 - s: where t is small
        // (deep, fast channel flow) 1 - s keeps only a few FP32 bits, and the
        // rounding of s alone moved the friction-corrected discharge by up to
        // 1e-3 of itself each step, one way (the 512^2 6 h watershed then
        // ponded up to 0.97 m away from the FP64 run).
        const T k = recip(T(1) + sq);
        qxij = T(2) * mx * k;
        qyij = T(2) * my * k;
      }
    } else {
      qxij = mx;
      qyij = my;
    }
  }
  ho = hij;
  qxo = qxij;
  qyo = qyij;
}

template <typename T>
__device__ __forceinline__ T shfl_up1(T v) {
  return __shfl_up_sync(0xffffffffu, v, 1);
}
template <typename T>
__device__ __forceinline__ T shfl_down1(T v) {
  return __shfl_down_sync(0xffffffffu, v, 1);
}


// Everything one tile of the flux kernel needs: the domain's arrays and the
// running step's constants (from its clock).
template <typename T>
struct FluxCtx {
  DevClock* clk;
  const T* hi;
  const T* qxi;
  const T* qyi;
  T* ho;
  T* qxo;
  T* qyo;
  BedMap<T> bed;
  const T* n2;
  const int32_t* zone;
  const T* rates;
  int rows, cols, rb, nstrips;
  int nroff, roff_rows, roff_row;
  uint32_t step;  // it_count of the running step (seeds the FP32 form's rounding of runoff)
  StepK<T> K;
  // Dry-tile skipping (null: every tile is computed).  tz_src[t] / tz_dst[t]:
  // tile t of the source / destination buffer holds only zero bits in h, qx
  // and qy; tpin[t]: tile t is never skipped (a later kernel of the step
  // writes into it: sources, external boundary cells, open boundaries).
  const uint8_t* tz_src;
  uint8_t* tz_dst;
  const uint8_t* tpin;
};

template <typename T>
__device__ __forceinline__ FluxCtx<T> flux_ctx(DevClock* clk, const StateBufs<T>& sb, const BedMap<T>& bed,
                                               const T* n2, const int32_t* zone, const T* rates, int rows, int cols,
                                               int rb, T dx, T rdx, T hextra) {
  FluxCtx<T> X;
  X.clk = clk;
  const int src = clk->src, dst = clk->dst;
  X.hi = sb.H(src);
  X.qxi = sb.QX(src);
  X.qyi = sb.QY(src);
  X.ho = sb.H(dst);
  X.qxo = sb.QX(dst);
  X.qyo = sb.QY(dst);
  X.bed = bed;
  X.n2 = n2;
  X.zone = zone;
  X.rates = rates;
  X.rows = rows;
  X.cols = cols;
  X.rb = rb;
  X.nstrips = (cols - 2 + kStripCols - 1) / kStripCols;
  X.nroff = clk->nroff;
  X.roff_rows = clk->roff_rows;
  X.roff_row = clk->runoff_row;
  X.step = (uint32_t)clk->it_count;
  X.K = step_k<T>(dx, T(clk->global_dt), rdx, T(clk->rdt), hextra);
  X.tz_src = nullptr;
  X.tz_dst = nullptr;
  X.tpin = nullptr;
  return X;
}

// Zero bits (+0): a tile is skipped only where every value it would write
// is +0 already, so skipping is exact.
__device__ __forceinline__ bool nonzero_bits(double v) { return __double_as_longlong(v) != 0; }
__device__ __forceinline__ bool nonzero_bits(float v) { return __float_as_uint(v) != 0u; }

// A tile whose cells and whose four neighbour tiles' cells hold only +0 in
// the source buffer computes exactly +0 everywhere (every face is dry-dry and
// contributes nothing; no runoff on such a domain), and if its cells in the
// destination buffer hold +0 already (it was all-zero two steps ago), it has
// nothing to write.  Called by lane 0, which takes the tiles.
template <typename T>
__device__ __forceinline__ bool tile_skippable(const FluxCtx<T>& X, unsigned tile) {
  if (X.tz_src == nullptr) return false;
  const int ns = X.nstrips, nty = (X.rows - 2 + X.rb - 1) / X.rb;
  const int sx = (int)(tile % ns), ry = (int)(tile / ns);
  if (!(X.tz_src[tile] & X.tz_dst[tile]) || X.tpin[tile]) return false;
  if (sx > 0 && !X.tz_src[tile - 1]) return false;
  if (sx < ns - 1 && !X.tz_src[tile + 1]) return false;
  if (ry > 0 && !X.tz_src[tile - ns]) return false;
  if (ry < nty - 1 && !X.tz_src[tile + ns]) return false;
  return true;
}

// The same pointer, opaque to the compiler: values read through it cannot be
// taken from an earlier read through the original.
template <typename P>
__device__ __forceinline__ const P* launder_ptr(const P* p) {
  const P* q;
  asm volatile("mov.b64 %0, %1;" : "=l"(q) : "l"(p));
  return q;
}

// One warp tile: strip sx (30 interior columns), rows r0..r1.  kTrack:
// record in X.tz_dst whether the tile wrote only +0 (dry-tile skipping; the
// kernels of domains that cannot skip are built without it).  kReload: the
// context (in shared memory) is read again every row, where each value is
// used, instead of being held in registers across the row loop; the batched
// kernels' member parameters are not kernel parameters, and holding them
// spilled (FP32 batched ensemble at 8 blocks per SM: 252 bytes of spill
// stores, 20 with the reads; 25.5 against 23.8 G cell-updates/s at the best
// launch shape).  The single-domain kernel keeps kReload off: its context
// comes from kernel parameters, which the compiler reads at each use.
template <typename T, bool kTrack, bool kReload = false>
__device__ __forceinline__ void flux_tile(const FluxCtx<T>& X0, unsigned tile, int lane) {
  const FluxCtx<T>& X = kReload ? *launder_ptr(&X0) : X0;
  const int rows = X.rows, cols = X.cols, rb = X.rb;
  const T hextra = X.K.hextra;
  const int sx = (int)(tile % X.nstrips), ry = (int)(tile / X.nstrips);
  const int c = sx * kStripCols + lane;  // = c0 - 1 + lane with c0 = 1 + 30*sx
  const int r0 = 1 + ry * rb;
  const int r1 = min(r0 + rb - 1, rows - 2);
  const bool incol = c < cols;
  const bool mid = (lane >= 1 && lane <= kStripCols);
  const bool upd = mid && c >= 1 && c <= cols - 2;
  const bool gcol = incol && (c == 0 || c == cols - 1);  // ghost column owned by this lane
  const bool owner = incol && (mid || gcol);
  constexpr bool kAcct = true;  // FP64 volume accounts in both forms
  double acc_b = 0.0, acc_r = 0.0, acc_c = 0.0;
  const double sxq = (double)X.K.dt / (double)X.K.dx;  // dt/dx of the boundary discharges

  bool wrote_nonzero = false;  // any value this lane writes is not +0
  auto copy_ghost = [&](const FluxCtx<T>& Z, int r) {
    const T* __restrict__ hi = Z.hi;
    const T* __restrict__ qxi = Z.qxi;
    const T* __restrict__ qyi = Z.qyi;
    T* __restrict__ ho = Z.ho;
    T* __restrict__ qxo = Z.qxo;
    T* __restrict__ qyo = Z.qyo;
    const size_t id = (size_t)r * Z.cols + c;
    if (kTrack) {
      const T gh = hi[id];
      ho[id] = gh;
      const T gqx = qxi[id];
      qxo[id] = gqx;
      const T gqy = qyi[id];
      qyo[id] = gqy;
      wrote_nonzero |= nonzero_bits(gh) | nonzero_bits(gqx) | nonzero_bits(gqy);
    } else {
      ho[id] = hi[id];
      qxo[id] = qxi[id];
      qyo[id] = qyi[id];
    }
  };

  // raw values of the next row are loaded one iteration ahead
  T lh = T(0), lqx = T(0), lqy = T(0), lz = T(0);
  double lzb = 0.0;
  auto fetch = [&](const FluxCtx<T>& Z, int r) {
    if (incol) {
      const size_t id = (size_t)r * Z.cols + c;
      lh = Z.hi[id];
      lqx = Z.qxi[id];
      lqy = Z.qyi[id];
      lz = Z.bed.z[id];  // FP32 form: the offset from the base of the cell's tile
      lzb = Z.bed.base_at(r, c);
    }
  };
  fetch(X, r0 - 1);
  CellQ<T> prev = make_cell<T>(lh, lqx, lqy, lz, hextra, lzb);
  if (r0 - 1 == 0 && owner) copy_ghost(X, 0);
  fetch(X, r0);
  RowParts<T> pp;
  pp.r0 = pp.r1 = pp.r2 = pp.w0 = pp.w1 = pp.w2 = pp.an = T(0);
  T pn2 = T(0);  // Manning of the previous row's cell

  for (int r = r0; r <= r1 + 1; ++r) {
    // the context is read where it is used, so with kReload none of it is
    // held across the face computations
    const FluxCtx<T>& XL = kReload ? *launder_ptr(&X0) : X0;
    const CellQ<T> cur = make_cell<T>(lh, lqx, lqy, lz, XL.K.hextra, lzb);
    T cn2 = T(0);
    if (r <= r1) {
      if (upd) cn2 = XL.n2[(size_t)r * XL.cols + c];
      fetch(XL, r + 1);  // r1 + 1 <= rows - 1
    }
    FaceOut<T> Y;
    Y.a0 = Y.a1 = Y.a2 = Y.b0 = Y.b1 = Y.b2 = T(0);
    if (upd) Y = face_flux<T, false>(cur, prev, XL.K);
    if (r - 1 >= r0 && upd) {
      const FluxCtx<T>& XU = kReload ? *launder_ptr(&X0) : X0;
      const int cols = XU.cols;
      const T dt = XU.K.dt, hextra = XU.K.hextra;
      const size_t id = (size_t)(r - 1) * cols + c;
      T hn, qn, vn;
      double clip;
      update_cell<T>(prev, pp, Y.b0, Y.b1, Y.b2, pn2, dt, hextra, hn, qn, vn, clip,
                     cell_hash((uint32_t)id, 2u * XU.step));
      if (kAcct) {
        // Inflow through the south face of a cell of the last interior row
        // (the other boundary faces are counted where their parts are
        // formed, below), and the depth the update clipped back to zero.
        if (r - 1 == XU.rows - 2) acc_b += sxq * (double)prev.qy - (double)Y.b0;
        acc_c += clip;
      }
      if (XU.nroff > 0) {  // update_runoff (kernels.h:128-149)
        const T h0 = hn;
        const T net = XU.rates[(size_t)XU.zone[id] * XU.roff_rows + XU.roff_row];
        if (sizeof(T) == 8) {
          hn += net * dt;
        } else if (net != T(0)) {
          // FP32 form: uniform rain adds the same increment to every cell of
          // a zone, so rounding h + r*dt to nearest would round the same way
          // in every cell of a binade; the FP64 sum is rounded
          // stochastically instead (unbiased), deterministic in (cell, step)
          float lo;
          hn = sr_add(hn, net * dt, cell_hash((uint32_t)id, 2u * XU.step + 1u), &lo);
        }
        if (hn < hextra) {
          if (hn < T(0)) hn = T(0);
          qn = T(0);
          vn = T(0);
        }
        if (kAcct) acc_r += (double)hn - (double)h0;
      }
      T* __restrict__ ho = XU.ho;
      T* __restrict__ qxo = XU.qxo;
      T* __restrict__ qyo = XU.qyo;
      ho[id] = hn;
      qxo[id] = qn;
      qyo[id] = vn;
      if (kTrack) wrote_nonzero |= nonzero_bits(hn) | nonzero_bits(qn) | nonzero_bits(vn);
    }
    if (r > r1) {
      if (r == XL.rows - 1 && owner) copy_ghost(XL, r);
      break;
    }
    // x faces of row r: lane l evaluates the face between lanes l-1 and l
    CellQ<T> left;
    left.h = shfl_up1(cur.h);
    left.qx = shfl_up1(cur.qx);
    left.qy = shfl_up1(cur.qy);
    left.z = shfl_up1(cur.z);
    left.sq = shfl_up1(cur.sq);
    left.u = shfl_up1(cur.u);
    left.v = shfl_up1(cur.v);
    left.zb = sizeof(T) == 4 ? __shfl_up_sync(0xffffffffu, cur.zb, 1) : 0.0;
    FaceOut<T> Xf;
    Xf.a0 = Xf.a1 = Xf.a2 = Xf.b0 = Xf.b1 = Xf.b2 = T(0);
    if (lane >= 1 && incol && c >= 1) Xf = face_flux<T, true>(left, cur, XL.K);
    const T e0 = shfl_down1(Xf.a0), e1 = shfl_down1(Xf.a1), e2 = shfl_down1(Xf.a2);
    if (kAcct && upd) {
      // Inflow through faces shared with ghost cells, in depth units.  The
      // update is in fluctuation form, so the mass flux through a face of
      // boundary cell i is F(Q_i).n plus the fluctuation it receives there:
      // west / south faces dt/dx*q - b, east / north faces -(a + dt/dx*q).
      if (c == 1) acc_b += sxq * (double)cur.qx - (double)Xf.b0;
      if (c == XL.cols - 2) acc_b -= (double)e0 + sxq * (double)cur.qx;
      if (r == 1) acc_b -= (double)Y.a0 + sxq * (double)cur.qy;
    }
    pp.r0 = e0 + Y.a0;
    pp.r1 = e1 + Y.a1;
    pp.r2 = e2 + Y.a2;
    pp.w0 = Xf.b0;
    pp.w1 = Xf.b1;
    pp.w2 = Xf.b2;
    if (sizeof(T) == 4) pp.an = dev_fabs(e0) + dev_fabs(Y.a0);
    pn2 = cn2;
    if (gcol) copy_ghost(XL, r);
    prev = cur;
  }
  if (kAcct) {
    acc_b = warp_sum<T>(acc_b);
    acc_r = warp_sum<T>(acc_r);
    acc_c = warp_sum<T>(acc_c);
    if (lane == 0) {
      if (acc_b != 0.0) atomicAdd(&X.clk->acc_step[kAccBoundary], acc_b);
      if (acc_r != 0.0) atomicAdd(&X.clk->acc_step[kAccRunoff], acc_r);
      if (acc_c != 0.0) atomicAdd(&X.clk->acc_step[kAccClip], acc_c);
    }
  }
  if (kTrack) {
    const bool nz = __any_sync(0xffffffffu, wrote_nonzero);
    if (lane == 0) X.tz_dst[tile] = (!nz && !X.tpin[tile]) ? 1 : 0;
  }
}

// kSkip: the domain keeps dry-tile flags (tzero) and skips dry tiles.
template <typename T, int MINB, bool kSkip>
__global__ void __launch_bounds__(128, MINB) k_flux_update(DevClock* __restrict__ clk, StateBufs<T> sb,
                                                     const BedMap<T> bed, const T* __restrict__ n2,
                                                     const int32_t* __restrict__ zone, const T* __restrict__ rates,
                                                     int rows, int cols, int rb, T dx, T rdx, T hextra,
                                                     uint8_t* __restrict__ tzero) {
  pdl_wait();
  if (!clk->active) return;
  FluxCtx<T> X = flux_ctx<T>(clk, sb, bed, n2, zone, rates, rows, cols, rb, dx, rdx, hextra);
  const int lane = threadIdx.x & 31;
  const unsigned ntiles = (unsigned)X.nstrips * (unsigned)((rows - 2 + rb - 1) / rb);
  if (kSkip) {  // [2][ntiles] zero flags by buffer, then [ntiles] pinned
    X.tz_src = tzero + (size_t)clk->src * ntiles;
    X.tz_dst = tzero + (size_t)clk->dst * ntiles;
    X.tpin = tzero + 2 * (size_t)ntiles;
  }
  unsigned skipped = 0;  // interior cells of the tiles this warp skipped (lane 0)
  while (true) {
    unsigned tile = 0;  // lane 0 takes the next tile; bit 31: skip it (tiles < 2^31)
    if (lane == 0) {
      tile = atomicAdd(&clk->tile_next, 1u);
      if (kSkip && tile < ntiles && tile_skippable<T>(X, tile)) {
        const int sx = (int)(tile % X.nstrips), r0 = 1 + (int)(tile / X.nstrips) * rb;
        skipped += (unsigned)((min(r0 + rb - 1, rows - 2) - r0 + 1) * min(kStripCols, cols - 2 - sx * kStripCols));
        tile |= 0x80000000u;
      }
    }
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((tile & 0x7FFFFFFFu) >= ntiles) break;
    if (kSkip && (tile >> 31)) continue;
    flux_tile<T, kSkip>(X, tile, lane);
  }
  pdl_trigger();  // no tile left for this warp
  if (kSkip && lane == 0 && skipped)  // spread over the slots: one address would serialize the atomics
    atomicAdd(&clk->skipped[0][(blockIdx.x * 4 + (threadIdx.x >> 5)) % kSkipSlots], (unsigned long long)skipped);
}

// ---------------------------------------------------------------------------
// Sparse kernels (run on the destination buffer after k_flux_update).
// 'order' lists the items of one conflict-free wave; items that touch the
// same cell are in different waves, launched in the reference's index order.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_sources(DevClock* __restrict__ clk, StateBufs<T> sb, const int32_t* __restrict__ order,
                          int count, int nsrc, const int32_t* __restrict__ cells, const double* __restrict__ hyg_t,
                          const T* __restrict__ hyg_v, T dx) {
  pdl_wait();
  pdl_trigger();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count || !clk->active) return;
  const int id = order[k];
  const int lo = clk->src_idx_low, hi = clk->src_idx_high;
  const T dt = T(clk->global_dt);
  const T simtime = T(clk->t_step);
  T* h = sb.H(clk->dst);
  const T flo = hyg_v[(size_t)lo * nsrc + id];
  const T fhi = hyg_v[(size_t)hi * nsrc + id];
  const T tlo = T(hyg_t[lo]), thi = T(hyg_t[hi]);
  T flow;
  if (lo == hi) {
    flow = flo;
  } else {
    const T td = simtime - tlo;
    const T td2 = thi - tlo;
    flow = flo + (((fhi - flo) * td) / td2);
  }
  const int sid = cells[id];
  T hij = h[sid];
  const T hs = (flow * dt) / (dx * dx);
  hij += hs;
  h[sid] = hij;
  atomicAdd(&clk->acc_step[kAccSources], (double)hs);
}

// Final values of copy_info_to_exterior_boundaries_west_east followed by
// _north_south (kernels.h:437-512), item k of max(rows, cols): ghost columns
// take the adjacent interior column (rows 1..rows-2), ghost rows take the
// adjacent interior row, corners the diagonal interior cell.
template <typename T>
__device__ __forceinline__ void open_bc_item(const DevClock* __restrict__ clk, const StateBufs<T>& sb, int rows,
                                             int cols, int k) {
  const int d = clk->dst;
  T* h = sb.H(d);
  T* qx = sb.QX(d);
  T* qy = sb.QY(d);
  auto cp = [&](size_t g, size_t i) {
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
  };
  if (k < rows) {
    const int r = k;
    if (r >= 1 && r <= rows - 2) {
      cp((size_t)r * cols, (size_t)r * cols + 1);
      cp((size_t)r * cols + cols - 1, (size_t)r * cols + cols - 2);
    }
  }
  if (k < cols) {
    const int cc = k;
    const int ci = cc == 0 ? 1 : (cc == cols - 1 ? cols - 2 : cc);
    cp((size_t)cc, (size_t)cols + ci);
    cp((size_t)(rows - 1) * cols + cc, (size_t)(rows - 2) * cols + ci);
  }
}

template <typename T>
__global__ void k_open_bc(const DevClock* __restrict__ clk, StateBufs<T> sb, int rows, int cols) {
  pdl_wait();
  pdl_trigger();
  if (!clk->active) return;
  open_bc_item<T>(clk, sb, rows, cols, blockIdx.x * blockDim.x + threadIdx.x);
}

// compute_extbc_values for one boundary cell (kernels.h:254-420), single rank.
template <typename T>
__device__ __forceinline__ void extbc_apply(DevClock* __restrict__ clk, const StateBufs<T>& sb, const BedMap<T>& bed,
                                            const T* __restrict__ n2, int id, const int32_t* __restrict__ cells,
                                            const int32_t* __restrict__ types, const int32_t* __restrict__ start,
                                            const int32_t* __restrict__ nrowsv, const T* __restrict__ var1,
                                            const T* __restrict__ var2, int rows, int cols) {
  const int d = clk->dst;
  T* h = sb.H(d);
  T* qx = sb.QX(d);
  T* qy = sb.QY(d);
  const T dt = T(clk->global_dt);
  const T simtime = T(clk->t_step);
  const int ii = cells[id];
  const int bt = types[id];
  const int s0 = start[id];
  const int ix = ii / cols, iy = ii % cols;
  const bool top = (ix == 1), btm = (ix == rows - 2), lt = (iy == 1), rt = (iy == cols - 2);
  if (!(top || lt || rt || btm)) return;
  bool corner = false;
  int ib = ii, ibc = ii;
  T f0 = T(1), f1 = T(0), f2 = T(0);
  if (lt) {
    ib = ii - 1;
    f1 = T(-1);
    f2 = T(0);
  }
  if (rt) {
    ib = ii + 1;
    f1 = T(1);
    f2 = T(0);
  }
  if (top) {
    ib = ii - cols;
    f1 = T(0);
    f2 = T(1);
    if (lt) {
      corner = true;
      ibc = ii - 1;
      f2 = T(0);
    }
    if (rt) {
      corner = true;
      ibc = ii + 1;
      f2 = T(0);
    }
  }
  if (btm) {
    ib = ii + cols;
    f1 = T(0);
    f2 = T(-1);
    if (lt) {
      corner = true;
      ibc = ii - 1;
      f2 = T(0);
    }
    if (rt) {
      corner = true;
      ibc = ii + 1;
      f2 = T(0);
    }
  }
  T hij = h[ii], qxij = qx[ii], qyij = qy[ii];
  if (bt == 0) {
    h[ib] = hij;
    qx[ib] = qxij;
    qy[ib] = qyij;
    if (corner) {
      h[ibc] = hij;
      qx[ibc] = qxij;
      qy[ibc] = qyij;
    }
    return;
  }
  if (bt == 1) {
    const T lvar = T(0.5) * (simtime + simtime + dt);
    int lo = 0, hi = nrowsv[id] - 1;
    if (lvar < var1[s0]) {
      lo = 0;
      hi = 0;
    } else if (lvar > var1[hi + s0]) {
      lo = hi;
    } else {
      lo = 0;  // a non-monotone table leaves the reference's index unset; clamp to row 0
      for (int i = 0; i < hi; i++) {
        if (var1[i + s0] <= lvar && var1[i + 1 + s0] > lvar) {
          lo = i;
          hi = i + 1;
          break;
        }
      }
    }
    T aux;
    if (lo == hi) {
      aux = var2[lo + s0];
    } else {
      const T td = lvar - var1[lo + s0];
      const T td2 = var1[hi + s0] - var1[lo + s0];
      aux = var2[lo + s0] + (((var2[hi + s0] - var2[lo + s0]) * td) / td2);
    }
    if (sizeof(T) == 8) {
      hij = dev_fmax(aux - (T)bed.absolute(ii, ix, iy), T(0));
    } else {  // FP32 form: level minus bed in FP64, then rounded
      hij = (T)fmax((double)aux - bed.absolute(ii, ix, iy), 0.0);
    }
    atomicAdd(&clk->acc_step[kAccExtbc], (double)hij - (double)h[ii]);
  } else {
    const T aux = var1[s0];
    T vel = T(0);
    if (bt == 2) vel = dev_sqrt(aux * hij * dev_cbrt(hij) / dev_fmax(n2[ii], T(1e-6)));
    if (bt == 3) vel = aux * dev_sqrt(T(kGravity) * hij);
    qxij = hij * vel;
    qyij = hij * vel;
  }
  h[ib] = hij * f0;
  qx[ib] = qxij * f1;
  qy[ib] = qyij * f2;
  h[ii] = hij * f0;
  qx[ii] = qxij * f1;
  qy[ii] = qyij * f2;
  if (corner) {
    h[ibc] = hij * f0;
    qx[ibc] = qxij * f1;
    qy[ibc] = qyij * f2;
  }
}

template <typename T>
__global__ void k_extbc(DevClock* __restrict__ clk, StateBufs<T> sb, const BedMap<T> bed, const T* __restrict__ n2,
                        const int32_t* __restrict__ order, int count, const int32_t* __restrict__ cells,
                        const int32_t* __restrict__ types, const int32_t* __restrict__ start,
                        const int32_t* __restrict__ nrowsv, const T* __restrict__ var1, const T* __restrict__ var2,
                        int rows, int cols) {
  pdl_wait();
  pdl_trigger();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count || !clk->active) return;
  extbc_apply<T>(clk, sb, bed, n2, order[k], cells, types, start, nrowsv, var1, var2, rows, cols);
}

// ---------------------------------------------------------------------------
// k_wetdry_dt: wet/dry masks and max depth on interior cells, then the CFL dt
// of every cell (ghosts included, as compute_dt_and_sqrt runs over rows*cols)
// reduced warp -> block -> one atomicMin on the ordered key of the slot the
// next k_clock reads.  With WETDRY=false it is the initial dt pass.
// Each thread walks one column down a band of rows, keeping h and the bed of
// the rows above and below in registers and loading the next row one
// iteration ahead; east/west neighbours come by shuffle (lanes 0 and 31 load
// theirs).  Every value is read once, with several loads in flight.
// ---------------------------------------------------------------------------
// Kahan fold of the step's volume terms into the domain's totals.
__device__ __forceinline__ void fold_accounts(DevClock* __restrict__ clk) {
  for (int k = 0; k < kAccTerms; k++) {
    const double y = clk->acc_step[k] - clk->acc_comp[k];
    const double t = clk->acc_sum[k] + y;
    clk->acc_comp[k] = (t - clk->acc_sum[k]) - y;
    clk->acc_sum[k] = t;
    clk->acc_step[k] = 0.0;
  }
}

// One block's band: columns bx*128 .. +127, rows by*band .. +band-1.
// Returns this thread's minimum dt key.
template <typename T, bool WETDRY>
__device__ __forceinline__ unsigned long long wetdry_band(const DevClock* __restrict__ clk, const StateBufs<T>& sb,
                                                          const BedMap<T>& bed, T* __restrict__ maxh, int rows,
                                                          int cols, int band, double dx, double cn, T hextra,
                                                          float* __restrict__ arrival, float arrival_depth, int bx,
                                                          int by) {
  const int buf = WETDRY ? clk->dst : clk->cur;
  const T* __restrict__ h = sb.H(buf);
  T* __restrict__ qx = sb.QX(buf);
  T* __restrict__ qy = sb.QY(buf);
  const T E12 = eps12<T>();
  const int lane = threadIdx.x & 31;
  const int c = bx * kWetCols + threadIdx.x;
  const int ra = by * band;
  const int rz = min(ra + band - 1, rows - 1);
  const bool incol = c < cols;
  const bool intcol = c >= 1 && c <= cols - 2;
  const double zref = bed.ref_of(ra, min(bx * kWetCols, cols - 1));
  const float simtime_now = WETDRY ? (float)clk->simtime : 0.0f;

  T hm = T(0), zm = T(0), h0 = T(0), z0 = T(0), hp = T(0), zp = T(0);
  T qx0 = T(0), qy0 = T(0), mh0 = T(0), qxp = T(0), qyp = T(0), mhp = T(0);
  auto load_row = [&](int r, T& hv, T& zv, T& qxv, T& qyv, T& mhv) {
    if (incol && r >= 0 && r < rows) {
      const size_t id = (size_t)r * cols + c;
      hv = h[id];
      zv = bed.local(id, r, c, zref);
      qxv = qx[id];
      qyv = qy[id];
      if (WETDRY && intcol && r >= 1 && r <= rows - 2) mhv = maxh[id];
    }
  };
  {
    T a, b, e;
    if (ra >= 1) load_row(ra - 1, hm, zm, a, b, e);
  }
  load_row(ra, h0, z0, qx0, qy0, mh0);
  unsigned long long key = kDtKeyInf;
  for (int r = ra; r <= rz; ++r) {
    if (r + 1 <= rows - 1) load_row(r + 1, hp, zp, qxp, qyp, mhp);
    // east / west neighbours of row r
    T he = __shfl_down_sync(0xffffffffu, h0, 1), ze = __shfl_down_sync(0xffffffffu, z0, 1);
    T hw = __shfl_up_sync(0xffffffffu, h0, 1), zw = __shfl_up_sync(0xffffffffu, z0, 1);
    const size_t id = (size_t)r * cols + c;
    const bool interior = WETDRY && intcol && r >= 1 && r <= rows - 2;
    if (interior) {
      if (lane == 31) {
        he = h[id + 1];
        ze = bed.local(id + 1, r, c + 1, zref);
      }
      if (lane == 0) {
        hw = h[id - 1];
        zw = bed.local(id - 1, r, c - 1, zref);
      }
    }
    T qxv = qx0, qyv = qy0;
    const T hij = h0;
    if (interior) {
      const T zij = z0;
      if (hij > hextra) {
        if ((hij + zij < ze && he < E12) || (hij + zij < zw && hw < E12)) {
          qxv = T(0);
          qx[id] = T(0);
        }
        if ((hij + zij < zm && hm < E12) || (hij + zij < zp && hp < E12)) {
          qyv = T(0);
          qy[id] = T(0);
        }
      }
      if (hij > mh0) maxh[id] = hij;
      if (arrival != nullptr && hij > arrival_depth && !(arrival[id] < 3.0e38f)) arrival[id] = simtime_now;
    }
    if (incol && hij > hextra) {  // wave speed of the CFL dt (reduced as its maximum)
      double d;
      if (sizeof(T) == 8) {  // FP64: the reference's denominator, bit for bit
        const double hd = (double)hij;
        const double sq = fmax(sqrt(hd), 0.0);
        const double maxu = fmax(fabs((double)qxv), fabs((double)qyv)) / hd;
        d = maxu + kSqrtG * sq;
      } else {  // FP32 form: speed in FP32, maximum and dt in FP64
        const T sq = dev_fmax(dev_sqrt(hij), T(0));
        const T maxu = fdiv(dev_fmax(dev_fabs(qxv), dev_fabs(qyv)), hij);
        d = (double)(maxu + T(kSqrtG) * sq);
      }
      const unsigned long long k = speed_key(d);
      key = k < key ? k : key;
    }
    hm = h0;
    zm = z0;
    h0 = hp;
    z0 = zp;
    qx0 = qxp;
    qy0 = qyp;
    mh0 = mhp;
  }
  return key;
}

// ---------------------------------------------------------------------------
// Staged wet-dry/dt: one block per band of WetStage<T>::kBand rows x
// kWetCols columns.  The block stages, in shared memory, its rows of h and
// the bed with a halo row above and below, and its rows of qx, qy and the
// maximum depth, each row from column c0-1 to c0+kWetCols (clipped to the
// grid) with one bulk asynchronous copy (cp.async.bulk: rounded out to
// 16-byte boundaries, which every field's kFieldPad allows at its end).  All
// copies are issued at once, in groups of kStageGroupRows output rows, each
// group completing on its own mbarrier: a thread walking its column down the band
// starts on the first two rows while the later rows are still in flight, so
// a block's loads overlap its own arithmetic even when every block of a wave
// starts at the same moment.  The FP32 form turns a staged bed offset into a
// level relative to the block's reference as it reads it (its tile's delta,
// added in registers), so no pass over shared memory and no block barrier
// sits between the copies and the arithmetic.
// ---------------------------------------------------------------------------
template <typename T>
struct WetStage {
  static constexpr int kBand = kStageBand<T>;                        // rows per block
  static constexpr int kVec = 16 / (int)sizeof(T);                   // elements per 16 bytes
  static constexpr int kCap = kWetCols + 2 + 2 * (kVec - 1);         // elements per row buffer
  static constexpr int kHRows = kBand + 2;                           // h and bed rows (with halos)
  static constexpr int kRows = 2 * kHRows + 3 * kBand;               // + qx, qy, max depth rows
  static constexpr size_t kData = (size_t)kRows * kCap * sizeof(T);
  // copy groups of kGR output rows: group 0 = h and bed staged rows
  // 0..kGR+1 and band rows 0..kGR-1 of qx, qy, max depth; group g > 0 = h and
  // bed staged rows g*kGR+2..g*kGR+kGR+1 and band rows g*kGR..g*kGR+kGR-1
  static constexpr int kGR = kStageGroupRows<T>;
  static constexpr int kGroups = kBand / kGR;
  static constexpr int kFirst = 2 * (kGR + 2) + 3 * kGR, kNext = 5 * kGR;
  static constexpr size_t kBarBytes = (8 * kGroups + 15) / 16 * 16;
  // FP32 form: the staged rows span at most 2 x 6 bed tiles of 32 x 32
  // (kBand + 2 <= 32 rows, kWetCols + 2 <= 5 * 32 + 2 columns)
  static constexpr int kTileCols = 6, kTileSlots = 2 * kTileCols;
  static constexpr size_t kBytes = kData + kBarBytes + 4 * kHRows + 4 * kTileSlots;  // + row offsets, tiles
};
static_assert(kStageBand<double> % kStageGroupRows<double> == 0 && kStageBand<float> % kStageGroupRows<float> == 0,
              "bands are whole copy groups");
static_assert(WetStage<double>::kFirst + (WetStage<double>::kGroups - 1) * WetStage<double>::kNext ==
                  WetStage<double>::kRows, "copy groups cover the staged rows");
static_assert(WetStage<float>::kFirst + (WetStage<float>::kGroups - 1) * WetStage<float>::kNext ==
                  WetStage<float>::kRows, "copy groups cover the staged rows");
static_assert(WetStage<float>::kBand + 2 <= 32, "staged rows span at most two bed tile rows");

// Gives up on a block whose copies did not land: reports it, waits (bounded)
// once more on every group from 'from' on so no copy still writes this
// block's shared memory when it exits.
template <int kGroups>
__device__ __forceinline__ void stage_abandon(DevClock* clk, uint64_t* bar, int from) {
  atomicExch(&clk->status, kStatusStageTimeout);
  for (int g = from; g < kGroups; ++g) mbar_wait(&bar[g], 0);
}

// Test hook (one thread of one block): a bounded wait on a barrier whose
// phase can never complete (its arrival count is met, but it expects 16 bytes
// that no copy delivers, and no copy is ever issued on it).  The wait gives up
// after clk->wait_test polls and records a device status as a stage timeout
// does, so the host's handling of a wait that gave up can be tested without
// disturbing any real copy.
static __device__ __noinline__ void wait_test(DevClock* clk) {
  __shared__ __align__(8) uint64_t bar;
  mbar_init(&bar, 1);
  mbar_arrive_expect_tx(&bar, 16);
  if (!mbar_wait(&bar, 0, clk->wait_test)) atomicExch(&clk->status, kStatusTestWait);
}

template <typename T>
__device__ __forceinline__ unsigned long long wetdry_staged(DevClock* __restrict__ clk, const StateBufs<T>& sb,
                                                            const BedMap<T>& bed, T* __restrict__ maxh, int rows,
                                                            int cols, T hextra, float* __restrict__ arrival,
                                                            float arrival_depth, int bx, int by, T* stage) {
  using S = WetStage<T>;
  constexpr bool kF32 = sizeof(T) == 4;
  const int buf = clk->dst;
  T* __restrict__ qx = sb.QX(buf);
  T* __restrict__ qy = sb.QY(buf);
  const T E12 = eps12<T>();
  const int tid = threadIdx.x, lane = tid & 31;
  const int c0 = bx * kWetCols;
  const int ra = by * S::kBand;
  const int rz = min(ra + S::kBand - 1, rows - 1);
  const int cl = max(c0 - 1, 0), ce = min(c0 + kWetCols + 1, cols);  // staged columns [cl, ce)
  unsigned char* tail = reinterpret_cast<unsigned char*>(stage) + S::kData;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tail);
  // offs[j]: column c of staged row ra-1+j sits at buffer index c + offs[j]
  int* offs = reinterpret_cast<int*>(tail + S::kBarBytes);
  // FP32 form: per bed tile the staged rows touch, its base minus the
  // block's reference level
  float* tdel = reinterpret_cast<float*>(offs + S::kHRows);
  const int rlo = max(ra - 1, 0), rhi = min(rz + 1, rows - 1);
  const int tr0 = rlo >> 5, tc0 = cl >> 5;
  if (tid < S::kGroups) mbar_init(&bar[tid], 1);
  if (tid < S::kHRows) {
    const int64_t r = (int64_t)(ra - 1 + tid);
    offs[tid] = (int)(r * cols - ((r * cols + cl) & ~(int64_t)(S::kVec - 1)));
  }
  if (kF32 && tid >= 32 && tid < 32 + S::kTileSlots) {
    const int s = tid - 32, tr = tr0 + s / S::kTileCols, tc = tc0 + s % S::kTileCols;
    if (tr <= (rhi >> 5) && tc <= ((ce - 1) >> 5))
      tdel[s] = (float)(bed.base_at(tr << 5, tc << 5) - bed.ref_of(ra, min(c0, cols - 1)));
  }
  __syncthreads();
  if (tid < 32) {
    for (int i = lane; i < S::kRows; i += 32) {
      // copy i -> group g, field f (0 h, 1 bed, 2 qx, 3 qy, 4 max depth) and
      // q: staged row (h, bed; global row ra-1+q) or band row (global ra+q)
      int g, f, q;
      if (i < S::kFirst) {
        g = 0;
        if (i < 2 * (S::kGR + 2)) {
          f = i / (S::kGR + 2);
          q = i % (S::kGR + 2);
        } else {
          f = 2 + (i - 2 * (S::kGR + 2)) / S::kGR;
          q = (i - 2 * (S::kGR + 2)) % S::kGR;
        }
      } else {
        const int t = (i - S::kFirst) % S::kNext;
        g = 1 + (i - S::kFirst) / S::kNext;
        if (t < 2 * S::kGR) {
          f = t / S::kGR;
          q = g * S::kGR + 2 + t % S::kGR;
        } else {
          f = 2 + (t - 2 * S::kGR) / S::kGR;
          q = g * S::kGR + (t - 2 * S::kGR) % S::kGR;
        }
      }
      int r, slot;
      const T* src;
      if (f < 2) {
        r = ra - 1 + q;
        if (r < 0 || r > rows - 1) continue;
        slot = f * S::kHRows + q;
        src = f == 0 ? (const T*)sb.H(buf) : (const T*)bed.z;
      } else {
        r = ra + q;
        if (r > rz) continue;
        slot = 2 * S::kHRows + (f - 2) * S::kBand + q;
        src = f == 2 ? (const T*)qx : (f == 3 ? (const T*)qy : (const T*)maxh);
      }
      const int64_t e0 = ((int64_t)r * cols + cl) & ~(int64_t)(S::kVec - 1);
      const int64_t e1 = ((int64_t)r * cols + ce + S::kVec - 1) & ~(int64_t)(S::kVec - 1);
      const uint32_t bytes = (uint32_t)((e1 - e0) * (int64_t)sizeof(T));
      mbar_expect_tx(&bar[g], bytes);
      bulk_g2s(stage + (size_t)slot * S::kCap, src + e0, bytes, &bar[g]);
    }
    __syncwarp();
    if (lane == 0)
      for (int g = 0; g < S::kGroups; ++g) mbar_arrive(&bar[g]);
  }
  const T* sh = stage;
  const T* sz = stage + (size_t)S::kHRows * S::kCap;
  const T* sqx = stage + (size_t)2 * S::kHRows * S::kCap;
  const T* sqy = sqx + (size_t)S::kBand * S::kCap;
  const T* smh = sqy + (size_t)S::kBand * S::kCap;
  const int c = c0 + tid;
  const bool incol = c < cols;
  const bool intcol = c >= 1 && c <= cols - 2;
  // FP32 form: tile deltas of columns c-1, c, c+1 in tile rows 0 and 1
  // (BedMap::local_v; where a delta is zero the level is the offset itself,
  // up to the sign of a zero, which no comparison below sees)
  T dw0 = T(0), dw1 = T(0), dc0 = T(0), dc1 = T(0), de0 = T(0), de1 = T(0);
  if (kF32 && intcol) {
    const int tw = ((c - 1) >> 5) - tc0, tc = (c >> 5) - tc0, te = ((c + 1) >> 5) - tc0;
    dw0 = (T)tdel[tw];
    dc0 = (T)tdel[tc];
    de0 = (T)tdel[te];
    if ((rhi >> 5) > tr0) {
      dw1 = (T)tdel[S::kTileCols + tw];
      dc1 = (T)tdel[S::kTileCols + tc];
      de1 = (T)tdel[S::kTileCols + te];
    }
  }
  const float simtime_now = (float)clk->simtime;
  // largest wave speed of the thread's cells (NaN speeds left out, as
  // speed_key does); one key at the end equals the minimum of per-cell keys
  T dmax = T(-1);
  if (incol) {
    // bed level of the thread's column at staged row j (buffer offset oj)
    auto zlev = [&](int j, int oj) -> T {
      T v = sz[j * S::kCap + c + oj];
      if (kF32) v += (((ra - 1 + j) >> 5) > tr0) ? dc1 : dc0;
      return v;
    };
    int om = offs[0], o = offs[1];
    T zm = T(0), z0 = T(0);
#pragma unroll
    for (int jq = 0; jq < S::kBand; ++jq) {
      const int r = ra + jq;
      if (r > rz) break;
      if (jq % S::kGR == 0 && !mbar_wait(&bar[jq / S::kGR], 0)) {
        stage_abandon<S::kGroups>(clk, bar, jq / S::kGR);
        return kDtKeyInf;
      }
      const int j = jq + 1;
      const int op = offs[j + 1];
      if (jq == 0) {
        zm = zlev(0, om);
        z0 = zlev(1, o);
      }
      const T zp = zlev(j + 1, op);
      const size_t id = (size_t)r * cols + c;
      const T* hrow = sh + j * S::kCap + o;
      const T hij = hrow[c];
      T qxv = sqx[jq * S::kCap + c + o], qyv = sqy[jq * S::kCap + c + o];
      if (intcol && r >= 1 && r <= rows - 2) {
        if (hij > hextra) {
          const T he = hrow[c + 1], hw = hrow[c - 1];
          const T hm = sh[(j - 1) * S::kCap + c + om];
          const T hp = sh[(j + 1) * S::kCap + c + op];
          const T* zrow = sz + j * S::kCap + o;
          T ze = zrow[c + 1], zw = zrow[c - 1];
          if (kF32) {
            const bool t1 = (r >> 5) > tr0;
            ze += t1 ? de1 : de0;
            zw += t1 ? dw1 : dw0;
          }
          if ((hij + z0 < ze && he < E12) || (hij + z0 < zw && hw < E12)) {
            qxv = T(0);
            qx[id] = T(0);
          }
          if ((hij + z0 < zm && hm < E12) || (hij + z0 < zp && hp < E12)) {
            qyv = T(0);
            qy[id] = T(0);
          }
        }
        if (hij > smh[jq * S::kCap + c + o]) maxh[id] = hij;
        if (arrival != nullptr && hij > arrival_depth && !(arrival[id] < 3.0e38f)) arrival[id] = simtime_now;
      }
      if (hij > hextra) {  // wave speed of the CFL dt (reduced as its maximum)
        T d;
        if (sizeof(T) == 8) {  // FP64: the reference's denominator, bit for bit
          const double hd = (double)hij;
          const double sq = fmax(sqrt(hd), 0.0);
          const double maxu = fmax(fabs((double)qxv), fabs((double)qyv)) / hd;
          d = (T)(maxu + kSqrtG * sq);
        } else {  // FP32 form: speed in FP32, maximum and dt in FP64
          const T sq = dev_fmax(dev_sqrt(hij), T(0));
          const T maxu = fdiv(dev_fmax(dev_fabs(qxv), dev_fabs(qyv)), hij);
          d = maxu + T(kSqrtG) * sq;
        }
        dmax = dev_fmax(dmax, d);
      }
      zm = z0;
      z0 = zp;
      om = o;
      o = op;
    }
  }
  return dmax >= T(0) ? speed_key((double)dmax) : kDtKeyInf;
}

// Block minimum of the threads' keys, folded into *slot with one atomic.
__device__ __forceinline__ void block_min_into(unsigned long long key, unsigned long long* slot) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  __shared__ unsigned long long s_min[kWetCols / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_min[warp] = key;
  __syncthreads();
  if (threadIdx.x == 0) {
    key = s_min[0];
    for (int w = 1; w < kWetCols / 32; w++) key = s_min[w] < key ? s_min[w] : key;
    // most blocks cannot lower the slot: read it first, then one atomic
    if (key < kDtKeyInf && key < *reinterpret_cast<volatile unsigned long long*>(slot)) atomicMin(slot, key);
  }
}

template <typename T, bool WETDRY>
__global__ void __launch_bounds__(kWetCols) k_wetdry_dt(DevClock* __restrict__ clk, StateBufs<T> sb,
                                                        const BedMap<T> bed, T* __restrict__ maxh, int rows,
                                                        int cols, int band, double dx, double cn, T hextra,
                                                        float* __restrict__ arrival, float arrival_depth) {
  if (WETDRY && !clk->active) return;
  if (WETDRY && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) fold_accounts(clk);
  const unsigned long long key = wetdry_band<T, WETDRY>(clk, sb, bed, maxh, rows, cols, band, dx, cn, hextra,
                                                        arrival, arrival_depth, blockIdx.x, blockIdx.y);
  block_min_into(key, &clk->dt_key[WETDRY ? clk->wr : clk->rd]);
}

// True when every flux tile covering this block's band holds only +0 in the
// step's destination buffer (tzero: the flux kernel's [2][tiles] flags).  A
// band without a wet cell has nothing to mask and no wave speed, and it
// records no max depth or arrival while no max depth is negative (a device
// flag set by max depth uploads) and the arrival depth is not (the host
// passes no flags then).  Cell (r, c) belongs to tile row max(r-1,0)/rb and
// strip max(c-1,0)/kStripCols, clamped: ghost rows and columns belong to the
// edge tiles that copy them.  Uniform over the block.
template <typename T>
__device__ __forceinline__ bool band_all_zero(const DevClock* clk, const uint8_t* __restrict__ tzero, int rows,
                                              int cols, int rb, int bx, int by) {
  const int ns = (cols - 2 + kStripCols - 1) / kStripCols, nty = (rows - 2 + rb - 1) / rb;
  const uint8_t* tz = tzero + (size_t)clk->dst * ((size_t)ns * nty);
  const int ra = by * WetStage<T>::kBand, rz = min(ra + WetStage<T>::kBand - 1, rows - 1);
  const int c0 = bx * kWetCols, c1 = min(c0 + kWetCols - 1, cols - 1);
  const int t0 = min(max(ra - 1, 0) / rb, nty - 1), t1 = min(max(rz - 1, 0) / rb, nty - 1);
  const int s0 = min(max(c0 - 1, 0) / kStripCols, ns - 1), s1 = min(max(c1 - 1, 0) / kStripCols, ns - 1);
  const int nsx = s1 - s0 + 1, count = (t1 - t0 + 1) * nsx;
  int nz = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) nz |= !tz[(size_t)(t0 + i / nsx) * ns + s0 + i % nsx];
  return !__syncthreads_or(nz);
}

template <typename T>
__global__ void __launch_bounds__(kWetCols) k_wetdry_staged(DevClock* __restrict__ clk, StateBufs<T> sb,
                                                            const BedMap<T> bed, T* __restrict__ maxh, int rows,
                                                            int cols, T hextra, float* __restrict__ arrival,
                                                            float arrival_depth, const uint8_t* __restrict__ tzero,
                                                            int rb, const int32_t* __restrict__ maxh_neg) {
  extern __shared__ __align__(128) unsigned char wet_smem[];
  pdl_wait();
  pdl_trigger();
  if (!clk->active) return;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    fold_accounts(clk);
    if (clk->wait_test) wait_test(clk);
  }
  if (tzero != nullptr && *maxh_neg == 0 && band_all_zero<T>(clk, tzero, rows, cols, rb, blockIdx.x, blockIdx.y)) {
    if (threadIdx.x == 0) {  // interior cells of the skipped band
      const int ra = max((int)blockIdx.y * WetStage<T>::kBand, 1);
      const int rz = min((int)blockIdx.y * WetStage<T>::kBand + WetStage<T>::kBand - 1, rows - 2);
      const int ca = max((int)blockIdx.x * kWetCols, 1), cz = min((int)blockIdx.x * kWetCols + kWetCols - 1, cols - 2);
      if (rz >= ra && cz >= ca)
        atomicAdd(&clk->skipped[1][(blockIdx.x + blockIdx.y * 7) % kSkipSlots],
                  (unsigned long long)(rz - ra + 1) * (cz - ca + 1));
    }
    return;
  }
  const unsigned long long key = wetdry_staged<T>(clk, sb, bed, maxh, rows, cols, hextra, arrival, arrival_depth,
                                                  blockIdx.x, blockIdx.y, reinterpret_cast<T*>(wet_smem));
  block_min_into(key, &clk->dt_key[clk->wr]);
}

// ===========================================================================
// Batched ensembles: one launch per kernel type advances every member of a
// batch by one of its own steps (each member keeps its own clock and dt).
// Members are described in device memory (MemberDev); the flux kernel's warps
// take tiles from one queue over all members' tiles, the wet-dry kernel's
// blocks are a concatenation of every member's bands.
// ===========================================================================
template <typename T>
__global__ void k_batch_clock(const MemberDev<T>* __restrict__ mem, int nm, BatchCtl* __restrict__ ctl) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) ctl->tile_next = 0;
  if (m < nm && clock_step(mem[m].clk)) atomicAdd(&ctl->halted, 1);
}

template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) k_batch_flux(const MemberDev<T>* __restrict__ mem,
                                                          const int32_t* __restrict__ tile_member,
                                                          BatchCtl* __restrict__ ctl, uint32_t ntiles) {
  __shared__ FluxCtx<T> s_ctx[4];  // the member context of each warp's tile
  const int lane = threadIdx.x & 31;
  while (true) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(&ctl->tile_next, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= ntiles) break;
    const MemberDev<T>& M = mem[tile_member[tile]];
    if (!M.clk->active) continue;
    __syncwarp();  // the warp's previous tile no longer reads its context
    if (lane == 0)
      s_ctx[threadIdx.x >> 5] = flux_ctx<T>(M.clk, M.sb, M.bed, M.n2, M.zone, M.rates, M.rows, M.cols, M.rb, M.dx,
                                            M.rdx, M.hextra);
    __syncwarp();
    flux_tile<T, false, true>(s_ctx[threadIdx.x >> 5], tile - M.tile_begin, lane);
  }
}

template <typename T>
__global__ void __launch_bounds__(kWetCols) k_batch_wetdry(const MemberDev<T>* __restrict__ mem,
                                                            const int32_t* __restrict__ wet_member) {
  extern __shared__ __align__(128) unsigned char wet_smem[];
  const MemberDev<T>& M = mem[wet_member[blockIdx.x]];
  DevClock* clk = M.clk;
  if (!clk->active) return;
  const uint32_t local = blockIdx.x - M.wet_begin;
  if (local == 0 && threadIdx.x == 0) fold_accounts(clk);
  const unsigned long long key =
      wetdry_staged<T>(clk, M.sb, M.bed, M.maxh, M.rows, M.cols, M.hextra, M.arrival, M.arrival_depth,
                       (int)(local % M.wet_nbx), (int)(local / M.wet_nbx), reinterpret_cast<T*>(wet_smem));
  block_min_into(key, &clk->dt_key[clk->wr]);
}

// Open-boundary ghosts of the batch members that have open edges: block row
// y serves member open_members[y].
template <typename T>
__global__ void k_batch_open_bc(const MemberDev<T>* __restrict__ mem, const int32_t* __restrict__ open_members) {
  const MemberDev<T>& M = mem[open_members[blockIdx.y]];
  if (!M.clk->active) return;
  open_bc_item<T>(M.clk, M.sb, M.rows, M.cols, blockIdx.x * blockDim.x + threadIdx.x);
}

// Point source `id` of member M (compute_flow, kernels.h:51-84).
template <typename T>
__device__ __forceinline__ void source_apply(const MemberDev<T>& M, int id) {
  DevClock* clk = M.clk;
  const int lo = clk->src_idx_low, hi = clk->src_idx_high;
  const T dt = T(clk->global_dt), simtime = T(clk->t_step);
  T* h = M.sb.H(clk->dst);
  const T flo = M.hyg_v[(size_t)lo * M.nsrc + id], fhi = M.hyg_v[(size_t)hi * M.nsrc + id];
  const T tlo = T(M.hyg_t[lo]), thi = T(M.hyg_t[hi]);
  T flow;
  if (lo == hi) {
    flow = flo;
  } else {
    const T td = simtime - tlo, td2 = thi - tlo;
    flow = flo + (((fhi - flo) * td) / td2);
  }
  const int sid = M.src_cells[id];
  T hij = h[sid];
  const T hs = (flow * dt) / (M.dx * M.dx);
  hij += hs;
  h[sid] = hij;
  atomicAdd(&clk->acc_step[kAccSources], (double)hs);
}

// Sparse forcing of a batch: items are (member, index) pairs of one
// conflict-free wave (a member's own waves keep its index order).
template <typename T>
__global__ void k_batch_sources(const MemberDev<T>* __restrict__ mem, const int2* __restrict__ items, int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const MemberDev<T>& M = mem[items[k].x];
  if (!M.clk->active) return;
  source_apply<T>(M, items[k].y);
}

template <typename T>
__global__ void k_batch_extbc(const MemberDev<T>* __restrict__ mem, const int2* __restrict__ items, int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const MemberDev<T>& M = mem[items[k].x];
  if (!M.clk->active) return;
  extbc_apply<T>(M.clk, M.sb, M.bed, M.n2, items[k].y, M.bc_cells, M.bc_types, M.bc_start, M.bc_nrows, M.bc_v1,
                 M.bc_v2, M.rows, M.cols);
}

// ===========================================================================
// Single-launch batches: k_batch_steps advances every member of a batch by
// `nsteps` of its own time steps in ONE launch.  Blocks stay resident and take
// work items from a ticket counter in a fixed order; per batched step s:
//   nm clock items (one per member), then the flux tiles of all members in
//   groups of four (one per warp), then nm forcing items (a member's point
//   sources, open-edge ghosts and external-boundary cells, wave by wave), then
//   the wet-dry/dt blocks of all members.
// An item waits only for items of its own member with lower tickets (flux
// tiles for the member's clock of step s, forcing for all its flux tiles of
// step s, wet-dry blocks for its forcing of step s, the clock of step s+1 for
// all its wet-dry blocks of step s), counted in MemberProgress.  Lower
// tickets were taken by blocks that are running, so the lowest unfinished
// ticket can always proceed and every wait ends: members advance without a
// barrier across members or across the grid, and the tail of one phase
// overlaps the next phase of members that are ahead.  Waits are bounded
// (kStepWaitPolls); one that gives up records a status, and the others then
// give up at once.  A producer publishes as a grid barrier does: a block (or
// warp) barrier, then one thread's gpu-scope fence and increment; a consumer
// polls with one thread's acquire load, then a block (or warp) barrier (and
// a proxy fence before bulk copies).  A block takes its next ticket while
// its current item runs, and acquires a (member, step) dependency once for
// consecutive items of the same kind.
// ===========================================================================
template <typename T>
__device__ __forceinline__ void forcing_block(const MemberDev<T>& M) {
  DevClock* clk = M.clk;
  for (int w = 0; w < M.src_nw; ++w) {
    for (int i = M.src_woff[w] + (int)threadIdx.x; i < M.src_woff[w + 1]; i += blockDim.x)
      source_apply<T>(M, M.src_order[i]);
    __syncthreads();
  }
  if (M.open) {
    const int n = max(M.rows, M.cols);
    for (int k = threadIdx.x; k < n; k += blockDim.x) open_bc_item<T>(clk, M.sb, M.rows, M.cols, k);
    __syncthreads();
  }
  for (int w = 0; w < M.bc_nw; ++w) {
    for (int i = M.bc_woff[w] + (int)threadIdx.x; i < M.bc_woff[w + 1]; i += blockDim.x)
      extbc_apply<T>(clk, M.sb, M.bed, M.n2, M.bc_order[i], M.bc_cells, M.bc_types, M.bc_start, M.bc_nrows,
                     M.bc_v1, M.bc_v2, M.rows, M.cols);
    __syncthreads();
  }
}

// Bounded wait until *counter >= target (acquire).  A wait that gives up
// records the status; once any wait of the launch has given up, the others
// give up at once instead of waiting out their own limit.
__device__ __forceinline__ void steps_wait(const uint32_t* counter, uint32_t target, BatchCtl* ctl,
                                           uint32_t polls = kStepWaitPolls) {
  for (uint32_t it = 0; it < polls; ++it) {
    if (ld_acquire_u32(counter) >= target) return;
    if (*reinterpret_cast<volatile int32_t*>(&ctl->status) != 0) return;
    if (it > 32) __nanosleep(128);
  }
  atomicExch(&ctl->status, kStatusStepWait);
}

// Publishes a block's item: after a block barrier (every thread's writes of
// the item happen before it), one thread makes them visible at gpu scope
// (a cumulative fence) and counts the item; the pattern of a grid barrier.
__device__ __forceinline__ void publish_block(uint32_t* counter) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
  }
}

// Thread 0 waits for *counter >= target (acquire); the block barrier after
// it orders every thread's later reads after what the producers published.
__device__ __forceinline__ void acquire_block(const uint32_t* counter, uint32_t target, BatchCtl* ctl) {
  if (threadIdx.x == 0) steps_wait(counter, target, ctl);
  __syncthreads();
}

// The kinds of block item.  The clock, forcing and wet-dry items are compiled
// out of line, so their registers are allocated apart from the flux tile's
// (the persistent loop keeps only a few values live across the calls).
// *seen caches the last (member, step) whose clock this warp has acquired:
// consecutive tiles of one member and step wait once.
template <typename T>
__device__ __forceinline__ void steps_flux_item(const MemberDev<T>* __restrict__ mem,
                                                const int32_t* __restrict__ tile_member, uint32_t ntiles,
                                                uint32_t r, uint32_t s, BatchCtl* __restrict__ ctl,
                                                MemberProgress* __restrict__ prog, uint32_t* seen_m,
                                                uint32_t* seen_s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t tile = 4u * r + (uint32_t)warp;  // one tile per warp
  if (tile >= ntiles) return;
  const int m = tile_member[tile];
  const MemberDev<T>& M = mem[m];
  if (*seen_m != (uint32_t)m || *seen_s != s) {
    if (lane == 0) steps_wait(&prog[m].clock, s + 1, ctl);
    __syncwarp();
    *seen_m = (uint32_t)m;
    *seen_s = s;
  }
  if (M.clk->active) {
    __shared__ FluxCtx<T> s_ctx[4];  // the member context of each warp's tile, reread every row
    if (lane == 0)
      s_ctx[warp] = flux_ctx<T>(M.clk, M.sb, M.bed, M.n2, M.zone, M.rates, M.rows, M.cols, M.rb, M.dx, M.rdx,
                                M.hextra);
    __syncwarp();
    flux_tile<T, false, true>(s_ctx[warp], tile - M.tile_begin, lane);
  }
  __syncwarp();
  if (lane == 0) {
    __threadfence();
    atomicAdd(&prog[m].flux, 1u);
  }
}

template <typename T>
__device__ __noinline__ void steps_clock_item(const MemberDev<T>& M, uint32_t m, uint32_t s,
                                              BatchCtl* __restrict__ ctl, MemberProgress* __restrict__ prog) {
  // test hook (tri_batch_set_wait_test): the first clock item waits for a
  // count no item ever reaches, bounded by ctl->wait_test polls, so the
  // handling of a wait that gave up can be tested with nothing else wrong
  if (ctl->wait_test != 0 && m == 0 && s == 0) steps_wait(&prog[0].clock, 0xFFFFFFFFu, ctl, ctl->wait_test);
  steps_wait(&prog[m].wet, s * M.wet_count, ctl);
  if (clock_step(M.clk)) atomicAdd(&ctl->halted, 1);
  __threadfence();
  atomicAdd(&prog[m].clock, 1u);
}

template <typename T>
__device__ __noinline__ void steps_forcing_item(const MemberDev<T>& M, uint32_t m, uint32_t s,
                                                BatchCtl* __restrict__ ctl, MemberProgress* __restrict__ prog) {
  acquire_block(&prog[m].flux, (s + 1) * (M.tile_end - M.tile_begin), ctl);
  if (M.clk->active) forcing_block<T>(M);
  publish_block(&prog[m].forcing);
}

// Returns true when the block must take no further item (a copy group of
// its staging never completed, so its shared memory may still be written).
// The forcing of (member, step) is acquired once per block: consecutive
// bands of one member and step do not wait again.
template <typename T>
__device__ __noinline__ bool steps_wet_item(const MemberDev<T>* __restrict__ mem,
                                            const int32_t* __restrict__ wet_member, uint32_t r, uint32_t s,
                                            BatchCtl* __restrict__ ctl, MemberProgress* __restrict__ prog,
                                            unsigned char* smem, uint32_t* seen_m, uint32_t* seen_s) {
  using S = WetStage<T>;
  const int m = wet_member[r];
  const MemberDev<T>& M = mem[m];
  if (*seen_m != (uint32_t)m || *seen_s != s) {
    acquire_block(&prog[m].forcing, s + 1, ctl);
    *seen_m = (uint32_t)m;
    *seen_s = s;
  }
  DevClock* clk = M.clk;
  bool broken = false;
  if (clk->active) {
    fence_proxy_async_global();  // the bulk copies read what other blocks wrote
    const uint32_t local = r - M.wet_begin;
    if (local == 0 && threadIdx.x == 0) fold_accounts(clk);
    const unsigned long long key =
        wetdry_staged<T>(clk, M.sb, M.bed, M.maxh, M.rows, M.cols, M.hextra, M.arrival, M.arrival_depth,
                         (int)(local % M.wet_nbx), (int)(local / M.wet_nbx), reinterpret_cast<T*>(smem));
    block_min_into(key, &clk->dt_key[clk->wr]);
    broken = __syncthreads_or(clk->status == kStatusStageTimeout) != 0;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S::kData);
    if (!broken && threadIdx.x < S::kGroups) mbar_inval(&bar[threadIdx.x]);
  }
  publish_block(&prog[m].wet);
  return broken;
}

// The next ticket is taken while the current item runs (its atomic's latency
// hidden); a block then holds two tickets, but its next one is higher than
// its current one, so the lowest unfinished ticket is always a current item
// and can proceed.
template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB)
    k_batch_steps(const MemberDev<T>* __restrict__ mem, int nm, const int32_t* __restrict__ tile_member,
                  uint32_t ntiles, const int32_t* __restrict__ wet_member, uint32_t nwet, int nsteps,
                  BatchCtl* __restrict__ ctl, MemberProgress* __restrict__ prog) {
  extern __shared__ __align__(128) unsigned char wet_smem[];
  __shared__ uint32_t s_ticket[2];
  const uint32_t nflux = (ntiles + 3) / 4;
  const uint32_t per_step = 2u * (uint32_t)nm + nflux + nwet;
  const uint32_t total = per_step * (uint32_t)nsteps;
  if (threadIdx.x == 0) s_ticket[0] = atomicAdd(&ctl->ticket, 1u);
  __syncthreads();
  uint32_t fm = 0xFFFFFFFFu, fs = 0, wm = 0xFFFFFFFFu, ws = 0;  // last acquired (member, step) per kind
  for (int cur = 0;; cur ^= 1) {
    const uint32_t t = s_ticket[cur];
    if (t >= total) return;
    if (threadIdx.x == 0) s_ticket[cur ^ 1] = atomicAdd(&ctl->ticket, 1u);
    const uint32_t s = t / per_step;
    uint32_t r = t - s * per_step;
    if (r < (uint32_t)nm) {  // clock of member r, step s
      if (threadIdx.x == 0) steps_clock_item<T>(mem[r], r, s, ctl, prog);
    } else if ((r -= (uint32_t)nm) < nflux) {
      steps_flux_item<T>(mem, tile_member, ntiles, r, s, ctl, prog, &fm, &fs);
    } else if ((r -= nflux) < (uint32_t)nm) {
      steps_forcing_item<T>(mem[r], r, s, ctl, prog);
    } else {
      r -= (uint32_t)nm;
      if (steps_wet_item<T>(mem, wet_member, r, s, ctl, prog, wet_smem, &wm, &ws)) return;
    }
    __syncthreads();  // the item is finished by every thread; the next ticket is visible
  }
}

}  // namespace tri
