/* tri_oracle.c -- CPU restatement of the TRITON time-stepping hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see tri_oracle.h.
 *
 * Each routine restates the arithmetic of one reference kernel with the same
 * operation order (C evaluates a*b/c as (a*b)/c, a-b-c as (a-b)-c; the
 * reference relies on the same rules), so that a build with
 * -ffp-contract=off reproduces the reference's serial CPU results bit for
 * bit.  Citations are file:line in the reference project (TRITON 2.1.1).
 *
 * Parity pinned against: the reference's golden ASCII outputs
 * (test/reference/{circular,paraboloid,allatoona}) and the reference compiled
 * from its own sources into oracle/_ref/triton_ref (binary FP64 outputs).
 */
#include "tri_oracle.h"

#include <math.h>
#include <stddef.h>
#include <string.h>

/* constants.h:117-118, 38-50 (double build) */
#define G_ACC 9.81
#define SQRT_G 3.132091953
#define EPS_12 1e-12
#define BIG_DT 1e10

/* ---------------------------------------------------------------------------
 * One face of the augmented Roe solver (kernels_flux.h:84-273 for x faces,
 * :367-556 for y faces; the two kernels differ only in the normal (nx,ny) and
 * in where the results are stored).  "1" is the cell that owns the face,
 * "2" the neighbour across it.  Returns 0 when both cells are dry
 * (h1 > 0 || h2 > 0 is false, :84); otherwise fills d1/d2 (already flushed
 * below EPS12, :255-265).
 * ------------------------------------------------------------------------- */
static int face_flux(double h1, double qx1, double qy1, double z1, double sqh1, double h2, double qx2, double qy2,
                     double z2, double sqh2, double nx, double ny, double dx, double dt, double hextra, double d1[3],
                     double d2[3]) {
  if (!(h1 > 0.0 || h2 > 0.0)) return 0;

  double alpha[3], beta[3], lam[3], lamE[3] = {0.0, 0.0, 0.0}, ev[3][3];
  double u1, v1, u2, v2;
  d1[0] = d1[1] = d1[2] = 0.0;
  d2[0] = d2[1] = d2[2] = 0.0;

  /* velocities, zero below hextra (:98-117) */
  if (h1 >= hextra) {
    u1 = qx1 / h1;
    v1 = qy1 / h1;
  } else {
    u1 = 0.0;
    v1 = 0.0;
  }
  if (h2 >= hextra) {
    u2 = qx2 / h2;
    v2 = qy2 / h2;
  } else {
    u2 = 0.0;
    v2 = 0.0;
  }

  /* Roe averages (:122-133) */
  double h12 = 0.5 * (h1 + h2);
  double dh = h2 - h1;
  double c12 = sqrt(G_ACC * h12);
  double u12 = (u1 * sqh1 + u2 * sqh2) / (sqh1 + sqh2);
  double v12 = (v1 * sqh1 + v2 * sqh2) / (sqh1 + sqh2);
  double un = u12 * nx + v12 * ny;
  lam[0] = un - c12;
  lam[1] = un;
  lam[2] = un + c12;

  /* entropy fix on the two acoustic waves (:137-152) */
  double e1 = u1 * nx + v1 * ny - SQRT_G * sqh1;
  double e2 = u2 * nx + v2 * ny - SQRT_G * sqh2;
  if (e1 < 0.0 && e2 > 0.0) {
    lamE[0] = lam[0] - e1 * (e2 - lam[0]) / (e2 - e1);
    lam[0] = e1 * (e2 - lam[0]) / (e2 - e1);
  }
  e1 = u1 * nx + v1 * ny + SQRT_G * sqh1;
  e2 = u2 * nx + v2 * ny + SQRT_G * sqh2;
  if (e1 < 0.0 && e2 > 0.0) {
    lamE[2] = lam[2] - e2 * (lam[2] - e1) / (e2 - e1);
    lam[2] = e2 * (lam[2] - e1) / (e2 - e1);
  }

  /* right eigenvectors (:154-162) */
  ev[0][0] = 1.0;
  ev[0][1] = u12 - c12 * nx;
  ev[0][2] = v12 - c12 * ny;
  ev[1][0] = 0.0;
  ev[1][1] = -c12 * ny;
  ev[1][2] = c12 * nx;
  ev[2][0] = 1.0;
  ev[2][1] = u12 + c12 * nx;
  ev[2][2] = v12 + c12 * ny;

  /* wave strengths (:164-166) */
  double dqx = qx2 - qx1, dqy = qy2 - qy1;
  alpha[0] = 0.5 * (dh - ((dqx * nx + dqy * ny) - un * dh) / c12);
  alpha[1] = ((dqy - v12 * dh) * nx - (dqx - u12 * dh) * ny) / c12;
  alpha[2] = 0.5 * (dh + ((dqx * nx + dqy * ny) - un * dh) / c12);

  /* upwinded bed-step source with the dry-step limit (:168-192) */
  double dz = z2 - z1;
  double l1 = z1 + h1;
  double l2 = z2 + h2;
  double dzp = dz;
  double hp;
  if (dz >= 0.0) {
    hp = h1;
    if (l1 < z2) dzp = h1;
  } else {
    hp = h2;
    if (l2 < z1) dzp = -h2;
  }
  beta[0] = 0.5 * G_ACC * (hp - 0.5 * fabs(dzp)) * dzp / c12;

  /* positivity ("wet-wet") limiter for subcritical faces (:195-200) */
  hp = h1 + alpha[0];
  if (lam[0] * lam[2] < 0.0 && hp > 0.0 && h1 > 0.0 && h2 > 0.0) {
    beta[0] = fmax(beta[0], lam[0] / (lam[0] + lamE[2]) * (alpha[0] * lam[0] - h1 * dx * 0.5 / dt + lamE[2] * h2));
    beta[0] = fmin(beta[0], lam[2] / (lam[2] + lamE[0]) * (-alpha[2] * lam[2] + h2 * dx * 0.5 / dt + lamE[0] * h1));
  }
  beta[1] = 0.0;
  beta[2] = -beta[0];

  /* intermediate states and dry-side redirection (:205-236) */
  l1 = hp - beta[0] / lam[0];
  l2 = hp + beta[2] / lam[2];
  if (l2 < -EPS_12 && h2 < EPS_12) {
    d1[0] += (lam[0] * alpha[0] - beta[0]) + (lam[2] * alpha[2] - beta[2]);
  } else if (l1 < -EPS_12 && h1 < EPS_12) {
    d2[0] += (lam[0] * alpha[0] - beta[0]) + (lam[2] * alpha[2] - beta[2]);
  } else {
    for (int i = 0; i < 3; i++) {
      double* d = (lam[i] > 0.0) ? d2 : d1;
      d[0] += (lam[i] * alpha[i] - beta[i]) * ev[i][0];
      d[1] += (lam[i] * alpha[i] - beta[i]) * ev[i][1];
      d[2] += (lam[i] * alpha[i] - beta[i]) * ev[i][2];
    }
  }
  /* entropy-fix parts (:238-253) */
  for (int i = 0; i < 3; i++) {
    double* d = (lamE[i] > 0.0) ? d2 : d1;
    d[0] += (lamE[i] * alpha[i]) * ev[i][0];
    d[1] += (lamE[i] * alpha[i]) * ev[i][1];
    d[2] += (lamE[i] * alpha[i]) * ev[i][2];
  }
  /* flush tiny contributions (:255-265) */
  for (int i = 0; i < 3; i++) {
    if (fabs(d1[i]) < EPS_12) d1[i] = 0.0;
    if (fabs(d2[i]) < EPS_12) d2[i] = 0.0;
  }
  return 1;
}

void tor_compute_dt_and_sqrt(int size, double dx, const double* qx, const double* qy, const double* h,
                             double* sqrth, double* dt_out, double cn, double hextra) {
#pragma omp parallel for schedule(static)
  for (int id = 0; id < size; id++) {
    dt_out[id] = BIG_DT;
    double hij = h[id];
    double s = fmax(sqrt(hij), 0.0);
    sqrth[id] = s;
    if (hij > hextra) {
      double maxu = fmax(fabs(qx[id]), fabs(qy[id])) / hij;
      dt_out[id] = cn * dx / (maxu + SQRT_G * s);
    }
  }
}

double tor_find_min_dt(int size, const double* dt) {
  /* Kokkos::Min starts from the largest finite value; "a < m ? a : m" never
   * selects a NaN.  The order of a min fold does not change its result. */
  double m = 1.7976931348623157e308;
  for (int id = 0; id < size; id++) m = dt[id] < m ? dt[id] : m;
  return m;
}

void tor_flux_x(int rows, int cols, double dx, double dt, const double* h, const double* qx, const double* qy,
                const double* z, const double* sqrth, double* rhsh0, double* rhsh1, double* rhsqx0,
                double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra) {
  /* active faces: rows 1..rows-2, owner columns 0..cols-2 (:62-71) */
#pragma omp parallel for schedule(static)
  for (int ix = 1; ix <= rows - 2; ix++) {
    for (int iy = 0; iy <= cols - 2; iy++) {
      size_t a = (size_t)ix * cols + iy, b = a + 1;
      double d1[3], d2[3];
      if (face_flux(h[a], qx[a], qy[a], z[a], sqrth[a], h[b], qx[b], qy[b], z[b], sqrth[b], 1.0, 0.0, dx, dt, hextra,
                    d1, d2)) {
        rhsh0[a] = dt * d1[0] / dx;
        rhsqx0[a] = dt * d1[1] / dx;
        rhsqy0[a] = dt * d1[2] / dx;
        rhsh1[b] = dt * d2[0] / dx;
        rhsqx1[b] = dt * d2[1] / dx;
        rhsqy1[b] = dt * d2[2] / dx;
      } else {
        rhsh0[a] = rhsqx0[a] = rhsqy0[a] = 0.0;
        rhsh1[b] = rhsqx1[b] = rhsqy1[b] = 0.0;
      }
    }
  }
}

void tor_flux_y(int rows, int cols, double dx, double dt, const double* h, const double* qx, const double* qy,
                const double* z, const double* sqrth, double* rhsh0, double* rhsh1, double* rhsqx0,
                double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra) {
  /* active faces: owner rows 1..rows-1 (north neighbour row-1), columns
   * 1..cols-2 (:342-354); results are accumulated (:550-556).  A face
   * writes rhs*0 of its owner and rhs*1 of the north neighbour, so no two
   * faces touch the same entry. */
#pragma omp parallel for schedule(static)
  for (int ix = 1; ix <= rows - 1; ix++) {
    for (int iy = 1; iy <= cols - 2; iy++) {
      size_t a = (size_t)ix * cols + iy, b = a - cols;
      double d1[3], d2[3];
      if (face_flux(h[a], qx[a], qy[a], z[a], sqrth[a], h[b], qx[b], qy[b], z[b], sqrth[b], 0.0, 1.0, dx, dt, hextra,
                    d1, d2)) {
        rhsh0[a] += dt * d1[0] / dx;
        rhsqx0[a] += dt * d1[1] / dx;
        rhsqy0[a] += dt * d1[2] / dx;
        rhsh1[b] += dt * d2[0] / dx;
        rhsqx1[b] += dt * d2[1] / dx;
        rhsqy1[b] += dt * d2[2] / dx;
      }
    }
  }
}

void tor_update_cells(int rows, int cols, double dt, double* h, double* qx, double* qy, const double* n2,
                      const double* rhsh0, const double* rhsh1, const double* rhsqx0, const double* rhsqx1,
                      const double* rhsqy0, const double* rhsqy1, double hextra) {
#pragma omp parallel for schedule(static)
  for (int ix = 1; ix <= rows - 2; ix++) {
    for (int iy = 1; iy <= cols - 2; iy++) {
      size_t id = (size_t)ix * cols + iy;
      double hn = h[id];
      double hij = hn - rhsh0[id] - rhsh1[id];
      double qxij, qyij;
      if (hij < 0.0) hij = 0.0;
      if (hij < hextra) {
        qxij = 0.0;
        qyij = 0.0;
      } else {
        double mx = qx[id] - rhsqx0[id] - rhsqx1[id];
        double my = qy[id] - rhsqy0[id] - rhsqy1[id];
        double modM = sqrt(mx * mx + my * my);
        /* semi-implicit Manning friction on the OLD depth hn (:86-91) */
        if (n2[id] > EPS_12 && hn >= hextra && modM > EPS_12) {
          double tt = dt * G_ACC * n2[id] * modM / (hn * hn * cbrt(hn));
          qxij = -0.5 * (mx - mx * sqrt(1.0 + 4.0 * tt)) / tt;
          qyij = -0.5 * (my - my * sqrt(1.0 + 4.0 * tt)) / tt;
        } else {
          qxij = mx;
          qyij = my;
        }
      }
      h[id] = hij;
      qx[id] = qxij;
      qy[id] = qyij;
    }
  }
}

void tor_update_runoff(int rows, int cols, double dt, const int32_t* runoff_id, int row_runoff, int n_rows_runoff,
                       const double* intensity, double* h, double* qx, double* qy, double hextra) {
#pragma omp parallel for schedule(static)
  for (int ix = 1; ix <= rows - 2; ix++) {
    for (int iy = 1; iy <= cols - 2; iy++) {
      size_t id = (size_t)ix * cols + iy;
      double hij = h[id];
      double net = intensity[(size_t)runoff_id[id] * n_rows_runoff + row_runoff];
      hij += net * dt;
      if (hij < hextra) {
        if (hij < 0.0) hij = 0.0;
        qx[id] = 0.0;
        qy[id] = 0.0;
      }
      h[id] = hij;
    }
  }
}

void tor_compute_flow(int nsrc, const double* hyg_t, const double* hyg_v, double dx, double dt, double simtime,
                      int idx_low, int idx_high, double* h, const int32_t* src_idx) {
  for (int id = 0; id < nsrc; id++) {
    double f_lo = hyg_v[(size_t)idx_low * nsrc + id];
    double f_hi = hyg_v[(size_t)idx_high * nsrc + id];
    double t_lo = hyg_t[idx_low];
    double t_hi = hyg_t[idx_high];
    double flow;
    if (idx_low == idx_high) {
      flow = f_lo;
    } else {
      double td = simtime - t_lo;
      double td2 = t_hi - t_lo;
      flow = f_lo + (((f_hi - f_lo) * td) / td2);
    }
    int sid = src_idx[id];
    double hij = h[sid];
    double hs = (flow * dt) / (dx * dx);
    hij += hs;
    h[sid] = hij;
  }
}

void tor_open_boundaries(int rows, int cols, double* h, double* qx, double* qy) {
  /* west/east ghost columns, all rows (kernels.h:437-460) */
  for (int r = 0; r < rows; r++) {
    size_t g = (size_t)r * cols, i = g + 1;
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
    g = (size_t)r * cols + cols - 1;
    i = g - 1;
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
  }
  /* then north/south ghost rows, all columns (kernels.h:477-512, rank 0 = last rank) */
  for (int c = 0; c < cols; c++) {
    size_t g = (size_t)c, i = (size_t)cols + c;
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
    g = (size_t)(rows - 1) * cols + c;
    i = (size_t)(rows - 2) * cols + c;
    h[g] = h[i];
    qx[g] = qx[i];
    qy[g] = qy[i];
  }
}

void tor_compute_extbc_values(int ncells, int rows, int cols, double dt, double* h, double* qx, double* qy,
                              const double* z, const double* n2, const int32_t* cell_idx, const int32_t* bctype,
                              const int32_t* start_idx, const int32_t* nrows_vars, const double* var1,
                              const double* var2, double simtime) {
  for (int id = 0; id < ncells; id++) {
    int ii = cell_idx[id];
    int bt = bctype[id];
    int s0 = start_idx[id];
    int corner = 0, ib = 0, ibc = 0;
    double fac[3] = {0.0, 0.0, 0.0};
    int ix = ii / cols, iy = ii % cols;
    int top = (ix == 1), btm = (ix == rows - 2), lt = (iy == 1), rt = (iy == cols - 2);
    if (!(top || lt || rt || btm)) continue; /* kernels.h:274-277 with rank 0 of 1 */

    /* orientation of the ghost cell and the sign factors (:279-320) */
    fac[0] = 1.0;
    if (lt) {
      ib = ii - 1;
      fac[1] = -1.0;
      fac[2] = 0.0;
    }
    if (rt) {
      ib = ii + 1;
      fac[1] = 1.0;
      fac[2] = 0.0;
    }
    if (top) {
      ib = ii - cols;
      fac[1] = 0.0;
      fac[2] = 1.0;
      if (lt) {
        corner = 1;
        ibc = ii - 1;
        fac[2] = 0.0;
      }
      if (rt) {
        corner = 1;
        ibc = ii + 1;
        fac[2] = 0.0;
      }
    }
    if (btm) {
      ib = ii + cols;
      fac[1] = 0.0;
      fac[2] = -1.0;
      if (lt) {
        corner = 1;
        ibc = ii - 1;
        fac[2] = 0.0;
      }
      if (rt) {
        corner = 1;
        ibc = ii + 1;
        fac[2] = 0.0;
      }
    }

    double hij = h[ii], qxij = qx[ii], qyij = qy[ii];
    if (bt == 0) { /* copy the inner state out (:329-337) */
      h[ib] = hij;
      qx[ib] = qxij;
      qy[ib] = qyij;
      if (corner) {
        h[ibc] = hij;
        qx[ibc] = qxij;
        qy[ibc] = qyij;
      }
      continue;
    }
    double aux = -999;
    if (bt == 1) { /* water level series, midpoint in time (:346-388) */
      double lvar = 0.5 * (simtime + simtime + dt);
      int lo = -999, hi = nrows_vars[id] - 1;
      if (lvar < var1[0 + s0]) {
        lo = 0;
        hi = 0;
      } else if (lvar > var1[hi + s0]) {
        lo = hi;
      } else {
        for (int i = 0; i < hi; i++) {
          if (var1[i + s0] <= lvar && var1[i + 1 + s0] > lvar) {
            lo = i;
            hi = i + 1;
            break;
          }
        }
      }
      /* lo stays -999 only for a non-monotone table; the reference then
       * indexes out of bounds.  Clamp to the first row instead. */
      if (lo < 0) lo = 0;
      double v1lo = var1[lo + s0], v1hi = var1[hi + s0];
      double v2lo = var2[lo + s0], v2hi = var2[hi + s0];
      if (lo == hi) {
        aux = v2lo;
      } else {
        double td = lvar - v1lo;
        double td2 = v1hi - v1lo;
        aux = v2lo + (((v2hi - v2lo) * td) / td2);
      }
      hij = fmax(aux - z[ii], 0.0);
    } else { /* normal slope (2) or Froude number (3) (:391-400) */
      aux = var1[0 + s0];
      double vel = 0.0;
      if (bt == 2) vel = sqrt(aux * hij * cbrt(hij) / fmax(n2[ii], 1e-6));
      if (bt == 3) vel = aux * sqrt(G_ACC * hij);
      qxij = hij * vel;
      qyij = hij * vel;
    }
    h[ib] = hij * fac[0];
    qx[ib] = qxij * fac[1];
    qy[ib] = qyij * fac[2];
    h[ii] = hij * fac[0];
    qx[ii] = qxij * fac[1];
    qy[ii] = qyij * fac[2];
    if (corner) {
      h[ibc] = hij * fac[0];
      qx[ibc] = qxij * fac[1];
      qy[ibc] = qyij * fac[2];
    }
  }
}

void tor_wet_dry(int rows, int cols, const double* h, double* qx, double* qy, const double* z, double* maxh,
                 double hextra) {
#pragma omp parallel for schedule(static)
  for (int ix = 1; ix <= rows - 2; ix++) {
    for (int iy = 1; iy <= cols - 2; iy++) {
      size_t id = (size_t)ix * cols + iy;
      double hij = h[id], zij = z[id];
      if (hij > hextra) {
        size_t e = id + 1, w = id - 1, n = id - cols, s = id + cols;
        if ((hij + zij < z[e] && h[e] < EPS_12) || (hij + zij < z[w] && h[w] < EPS_12)) qx[id] = 0.0;
        if ((hij + zij < z[n] && h[n] < EPS_12) || (hij + zij < z[s] && h[s] < EPS_12)) qy[id] = 0.0;
      }
      if (hij > maxh[id]) maxh[id] = hij;
    }
  }
}

void tor_copy_observation_points(int nobs, const double* arr, double* out, const int32_t* obs_idx) {
  for (int i = 0; i < nobs; i++) out[i] = arr[obs_idx[i]];
}

/* ---------------------------------------------------------------------------
 * The loop (triton_simulate.h).
 * ------------------------------------------------------------------------- */
void tor_step(tor_sim* s) {
  const int R = s->rows, C = s->cols, N = R * C;
  s->it_count++;
  s->it_count_average++;
  if (!s->time_increment_fixed) {
    /* compute_local_dt (:191-199) */
    tor_compute_dt_and_sqrt(N, s->dx, s->qx, s->qy, s->h, s->sqrth, s->dtv, s->courant, s->hextra);
    double local_dt = tor_find_min_dt(N, s->dtv);
    /* compute_global_dt (:202-226), single rank */
    double g = local_dt;
    if (g >= BIG_DT - 1.0) g = s->init_dt;
    if (s->simtime + g > s->print_interval * (s->print_id + 1)) g = s->print_interval * (s->print_id + 1) - s->simtime;
    s->global_dt = g;
  }
  const double dt = s->global_dt;
  /* compute_new_state (:230-346) */
  tor_flux_x(R, C, s->dx, dt, s->h, s->qx, s->qy, s->z, s->sqrth, s->rhsh0, s->rhsh1, s->rhsqx0, s->rhsqx1, s->rhsqy0,
             s->rhsqy1, s->hextra);
  tor_flux_y(R, C, s->dx, dt, s->h, s->qx, s->qy, s->z, s->sqrth, s->rhsh0, s->rhsh1, s->rhsqx0, s->rhsqx1, s->rhsqy0,
             s->rhsqy1, s->hextra);
  tor_update_cells(R, C, dt, s->h, s->qx, s->qy, s->n2, s->rhsh0, s->rhsh1, s->rhsqx0, s->rhsqx1, s->rhsqy0, s->rhsqy1,
                   s->hextra);
  if (s->nroff > 0) {
    /* runoff row: jumps to the last row after the table, else advances by at most one (:248-258) */
    if (s->simtime > s->roff_t[s->roff_rows - 1]) {
      s->runoff_row = s->roff_rows - 1;
    } else if (s->runoff_row + 1 < s->roff_rows && s->simtime > s->roff_t[s->runoff_row + 1]) {
      s->runoff_row++;
    }
    tor_update_runoff(R, C, dt, s->runoff_id, s->runoff_row, s->roff_rows, s->roff_v, s->h, s->qx, s->qy, s->hextra);
  }
  if (s->nsrc > 0) {
    /* hydrograph bracket search from the last lower index (:266-281) */
    int found = 0, hi = s->hyg_rows - 1;
    for (int i = s->src_idx_low; i < hi; i++) {
      if (s->hyg_t[i + 1] > s->simtime) {
        s->src_idx_low = i;
        hi = i + 1;
        found = 1;
        break;
      }
    }
    if (!found) s->src_idx_low = hi;
    tor_compute_flow(s->nsrc, s->hyg_t, s->hyg_v, s->dx, dt, s->simtime, s->src_idx_low, hi, s->h, s->src_idx);
  }
  if (s->open_boundaries) tor_open_boundaries(R, C, s->h, s->qx, s->qy);
  if (s->nbc > 0)
    tor_compute_extbc_values(s->nbc, R, C, dt, s->h, s->qx, s->qy, s->z, s->n2, s->bc_idx, s->bc_type, s->bc_start,
                             s->bc_nrows, s->bc_v1, s->bc_v2, s->simtime);
  tor_wet_dry(R, C, s->h, s->qx, s->qy, s->z, s->maxh, s->hextra);
  s->simtime += dt;
  s->average_dt += dt;
}

static int32_t tor_events(const tor_sim* s) {
  int32_t ev = 0;
  if (s->it_print > 0 && s->it_count % s->it_print == 0) ev |= TOR_EV_LOG;
  if (s->time_series && s->simtime - s->last_obs_time >= s->print_observation) ev |= TOR_EV_OBS;
  if (s->simtime >= s->print_interval * (s->print_id + 1)) ev |= TOR_EV_PRINT;
  if (!(s->simtime < s->sim_duration)) ev |= TOR_EV_END;
  return ev;
}

int tor_advance(tor_sim* s, int max_steps, int32_t* events) {
  *events = 0;
  if (!(s->simtime < s->sim_duration)) {
    *events = TOR_EV_END;
    return 0;
  }
  int n = 0;
  while (n < max_steps) {
    tor_step(s);
    n++;
    int32_t ev = tor_events(s);
    if (ev) {
      *events = ev;
      break;
    }
  }
  return n;
}
