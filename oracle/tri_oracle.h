/* tri_oracle.h -- CPU restatement of the TRITON time-stepping hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against: tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it; the product library never does.
 *
 * Every function restates one reference kernel (file:line in the reference
 * project, TRITON 2.1.1) in plain C with the same floating-point operation
 * order, no FMA contraction (-ffp-contract=off) and IEEE division/sqrt, so the
 * results are bit-identical to the reference's own serial CPU build.  That is
 * checked by the reference's golden vectors (test/reference/{circular,
 * paraboloid,allatoona}) and by the reference itself compiled from its sources
 * into oracle/_ref (see oracle/Makefile).
 *
 * Layout (as the reference's device arrays, triton_init.h:1452-1591): SoA,
 * row-major (rows x cols) doubles INCLUDING the 1-cell ghost ring, id =
 * row*cols + col, row 0 = north.
 */
#ifndef TRI_ORACLE_H
#define TRI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-step kernels.  Arguments follow the reference's Kernels:: signatures. */

/* kernels.h:167-187 */
void tor_compute_dt_and_sqrt(int size, double dx, const double* qx, const double* qy, const double* h,
                             double* sqrth, double* dt_out, double cn, double hextra);
/* kernels.h:196-212 (Min reduction; NaN entries are never selected) */
double tor_find_min_dt(int size, const double* dt);
/* kernels_flux.h:32-285 */
void tor_flux_x(int rows, int cols, double dx, double dt, const double* h, const double* qx, const double* qy,
                const double* z, const double* sqrth, double* rhsh0, double* rhsh1, double* rhsqx0,
                double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra);
/* kernels_flux.h:309-561 */
void tor_flux_y(int rows, int cols, double dx, double dt, const double* h, const double* qx, const double* qy,
                const double* z, const double* sqrth, double* rhsh0, double* rhsh1, double* rhsqx0,
                double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra);
/* kernels_state.h:31-104 */
void tor_update_cells(int rows, int cols, double dt, double* h, double* qx, double* qy, const double* n2,
                      const double* rhsh0, const double* rhsh1, const double* rhsqx0, const double* rhsqx1,
                      const double* rhsqy0, const double* rhsqy1, double hextra);
/* kernels.h:103-152 */
void tor_update_runoff(int rows, int cols, double dt, const int32_t* runoff_id, int row_runoff, int n_rows_runoff,
                       const double* intensity, double* h, double* qx, double* qy, double hextra);
/* kernels.h:51-84 (executed serially in source order, as the serial build does) */
void tor_compute_flow(int nsrc, const double* hyg_t, const double* hyg_v, double dx, double dt, double simtime,
                      int idx_low, int idx_high, double* h, const int32_t* src_idx);
/* kernels.h:437-460 then kernels.h:477-512 (single rank) */
void tor_open_boundaries(int rows, int cols, double* h, double* qx, double* qy);
/* kernels.h:237-424 (single rank; serial in cell order) */
void tor_compute_extbc_values(int ncells, int rows, int cols, double dt, double* h, double* qx, double* qy,
                              const double* z, const double* n2, const int32_t* cell_idx, const int32_t* bctype,
                              const int32_t* start_idx, const int32_t* nrows_vars, const double* var1,
                              const double* var2, double simtime);
/* kernels_wetdry.h:25-93 (single rank, mpi_tasks == 1) */
void tor_wet_dry(int rows, int cols, const double* h, double* qx, double* qy, const double* z, double* maxh,
                 double hextra);
/* kernels.h:522-535 */
void tor_copy_observation_points(int nobs, const double* arr, double* out, const int32_t* obs_idx);

/* ------------------------------------------------------------------------
 * Whole-loop restatement of triton<T>::simulate() (triton_simulate.h:12-160,
 * 163-346) for one rank.  The caller owns every array.  tor_advance runs
 * steps until one of them raises an event (the conditions the reference
 * checks after each step) or max_steps is reached, and reports them so the
 * caller can write outputs exactly where the reference does.
 * ------------------------------------------------------------------------ */
enum {
  TOR_EV_END = 1,   /* simtime >= sim_duration: the while loop ends        */
  TOR_EV_PRINT = 2, /* simtime >= print_interval*(print_id+1)              */
  TOR_EV_OBS = 4,   /* time_series && simtime - last_obs >= print_obs      */
  TOR_EV_LOG = 8    /* it_count % it_print == 0                            */
};

typedef struct tor_sim {
  /* grid (padded) */
  int32_t rows, cols;
  double dx, courant, hextra;
  int32_t open_boundaries;
  /* state and static fields, rows*cols each */
  double *h, *qx, *qy, *z, *n2, *maxh;
  /* scratch, rows*cols each (the reference's SQRTH, DT and six RHS arrays) */
  double *sqrth, *dtv, *rhsh0, *rhsh1, *rhsqx0, *rhsqx1, *rhsqy0, *rhsqy1;
  /* runoff: zone id per cell, intensity[zone*roff_rows + row] in m/s, times in s */
  int32_t nroff, roff_rows;
  int32_t* runoff_id;
  double *roff_t, *roff_v;
  /* point sources: padded cell index, hyg_v[row*nsrc + src] in m3/s */
  int32_t nsrc, hyg_rows;
  int32_t* src_idx;
  double *hyg_t, *hyg_v;
  /* external boundary cells (flattened tables, triton_init.h:913-1055) */
  int32_t nbc;
  int32_t *bc_idx, *bc_type, *bc_start, *bc_nrows;
  double *bc_v1, *bc_v2;
  /* clock: mirrors the loop variables of triton<T>::simulate */
  double simtime, sim_duration, print_interval, print_observation, last_obs_time;
  double init_dt, time_step, global_dt, average_dt;
  int32_t print_id, it_count, it_count_average, it_print;
  int32_t time_series, time_increment_fixed;
  int32_t runoff_row, src_idx_low;
} tor_sim;

/* Runs at most max_steps steps; returns the number of steps run and writes
 * the OR of the events raised by the last step into *events. */
int tor_advance(tor_sim* s, int max_steps, int32_t* events);

/* One time step with the reference's step order (compute_local_dt,
 * compute_global_dt, compute_new_state); updates simtime/it_count. */
void tor_step(tor_sim* s);

#ifdef __cplusplus
}
#endif
#endif
