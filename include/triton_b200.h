/* triton_b200.h -- C ABI of the B200-native TRITON time-stepping library.
 *
 * One shared library (triton_b200/lib/libtriton_b200.so) exports every symbol
 * below with C linkage: plain pointers, sizes and status codes, no C++ or
 * framework types.  Two layers are offered:
 *
 *  1. Kernel entry points (tri_kernel_*): one per reference device kernel,
 *     same arguments and meaning as the reference's Kernels:: templates over
 *     raw device pointers (reference files src/kernels*.h, TRITON 2.1.1), plus
 *     the stream to launch on.  A maintainer replaces each Kernels::X(...) call
 *     in triton_simulate.h with tri_kernel_X_f64(..., stream) and keeps the
 *     rest of the reference loop unchanged.
 *
 *  2. Domain entry points (tri_domain_*): the B200 path.  The library owns the
 *     device state of one simulation domain and runs whole time steps with
 *     fused kernels, the CFL dt reduction and the reference's dt policy on the
 *     device, stopping at the same events the reference loop reacts to
 *     (triton_simulate.h:54-134).  This replaces compute_local_dt,
 *     compute_global_dt and compute_new_state (triton_simulate.h:191-346) and
 *     the device arrays of create_device_vectors (triton_init.h:1452-1591).
 *
 * Grid layout (both layers, as the reference's device arrays): row-major
 * rows x cols values INCLUDING the one-cell ghost ring, id = row*cols + col,
 * row 0 is the northern edge.  Manning values are stored squared (n^2), the
 * closed-boundary walls are DEM ghost values of 1e6 (triton_init.h:212-237).
 *
 * Errors: every call returns a tri_status; tri_last_error() gives the message
 * of the last failure on the calling thread.  Nothing exits the process.
 */
#ifndef TRITON_B200_H
#define TRITON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TRI_ABI_VERSION 1

typedef enum tri_status {
  TRI_OK = 0,
  TRI_E_INVALID = 1, /* bad argument (null pointer, size mismatch, out-of-range index) */
  TRI_E_CUDA = 2,    /* a CUDA runtime call failed (message has the CUDA error string) */
  TRI_E_NOMEM = 3,   /* device allocation failed or the HBM budget would be exceeded */
  TRI_E_STATE = 4,   /* call not valid in the current state */
  TRI_E_IO = 5,      /* file could not be read or written */
  TRI_E_TIMEOUT = 6  /* a bounded device-side wait gave up (no GPU state was lost) */
} tri_status;

typedef enum tri_precision {
  TRI_FP64 = 0, /* plain form: FP64 throughout, matches the reference */
  TRI_FP32 = 1  /* precision form: FP32 state, FP64 dt reduction and volume sums */
} tri_precision;

/* Field ids follow the reference's slot ids (constants.h:82-87). */
typedef enum tri_field {
  TRI_FIELD_H = 0,
  TRI_FIELD_QX = 1,
  TRI_FIELD_QY = 2,
  TRI_FIELD_NMAN2 = 3, /* Manning n squared */
  TRI_FIELD_DEM = 4,
  TRI_FIELD_MAXH = 5
} tri_field;

/* Events raised by the step that ends a tri_domain_advance call; the names
 * are the conditions triton_simulate.h checks after every step. */
enum {
  TRI_EV_END = 1,   /* simtime >= sim_duration (:54)                    */
  TRI_EV_PRINT = 2, /* simtime >= print_interval*(print_id+1) (:92)     */
  TRI_EV_OBS = 4,   /* time_series && simtime-last_obs >= print_obs (:78) */
  TRI_EV_LOG = 8    /* it_count % it_print == 0 (:69)                   */
};

typedef struct tri_grid_desc {
  int32_t rows, cols;      /* padded sizes: interior + 2 ghost rows/columns */
  double cell_size;        /* dx = dy (dem header) */
  double courant;          /* cfg "courant" */
  double hextra;           /* cfg "hextra" */
  int32_t open_boundaries; /* cfg "open_boundaries" */
  int32_t precision;       /* tri_precision */
} tri_grid_desc;

/* The loop variables of triton<T>::simulate (triton_simulate.h:41-52) plus
 * the dt-policy inputs (compute_init_dt :163-187, cfg time_step). */
typedef struct tri_clock {
  double simtime;
  double sim_duration;
  double print_interval;
  double print_observation;
  double last_obs_time;
  double init_dt;    /* dt used when every cell is dry (:217-220) */
  double time_step;  /* fixed dt when time_increment_fixed (cfg) */
  double average_dt; /* running dt sum, reset by the caller on TRI_EV_LOG */
  double global_dt;  /* out: dt of the last step */
  int32_t print_id;
  int32_t it_count;
  int32_t it_print;
  int32_t time_series;
  int32_t time_increment_fixed;
  int32_t runoff_row;  /* index_row_runoff (triton_init.h:1299-1310) */
  int32_t src_idx_low; /* idx_low of the hydrograph search (triton.h:79) */
  int32_t last_events; /* out: OR of TRI_EV_* raised by the last advance
                          (domain or batch); ignored by set_clock */
} tri_clock;

typedef struct tri_progress {
  int32_t steps;  /* steps run by this call */
  int32_t events; /* OR of TRI_EV_* raised by the last step (0: max_steps reached) */
} tri_progress;

typedef struct tri_domain tri_domain;

/* ---- library ---------------------------------------------------------- */
int tri_abi_version(void);
const char* tri_last_error(void);
/* Device memory one domain needs for this grid, in bytes. */
int tri_domain_footprint(const tri_grid_desc* desc, int64_t* bytes);

/* ---- domain ------------------------------------------------------------ */
/* stream: a cudaStream_t to launch on, or NULL for a stream owned by the
 * domain.  Replaces create_device_vectors (triton_init.h:1452-1591). */
int tri_domain_create(const tri_grid_desc* desc, void* stream, tri_domain** out);
int tri_domain_destroy(tri_domain* d);

/* Host <-> device copies of whole padded fields (n = rows*cols values).
 * Host arrays are always double; an FP32 domain rounds on upload.  Uploading
 * H, QX or QY (or DEM) invalidates the cached CFL dt. */
int tri_domain_upload(tri_domain* d, int32_t field, const double* host, int64_t n);
int tri_domain_download(tri_domain* d, int32_t field, double* host, int64_t n);
/* Max depth := the current depth, on the device (the reference starts its max
 * depth array from the initial depth, triton_init.h:1239-1248, and copies it
 * up with the rest): a caller without a max depth of its own saves one field
 * of host-to-device traffic. */
int tri_domain_init_max_depth(tri_domain* d);

/* Forcing tables, flattened as in triton_init.h.
 *  runoff  (:1299-1357): zone id per padded cell (values in [0, nzones)),
 *          times[nrows] in s, rates[zone*nrows + row] in m/s.
 *  sources (:723-816):   padded cell index per source, times[nrows] in s,
 *          flows[row*nsrc + src] in m3/s.
 *  extbc   (:913-1055):  per boundary cell its padded index, type (0..3),
 *          start row in var1/var2 and row count; var1/var2 concatenated
 *          tables (type 1: hours already converted to s).
 *  observations (:818-911): padded cell indices. */
int tri_domain_set_runoff(tri_domain* d, int32_t nzones, int32_t nrows, const double* times, const double* rates,
                          const int32_t* zone_of_cell, int64_t ncells);
int tri_domain_set_sources(tri_domain* d, int32_t nsrc, const int32_t* cells, int32_t nrows, const double* times,
                           const double* flows);
int tri_domain_set_extbc(tri_domain* d, int32_t ncells, const int32_t* cells, const int32_t* types,
                         const int32_t* start, const int32_t* nrows, int32_t nvars, const double* var1,
                         const double* var2);
int tri_domain_set_observations(tri_domain* d, int32_t nobs, const int32_t* cells);

int tri_domain_set_clock(tri_domain* d, const tri_clock* clock);
int tri_domain_get_clock(tri_domain* d, tri_clock* clock);

/* Runs up to max_steps time steps on the device and returns after the first
 * step that raises an event (or after max_steps).  The caller reacts to the
 * events as the reference loop does (write outputs, advance print_id /
 * last_obs_time, reset average_dt) and writes the clock back before the next
 * call.  Blocks until the steps have finished. */
int tri_domain_advance(tri_domain* d, int32_t max_steps, tri_progress* progress);

/* CFL dt of the current state (compute_dt_and_sqrt + find_min_dt, kernels.h:167-212). */
int tri_domain_compute_dt(tri_domain* d, double* local_dt);
/* Values at the observation cells (copy_observation_points, kernels.h:522-535);
 * any output pointer may be NULL. */
int tri_domain_observe(tri_domain* d, double* h, double* qx, double* qy);
/* Sum of h over interior cells times dx^2, accumulated in FP64. */
int tri_domain_volume(tri_domain* d, double* volume);
int tri_domain_synchronize(tri_domain* d);
/* Volume accounts (both forms), m^3: out[0] interior
 * volume now (FP64 sum), then the cumulative Kahan-compensated FP64 totals of
 * inflow through boundary faces, point sources, runoff, external-boundary
 * depth resets and negative-depth clipping since the last H upload.  Volume
 * conservation: out[0] - V0 == out[1] + ... + out[5]. */
int tri_domain_mass_balance(tri_domain* d, double* out6);
/* Records, per cell, the first simtime at which h exceeds 'depth' (arrival
 * time); download gives -1 for cells never reached. */
int tri_domain_track_arrival(tri_domain* d, double depth);
int tri_domain_download_arrival(tri_domain* d, double* host, int64_t n);
/* Kernel timing with CUDA events on the domain's stream: when enabled,
 * advance() records the flux/update kernel and the wet-dry/dt kernel.
 * Reports total milliseconds and launch counts since the last reset. */
int tri_domain_set_timing(tri_domain* d, int32_t enabled);
int tri_domain_get_timing(tri_domain* d, double* flux_ms, int32_t* flux_launches, double* wetdry_ms,
                          int32_t* wetdry_launches);
/* Interior cells of the flux tiles and wet-dry bands that advance() calls
 * computed since the last tri_domain_set_timing (steps run x interior cells,
 * less the cells of tiles skipped as dry: tiles whose cells and neighbours
 * hold only zeros, whose update is exactly the identity).  No reference
 * counterpart (the reference updates every cell every step). */
int tri_domain_get_work(tri_domain* d, int64_t* flux_cells, int64_t* wetdry_cells);
/* Test hook for the bounded device waits (no reference counterpart; the
 * reference's kernels never wait).  While polls > 0, every step's wet-dry
 * launch also waits, at most 'polls' polls, on a barrier that nothing
 * completes; the wait gives up, the launch records a device status, and
 * tri_domain_advance returns TRI_E_TIMEOUT once the steps have run (the
 * computation itself is untouched).  0 (the default) turns it off. */
int tri_domain_set_wait_test(tri_domain* d, uint32_t polls);

/* Launch-shape autotuner of the flux kernel.  Runs trial_steps steps of the
 * domain's own state for every candidate (register budget x tile height),
 * keeps the fastest, and restores the state and clock, so the simulation is
 * unchanged.  The choice stays with the domain. */
typedef struct tri_tuning {
  int32_t variant;        /* register-budget variant of the flux kernel */
  int32_t rows_per_tile;  /* tile height (rows per warp tile, 30 columns wide) */
  int32_t candidates;     /* how many shapes were timed */
  int32_t flux_blocks;    /* blocks in the flux kernel's grid */
  double ms_per_step;     /* best trial time per step */
} tri_tuning;
int tri_domain_autotune(tri_domain* d, int32_t trial_steps, tri_tuning* out);
int tri_domain_get_tuning(tri_domain* d, tri_tuning* out);
/* Sets the flux kernel's launch shape directly (variant 0..2, rows per tile >= 1). */
int tri_domain_set_tuning(tri_domain* d, int32_t variant, int32_t rows_per_tile);

/* Self-check of the exact divisions by a reused divisor used in the kernels:
 * for each of n pseudo-random indices from 'seed', one (a, b) pair over the
 * magnitudes the step produces and one over all finite dividends (subnormals
 * and signed zeros included) and divisors 1e-30 .. 1e30; counts quotients
 * that differ in any bit from IEEE a/b. */
int tri_selftest_division(int64_t n, uint64_t seed, int64_t* mismatches);

/* ---- batches of member domains ------------------------------------------ */
/* Ensemble members advanced together on one GPU.  Replaces the reference's
 * ensemble runs (src/Ensify.h:43-72), which give every member its own group
 * of MPI ranks and processes.  Each batched step moves every member by one of
 * its own time steps (own dt policy, own events); one launch per kernel type
 * covers all members, the flux kernel taking tiles from a single queue over
 * all members.  Members stay tri_domain objects: upload, download, forcing,
 * observe and set_clock work on them between batch advances.  Members must
 * share one precision; closed, open and external-boundary edges all batch.
 * A member whose forcing changes after tri_batch_create needs a new batch. */
typedef struct tri_batch tri_batch;
typedef struct tri_batch_progress {
  int32_t steps;               /* most steps any member took */
  int32_t members_with_events; /* members that stopped on an event */
  int32_t members_ended;       /* members with simtime >= sim_duration */
  int32_t reserved;
  int64_t cell_updates;        /* sum over members of steps x interior cells */
} tri_batch_progress;
/* stream: cudaStream_t for the batched launches, NULL = the batch makes one. */
int tri_batch_create(int32_t nmembers, tri_domain* const* members, void* stream, tri_batch** out);
int tri_batch_destroy(tri_batch* b);
/* Replaces the member list (0 members allowed; same rules as create).  For a
 * request loop that admits and retires domains between advances. */
int tri_batch_set_members(tri_batch* b, int32_t nmembers, tri_domain* const* members);
/* Advances every member until it raises an event (its clock then halts, as in
 * tri_domain_advance) or until max_steps batched steps have run.  Members
 * already at their end take no steps.  Blocks until done. */
int tri_batch_advance(tri_batch* b, int32_t max_steps, tri_batch_progress* out);
/* Split form for a host loop that works while the GPU steps: launch queues
 * 'steps' batched steps and returns at once (members that end or raise an
 * event halt on the device and idle for the rest); wait blocks until they are
 * done and reads the members' clocks.  Between the two, the members and the
 * batch must not be touched; other batches may launch. */
int tri_batch_launch(tri_batch* b, int32_t steps);
int tri_batch_wait(tri_batch* b, tri_batch_progress* out);
/* Launch-shape autotuner of the batched flux kernel; members' states, maximum
 * depths and clocks are restored afterwards. */
int tri_batch_autotune(tri_batch* b, int32_t trial_steps, tri_tuning* out);
/* How batched steps are launched (no reference counterpart).
 * TRI_BATCH_GRAPHS (default): per batched step one launch per kernel type
 * (clock, flux, forcing waves, wet-dry/dt), 8 steps captured as a CUDA graph.
 * TRI_BATCH_SINGLE_LAUNCH: one persistent launch runs up to 32 batched
 * steps; its blocks take work items (a member's clock, four flux tiles, a
 * member's forcing, a wet-dry block) in a fixed order and each item waits,
 * bounded, only for the items of its own member it depends on, so members
 * advance without any grid-wide barrier.  Both compute exactly what every
 * member computes alone.  A dependency wait that gives up makes the advance
 * return TRI_E_TIMEOUT. */
enum { TRI_BATCH_GRAPHS = 0, TRI_BATCH_SINGLE_LAUNCH = 1 };
int tri_batch_set_mode(tri_batch* b, int32_t mode);
/* Test hook of the single-launch mode (no reference counterpart): with
 * polls > 0 the first clock item of the next advances also waits for a count
 * that no item ever reaches, giving up after `polls` polls, so the advance
 * returns TRI_E_TIMEOUT with nothing else wrong (every other wait then gives
 * up at once; the members' states are not valid afterwards).  0 turns it
 * off.  No effect in TRI_BATCH_GRAPHS mode. */
int tri_batch_set_wait_test(tri_batch* b, uint32_t polls);
int tri_batch_set_tuning(tri_batch* b, int32_t variant, int32_t rows_per_tile);

/* ---- reference kernels (FP64, device pointers) -------------------------- */
/* Each launches on 'stream' (cudaStream_t, NULL = default stream) and does not
 * synchronize.  size/rows/cols as in the reference; 'stream' is added last. */
int tri_kernel_compute_dt_and_sqrt_f64(int size, double dx, const double* qx, const double* qy, const double* h,
                                       double* sqrth, double* dt_out, double cn, double hextra, void* stream);
/* find_min_dt: writes the minimum into *min_out (a DEVICE double) with one
 * kernel and no scratch memory. */
int tri_kernel_find_min_dt_f64(int size, const double* dt, double* min_out, void* stream);
int tri_kernel_flux_x_f64(int size, int nrows, int ncols, double dx, double dt, const double* h, const double* qx,
                          const double* qy, const double* dem, const double* sqrth, double* rhsh0, double* rhsh1,
                          double* rhsqx0, double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra,
                          void* stream);
int tri_kernel_flux_y_f64(int size, int nrows, int ncols, double dx, double dt, const double* h, const double* qx,
                          const double* qy, const double* dem, const double* sqrth, double* rhsh0, double* rhsh1,
                          double* rhsqx0, double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra,
                          void* stream);
int tri_kernel_update_cells_f64(int size, int nrows, int ncols, double dt, double* h, double* qx, double* qy,
                                const double* dem, const double* n, double* rhsh0, double* rhsh1, double* rhsqx0,
                                double* rhsqx1, double* rhsqy0, double* rhsqy1, double hextra, void* stream);
int tri_kernel_update_runoff_f64(int size, int nrows, int ncols, double dt, const int32_t* runoff_id,
                                 int index_row_runoff, int n_rows_runoff, const double* runoff_intensity, double* h,
                                 double* qx, double* qy, double hextra, void* stream);
/* compute_flow: sources that share a cell are applied in source order. */
int tri_kernel_compute_flow_f64(int size, const double* hyd_time, const double* hyd_val, double dx, double dt,
                                double simtime, int idx_low, int idx_high, double* h, const int32_t* pos,
                                void* stream);
int tri_kernel_copy_info_to_exterior_boundaries_west_east_f64(int size, int nrows, int ncols, double* h, double* qx,
                                                              double* qy, void* stream);
int tri_kernel_copy_info_to_exterior_boundaries_north_south_f64(int size, int nrows, int ncols, double* h,
                                                                double* qx, double* qy, int rank,
                                                                int total_process, void* stream);
/* compute_extbc_values: cells that touch the same cell (corners shared by two
 * segments, repeated cells) are applied in index order, as the reference's
 * serial build does; to schedule them the entry reads the cell list back to
 * the host, so it synchronizes 'stream'.  The order is cached per host thread
 * and device, in device memory allocated on first use and grown for longer
 * lists (freed when the thread exits). */
int tri_kernel_compute_extbc_values_f64(int size, int nrows, int ncols, double dt, double* h, double* qx, double* qy,
                                        const double* dem, const double* n, const int32_t* relative_index,
                                        const int32_t* extbctype, const int32_t* start_index,
                                        const int32_t* nrows_vars, const double* extbcvar1, const double* extbcvar2,
                                        double simtime, int rank, int total_process, void* stream);
/* No-alloc variant of tri_kernel_compute_extbc_values_f64; it has no
 * counterpart in the reference.  Same arguments, same results, and it also
 * synchronizes 'stream'.  It allocates no device memory: the application
 * order is kept in a fixed array inside the library of
 * TRI_NOALLOC_EXTBC_MAX_CELLS entries (256 KiB), and a longer cell list is
 * rejected with TRI_E_INVALID.  For callers that cannot allocate device
 * memory inside their time loop: a host that claimed the GPU's free memory
 * before the loop (a memory pool or caching allocator in the same process)
 * would see cudaMalloc fail mid-run, and cudaMalloc/cudaFree synchronize the
 * whole device.  The first call on each device looks up the array's address
 * (which may load the library's device code); make it before any stream
 * capture.  The array is shared by every call on a device: calls that
 * overlap in time (from other host threads, or while kernels of an earlier
 * call with another cell list still run on another stream) race on it.  A
 * call that writes a new order waits for the copy to land before it returns,
 * so a later call with the same list, on any stream, finds it in place. */
#define TRI_NOALLOC_EXTBC_MAX_CELLS 65536
int tri_kernel_compute_extbc_values_noalloc_f64(int size, int nrows, int ncols, double dt, double* h, double* qx,
                                                double* qy, const double* dem, const double* n,
                                                const int32_t* relative_index, const int32_t* extbctype,
                                                const int32_t* start_index, const int32_t* nrows_vars,
                                                const double* extbcvar1, const double* extbcvar2, double simtime,
                                                int rank, int total_process, void* stream);
int tri_kernel_wet_dry_f64(int size, int nrows, int ncols, double dt, const double* h, double* qx, double* qy,
                           const double* dem, double* max_h, double hextra, int mpi_tasks, void* stream);
int tri_kernel_copy_observation_points_f64(int size, const double* arr, double* obs_arr,
                                           const int32_t* relative_index, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TRITON_B200_H */
