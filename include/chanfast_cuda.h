/*
 * chanfast_cuda -- B200 (sm_100a) FP64 implementation of the RK3 substep of the
 * staggered-grid channel-flow DNS of nasilemakbox/ubiquitous-spoon, behind a
 * plain C ABI.  Two shared libraries implement it:
 *
 *   libchanfast_cuda.so  device engine + this instance API (cf_*)
 *   libchanfast.so       drop-in drivers chanfast2 / chanfast4 / channel2 /
 *                        channel4 in C, on top of the instance API
 *
 * Conventions
 *  - Every cf_* function returns an int status: CF_OK (0) or a negative CF_E*
 *    code; nothing aborts the process.  cf_strerror() names a code.
 *  - Fields cross the ABI as flat FP64 arrays in one of two layouts:
 *      CF_LAYOUT_PADDED   [nx+2*ngx][ny+2*ngy][nz+2*ngz], wall-normal index
 *                         fastest, ghosts included -- the reference's field
 *                         layout (d3tensor.c:9-42, chanfast.c:105-137)
 *      CF_LAYOUT_INTERIOR [nx][ny][nz], interior only -- the reference's
 *                         restart-file layout (io.c:211-297)
 *    Axes are the reference's: x streamwise (periodic), y spanwise (periodic),
 *    z wall-normal (walls, cosine-stretched).
 *  - An instance owns its device memory and is bound to the CUDA device that
 *    was current at cf_create.  Calls on one instance must be serialised by
 *    the caller; distinct instances may be driven from distinct threads.
 */
#ifndef CHANFAST_CUDA_H
#define CHANFAST_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CF_OK = 0,
    CF_EINVAL = -1,      /* bad argument or unsupported configuration */
    CF_ENOMEM = -2,      /* device or host allocation failed */
    CF_ECUDA = -3,       /* a CUDA runtime call failed */
    CF_EPIVOT = -4,      /* zero pivot in a band factorisation */
    CF_ENONFINITE = -5,  /* the state went NaN or Inf (see cf_sync) */
    CF_EIO = -6,         /* restart / log file error (drivers) */
    CF_ETIMEOUT = -7     /* a kernel gave up (after about a second) waiting for
                            one of its own asynchronous copies; the substep's
                            results are invalid (see cf_sync) */
};

enum { CF_U = 0, CF_V = 1, CF_W = 2, CF_C = 3, CF_P = 4 };
enum { CF_LAYOUT_PADDED = 0, CF_LAYOUT_INTERIOR = 1 };

/* Arguments of chanfast2 / chanfast4 / channel2 / channel4 (reference
 * chanfast.h:1-21, channel.h:1-21) that determine one run, plus the scheme
 * that tells the two driver families apart; p_row = p_col = 1,
 * it/nt/istat/cfl belong to the driver.  Zero-initialise the struct: a zero
 * scheme is CF_SCHEME_CHANFAST. */
typedef struct cf_config {
    int order;               /* 2 (chanfast2) or 4 (chanfast4) */
    int nx, ny, nz;          /* interior grid */
    int ngx, ngy, ngz;       /* ghost widths of the padded layout; ngz must be 3 */
    int uvolavgmode;         /* 1: constant flow rate (chanfast.c:515) */
    int cvolavgmode;         /* 1: constant scalar mean (chanfast.c:602) */
    double lx, ly, lz;       /* box; lz = channel height */
    double dt, nu, prandtl, dpdx;
    double want_uvolavg, want_cvolavg;
    double setuframe, setvframe;      /* Galilean frame (chanfast.c:61-64) */
    double betg_x, betg_y, betg_z;    /* buoyancy */
    int scheme;              /* CF_SCHEME_CHANFAST (0) or CF_SCHEME_CHANNEL (1) */
} cf_config;

/* Time-integration schemes.  CHANFAST: diffusion implicit in z only, x-y
 * diffusion explicit (chanfast2/chanfast4, chanfast.c:395-656).  CHANNEL:
 * diffusion fully implicit, solved per (kx, ky) wavenumber after a 2-D FFT
 * (channel2/channel4, channel.c:392-690 / 1342-1640); needs nx in
 * {64, 128, 256, 512} and, at order 4, nz >= 8. */
#define CF_SCHEME_CHANFAST 0
#define CF_SCHEME_CHANNEL 1

typedef struct cf_instance cf_instance;

/* Create / destroy an instance on the current CUDA device.  Replaces the
 * setup part of chanfast2/chanfast4 (chanfast.c:85-301): grid metrics,
 * field allocation, FFT plans, line-solve factorisations.  `stream` is a
 * cudaStream_t (NULL: the instance creates its own). */
int cf_create(const cf_config *cfg, void *stream, cf_instance **out);
int cf_destroy(cf_instance *inst);

/* Copy a field in or out.  Host pointers; `layout` as above.  cf_get_field
 * fills the x/y ghosts of the padded layout periodically and returns the
 * wall-normal ghost rows as they are held on the device.  Replaces io_read /
 * io_write + ghostz_pad/ghostz_truncate (io.c:211-297, ghostz.c:152-177).
 * CF_P is read-only. */
int cf_set_field(cf_instance *inst, int field, const double *host, int layout);
int cf_get_field(cf_instance *inst, int field, double *host, int layout);

/* Seeded initial state, generated on the device: laminar Poiseuille u plus a
 * uniform random perturbation of amplitude amp*1.5 on u, v, w (SplitMix64 of
 * seed/field/global index), scalar -0.5 + z/2 plus c_amp noise, then made
 * discretely divergence-free by one projection with dt = 1 (cases.c:426-470). */
int cf_init_fields(cf_instance *inst, unsigned long long seed, double amp, double c_amp);

/* Advance `nsub` RK3 substeps (3 per time step) -- the body of
 * chanfast.c:395-656 (order 2) / 1319-1580 (order 4) -- asynchronously on
 * the instance stream.  The substep counter and the previous-stage
 * right-hand sides persist across calls. */
int cf_step(cf_instance *inst, int nsub);

/* Same as cf_step for nsteps full RK3 time steps, replaying a CUDA graph of
 * two time steps (6 substeps) captured on first use; a leftover odd step and
 * any substeps needed to reach the start of a time step run as cf_step. */
int cf_step_graph(cf_instance *inst, int nsteps);

/* Wait for all work of the instance.  Returns CF_ENONFINITE once a substep
 * has found the bulk mean of u or c (a sum over every interior point) NaN or
 * Inf: a blown-up or NaN-seeded state is detected within one substep, and
 * within two for v, w and p, which feed u in the next substep.  The
 * reference has no such check (its check(), check.h:8-12, aborts only on
 * allocation, order and pivot failures).  Returns CF_ETIMEOUT once a
 * kernel has given up waiting for one of its own asynchronous copies.  The
 * flags stay set until cf_set_field or cf_init_fields loads new fields. */
int cf_sync(cf_instance *inst);

/* Per-substep log rows (10 doubles each): mdpdx, nu du/dz bottom, top, bulk
 * velocity, centreline velocity, then dcdt and the same four scalar
 * statistics -- the values chanfast appends to pstat.dat / cstat.dat
 * (chanfast.c:525-528, 612-615).  Returns the number of rows written into
 * `out` (at most max_rows, most recent last) or a negative status
 * (CF_ENONFINITE as for cf_sync). */
long cf_get_log(cf_instance *inst, double *out, long max_rows);

/* Number of substeps done so far. */
long cf_substeps_done(const cf_instance *inst);

/* max |div u| over the interior cells with the reference operator
 * divergence{2,4} (pressure.c:40-117), evaluated on the device. */
int cf_max_divergence(cf_instance *inst, double *out);

/* Same result as cf_max_divergence, without allocating anything.  It has no
 * counterpart in the reference; it exists for callers that cannot call
 * cudaMalloc or cudaFree at the point where they check the flow, e.g. a
 * serving loop that has budgeted the whole device memory to resident
 * instances (an allocation there can fail), or a monitor that runs between
 * the steps of live instances on other streams (cudaFree synchronises the
 * whole device and would stall them).  The partial maxima live in a
 * file-scope device array of one double per interior k-plane, at most 8191
 * planes: an instance with nz > 8191 is rejected with CF_EINVAL before any
 * work is queued.  The array is shared by every call on a device,
 * keeps the last call's contents and needs no zeroing (each call rewrites
 * every entry it reads); calls that overlap on one GPU, e.g. for two
 * instances on different streams, race on it.  The first call on each
 * device looks up the array's device address with that device current;
 * make that first call before any stream capture. */
int cf_max_divergence_noalloc(cf_instance *inst, double *out);

/* CFL number of the current velocity field for time step dt, as get_cfl
 * (get.c:390-416): max over interior cells of |u| dt/dx, |v| dt/dy,
 * |w| dt/dzph, evaluated on the device; synchronises the instance. */
int cf_cfl(cf_instance *inst, double dt, double *cfl);

/* Change the time step (rebuilds the per-substep line-solve factorisations;
 * used by the drivers when cflmode == 1, chanfast.c:385-391). */
int cf_set_dt(cf_instance *inst, double dt);

/* Device pointer of a field in the engine layout [n2][nx][ny] (k slowest),
 * for callers that keep data on the device. */
int cf_device_field(cf_instance *inst, int field, double **dev_ptr, long long *n_elems);

/* Run nsub substeps with CUDA events between the kernel groups on the
 * instance stream and return the summed device time of each group (ms) in
 * ms[CF_NKERNEL_GROUPS], in this order:
 *   0 ghosts (apply_bc), 1 rhs with the forward sweeps of the implicit
 *   solves, 2 back substitution of u, v, c and w (one launch), 3 mass-flux
 *   control u, 4 scalar-mean control c, 5 divergence + x FFT, 6 y FFT,
 *   7 Poisson, 8 inverse y FFT, 9 inverse x FFT, 10 projection.
 * With power-of-two ny the y transforms run inside the Poisson launch
 * (k_poisson_fft): groups 6 and 8 are then empty and 7 holds all three.
 * Synchronises after every substep (timing only). */
#define CF_NKERNEL_GROUPS 11
int cf_profile(cf_instance *inst, int nsub, double *ms);

/* Number of kernel launches the engine issues per substep. */
int cf_launches_per_substep(const cf_instance *inst);

/* 1 when the instance runs its y transforms and Poisson solve as one launch
 * (k_poisson_fft), 0 when as three, CF_EINVAL for a null instance.  The
 * fused launch needs ny = 256 or 512; it is taken by default where its one
 * block per kx gives the GPU enough blocks (nx/2 + 1 at least half the SM
 * count).  CF_FUSE_PRESSURE=1 in the environment at creation takes it
 * wherever supported, CF_FUSE_PRESSURE=0 never. */
int cf_pressure_fused(const cf_instance *inst);

/* Test hook for the bounded waits: with on != 0, the instance's fused pressure
 * launches (cf_pressure_fused) leave their forward row copies unissued, so
 * that the first wait of every block runs out after about a second; the
 * kernel then finishes without data and cf_sync returns CF_ETIMEOUT.  Nothing
 * faults or hangs.  The hook stays until called with on = 0; the status
 * clears with cf_set_field / cf_init_fields. */
int cf_debug_stall_copies(cf_instance *inst, int on);

const char *cf_strerror(int status);

/* ------------------------------------------------------------------------
 * Statistics written every istat steps by the drivers (chanfast.c:658-857,
 * get.c), computed on the device; output to host arrays, synchronous.
 * Profiles have n2 = nz + 2*ngz entries (wall-normal rows, ghosts included),
 * spectra (nx/2+1)*n2*2 and (ny/2+1)*n2*2 doubles laid out [i][k][re, im].
 * Sums run in a fixed order different from the reference's serial loops,
 * so results agree to rounding.
 * ------------------------------------------------------------------------ */
int cf_xy_avg(cf_instance *inst, int field, double *avg);                 /* get_xy_avg */
int cf_xy_corr(cf_instance *inst, int fa, int fb, double *corr);          /* get_xy_corr */
int cf_xy_moment(cf_instance *inst, int field, double en, double *mom);   /* get_xy_moment */
int cf_xy_spec(cf_instance *inst, int fa, int fb, double *specx, double *specy);  /* FFT3D_FWD + get_xy_spec */
int cf_z_coords(const cf_instance *inst, double *zp, double *zw);         /* get_z_at_p / get_z_at_w */

/* ------------------------------------------------------------------------
 * Batches: many independent instances stepped together, one kernel launch
 * per stage of the substep covering all of them (per-instance work records
 * in device memory: geometry, arguments, own grid).  Members may differ in
 * grid size, order and physical parameters; they must use
 * CF_SCHEME_CHANFAST and live on one device.  Each member's results are the
 * same, bit for bit, as stepping it alone with cf_step.
 *
 * cf_batch_step: advance every member by nsub substeps on `stream` (NULL:
 * the first member's stream), recording the launches on the spot.  Ordered
 * after, and before, work on the members' own streams.
 *
 * cf_batch_create / cf_batch_run: record a two-step cycle once (uploaded
 * per-instance records) and replay it as a CUDA graph for nsteps RK3 steps
 * (an odd step runs eagerly).  While in a batch, a member must not be stepped
 * otherwise or have its dt changed; cf_batch_run then returns CF_EINVAL and
 * the batch must be created again.  Fields, logs and the other cf_* calls of
 * a member remain available (after cf_batch_sync).
 * ------------------------------------------------------------------------ */
typedef struct cf_batch cf_batch;
int cf_batch_step(cf_instance **members, int n, int nsub, void *stream);
int cf_batch_create(cf_instance **members, int n, void *stream, cf_batch **out);
/* cf_batch_create with options: CF_BATCH_NO_TUNE skips the launch-shape
 * trials (a member set tuned before keeps its cached shape, others take the
 * defaults) -- for a caller that forms a new batch whenever its member set
 * changes, as the serving loop does. */
#define CF_BATCH_NO_TUNE 1
int cf_batch_create_opts(cf_instance **members, int n, void *stream, int flags, cf_batch **out);
int cf_batch_run(cf_batch *batch, int nsteps);
int cf_batch_sync(cf_batch *batch);
/* Batched launches per substep of the whole batch (all members together). */
int cf_batch_launches_per_substep(const cf_batch *batch);
int cf_batch_destroy(cf_batch *batch);

/* ------------------------------------------------------------------------
 * Launch-shape autotuning.  Three kernels run with any of a few block shapes
 * and give the same results bit for bit: the back substitution (columns per
 * block: 64, 128), the Poisson / spectral Helmholtz band solve (column
 * pairs per block: 64, 128) and the projection (block of j by i: 32x2, 32x4,
 * 32x8, 64x2).  cf_create times the candidates on the new instance (before
 * it holds state) and keeps the fastest; cf_batch_create does the same on
 * the batch's own launches with their outputs in scratch memory.  Results
 * are cached per configuration (per member set for a batch) for the process
 * and, when the environment variable CF_TUNE_CACHE names a file, across
 * processes (one line per key: "key solve pois proj_bx proj_by").
 * cf_batch_step uses the cached shape of its member set, else the defaults.
 *
 * cf_set_tuning(0) (or CF_TUNE=0 in the environment) turns tuning off: new
 * instances and batches use the default shapes 128, 128, 32x4.
 * A shape is four ints: solve threads, Poisson threads, projection block x,
 * projection block y.  cf_set_launch_shape rejects shapes outside the
 * candidates with CF_EINVAL.
 * ---------------------------------------------------------------------- */
int cf_set_tuning(int on);
int cf_get_launch_shape(const cf_instance *inst, int shape[4]);
int cf_set_launch_shape(cf_instance *inst, const int shape[4]);
int cf_batch_get_launch_shape(const cf_batch *batch, int shape[4]);

/* ------------------------------------------------------------------------
 * Serving: a request loop over the instance and batch calls.
 *
 * cf_instance_bytes: device memory an instance of this configuration holds
 * (fields, right-hand sides, spectrum, solver scratch, tables, the staging
 * buffer of one padded field); 0 for an invalid configuration.
 *
 * cf_serve: serve n requests that arrive at arrival_s seconds after the call
 * (non-decreasing).  In arrival order, a request is admitted (instance
 * created, seeded initial state, cf_init_fields) once it has arrived, while
 * the resident instances' cf_instance_bytes plus its own stay within
 * hbm_budget_bytes and fewer than max_active are resident.  Each round
 * advances every resident solve by min(quantum, steps left) RK3 steps with
 * cf_batch_step (new arrivals join at the next round); a solve that has run
 * its steps is retired at once: on_done(index, inst, user) may read its
 * fields, then its memory is released (inst is NULL for a request that
 * failed; its status says why).  A solve whose state goes NaN or Inf
 * (cf_sync) is retired at the end of that round with status CF_ENONFINITE
 * while the others run on.  Requests use CF_SCHEME_CHANFAST.  Each
 * solve's result is the same, bit for bit, as stepping it alone with
 * cf_batch_step.  Times in results are seconds after the call.
 * ------------------------------------------------------------------------ */
typedef struct cf_request {
    cf_config cfg;
    unsigned long long seed;     /* cf_init_fields arguments */
    double amp, c_amp;
    int nsteps;                  /* RK3 steps to run */
    double arrival_s;
} cf_request;

typedef struct cf_result {
    double admit_s, finish_s;
    int status;
    long long steps_done;
} cf_result;

typedef void (*cf_done_fn)(int index, cf_instance *inst, void *user);

unsigned long long cf_instance_bytes(const cf_config *cfg);
int cf_serve(const cf_request *reqs, int n, double hbm_budget_bytes, int max_active, int quantum,
             void *stream, cf_done_fn on_done, void *user, cf_result *results);

/* ------------------------------------------------------------------------
 * Drop-in drivers (libchanfast.so).  Same names and arguments as the
 * reference (chanfast.h:1-21, called at main.c:56-60); they read
 * outputdir/{u,v,w,c}_it<it>.dat, run nt - it time steps on the current
 * CUDA device, append outputdir/cfl.dat, pstat.dat and cstat.dat, and write
 * outputdir/{u,v,w,c}_it<N>.dat every istat steps.  One GPU holds the whole
 * grid: a single process accepts any p_row x p_col (main.c passes 2 x 2,
 * main.c:9-10) with a note on stderr; under an MPI launcher with N > 1
 * ranks (read from the launcher's environment: Open MPI, MPICH / Hydra,
 * PMIx, Slurm), p_row * p_col must be N as in the reference
 * (chanfast.c:87), rank 0 runs the whole grid and writes every file, and
 * the other ranks return at once.  The reference main.c therefore builds
 * and runs unchanged against this library.  A NaN / Inf state stops the run
 * with CF_ENONFINITE (see cf_sync).
 * The reference returns nothing and aborts on error; these print the
 * failing status to stderr and return.  chanfast2_status / chanfast4_status
 * return it instead.  channel2 / channel4 (channel.h:1-21) are the same with
 * the fully implicit scheme (CF_SCHEME_CHANNEL and its size limits).
 * ------------------------------------------------------------------------ */
void chanfast2(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
               int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
               double dt, double want_cfl, int cflmode, double nu, double prandtl,
               double dpdx, double want_uvolavg, int uvolavgmode,
               double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
               double betg_x, double betg_y, double betg_z);
void chanfast4(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
               int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
               double dt, double want_cfl, int cflmode, double nu, double prandtl,
               double dpdx, double want_uvolavg, int uvolavgmode,
               double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
               double betg_x, double betg_y, double betg_z);
int chanfast2_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                     int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                     double dt, double want_cfl, int cflmode, double nu, double prandtl,
                     double dpdx, double want_uvolavg, int uvolavgmode,
                     double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                     double betg_x, double betg_y, double betg_z);
int chanfast4_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                     int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                     double dt, double want_cfl, int cflmode, double nu, double prandtl,
                     double dpdx, double want_uvolavg, int uvolavgmode,
                     double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                     double betg_x, double betg_y, double betg_z);
void channel2(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
              int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
              double dt, double want_cfl, int cflmode, double nu, double prandtl,
              double dpdx, double want_uvolavg, int uvolavgmode,
              double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
              double betg_x, double betg_y, double betg_z);
void channel4(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
              int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
              double dt, double want_cfl, int cflmode, double nu, double prandtl,
              double dpdx, double want_uvolavg, int uvolavgmode,
              double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
              double betg_x, double betg_y, double betg_z);
int channel2_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                    int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                    double dt, double want_cfl, int cflmode, double nu, double prandtl,
                    double dpdx, double want_uvolavg, int uvolavgmode,
                    double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                    double betg_x, double betg_y, double betg_z);
int channel4_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                    int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                    double dt, double want_cfl, int cflmode, double nu, double prandtl,
                    double dpdx, double want_uvolavg, int uvolavgmode,
                    double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                    double betg_x, double betg_y, double betg_z);

#ifdef __cplusplus
}
#endif

#endif /* CHANFAST_CUDA_H */
