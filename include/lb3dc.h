/*
 * lb3dc.h -- C ABI of the B200 (sm_100a) implementation of LB3D's
 * per-timestep hot path.
 *
 * The entry points mirror the calls LB3D's time loop makes
 * (code/lb3d_time_loop.F90:58-92):
 *
 *     lb3d_force_apply(6); lb3d_bc_apply(6)      -> lb3dc_force_apply, lb3dc_bc_apply
 *     lb3d_advection                             -> lb3dc_advection
 *     lb3d_bc_apply(8); lb3d_force_apply(8)      -> lb3dc_bc_apply, lb3dc_force_apply
 *     lb3d_collision                             -> lb3dc_collision
 *
 * plus the state transfer a Fortran ISO_C_BINDING shim needs to hand its
 * lattice (whole_N, code/lb3d_lattice.F90:235-239,274-287) to the device and
 * back.  Plain pointers and sizes only; every function returns an int status
 * (0 = LB3DC_OK, negative = error) and the message of the last error of a
 * handle is available from lb3dc_last_error.
 *
 * Threading: one host thread per handle; each handle owns one CUDA stream.
 * Calls are asynchronous on that stream except the ones documented as
 * synchronising (downloads, reductions, dumps, lb3dc_sync).
 */
#ifndef LB3DC_H
#define LB3DC_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define LB3DC_OK 0
#define LB3DC_EINVAL (-22)   /* bad argument or unsupported parameter set */
#define LB3DC_ENOMEM (-12)   /* device or host allocation failed          */
#define LB3DC_ECUDA (-5)     /* a CUDA runtime call failed                */
#define LB3DC_ETIMEOUT (-110)/* a bounded device-side wait gave up        */
#define LB3DC_ENAN (-33)     /* non-finite populations detected           */
#define LB3DC_ENOTSUP (-95)  /* valid request this build does not support */
#define LB3DC_ESTATE (-71)   /* call out of order (e.g. no state loaded)  */

/* ---- precision modes ------------------------------------------------- */
#define LB3DC_FP64 0         /* plain drop-in: FP64 populations, FP64 math */
#define LB3DC_FP32_DEV 1     /* FP32 storage of n - w_i rho0, FP32 collide */

/*
 * Hot-path parameters: the &fixed_input / &variable_input / &lbe_input
 * scalars that the per-step path reads (code/lb3d_config.F90:44-297), after
 * the reference's derived-value rules (rock_colour -> rock_colour_r/_b,
 * g_accn_max* defaults; code/lb3d_config.F90:661-664,931-933).
 * Component order: red, blue, surfactant.  ncomp is 2 (the reference's
 * -DNOSURFACTANT build) or 3 (its default ternary build).
 */
typedef struct lb3dc_params {
  int nx, ny, nz, ncomp;
  double tau_r, tau_b, tau_s, tau_d;
  double amass_r, amass_b, amass_s;
  double g_br, g_bs, g_ss, g_wr, g_wb, tau_wr, tau_wb;
  double beta, d_0;
  double g_accn, g_accn_x, g_accn_y;
  int g_accn_min, g_accn_max, g_accn_min_x, g_accn_max_x, g_accn_min_y, g_accn_max_y;
  double shear_u, shear_omega;
  int boundary_cond, inv_fluid;
  double rock_colour_r, rock_colour_b;
  int bdist;    /* must be 2 (the third-order equilibrium)               */
  int restore;  /* 1 when the state comes from a checkpoint (init_cond 7) */
  /* Zou-He boundaries on the z planes (boundary_cond != 0).  Flux
   * boundaries (inv_fluid = 12, code/lb3d_invasion.F90:2143-2457): inv_type
   * selects the closure (0, 1 or -1: pr/pg/pb are fluxes rather than
   * velocities), and pr, pg, pb are the red, surfactant and blue inflow
   * values.  Density boundaries (inv_fluid = 11, :1459-1796): fr, fb are
   * the red and blue densities at z = 1, pr, pb those at z = nz.  fr, fg,
   * fb default to 1.0, 0.1, 0.5 (code/lb3d_config.F90:169).  Both
   * precisions; the FP32 path runs them with the staged split strategy.  */
  int inv_type;
  double pr, pg, pb;
  double fr, fg, fb;
  int precision;/* LB3DC_FP64 or LB3DC_FP32_DEV                           */
  double rho0;  /* reference density of the FP32 deviation storage        */
} lb3dc_params;

typedef struct lb3dc_handle lb3dc_handle;

/* ---- lifetime --------------------------------------------------------- */
/* Validates p (the fatal combinations of code/lb3d_compatibility.F90:105-111
 * are rejected with LB3DC_EINVAL), allocates the device lattice on the
 * current CUDA device.  Replaces the allocation of whole_N
 * (code/lb3d_lattice.F90:274-287). */
int lb3dc_create(const lb3dc_params *p, lb3dc_handle **out);
int lb3dc_destroy(lb3dc_handle *h);
/* Copies the last error message of h (or of the last failed lb3dc_create
 * when h is NULL) into buf; returns the status code of that error. */
int lb3dc_last_error(const lb3dc_handle *h, char *buf, int len);
/* Bytes of device memory the handle holds. */
long long lb3dc_device_bytes(const lb3dc_handle *h);
/* Device bytes a handle with these parameters would allocate. */
long long lb3dc_footprint(const lb3dc_params *p);

/* ---- state transfer (synchronising) ----------------------------------- */
/*
 * Loads a restored lattice and performs what the reference does after a
 * restore: zero populations at rock sites and colour them
 * (lbe_init_rock_colour, code/lb3d_ic_rock.F90:146-189), then
 * lb3d_bc_init(4) (code/lb3d_bc.F90:48-90: the Lees-Edwards shear_u
 * correction and shear_sum bookkeeping).
 *   n    : [ncomp][19][nz][ny][nx] populations, x fastest
 *   db   : [3][nz][ny][nx] surfactant dipoles (ternary; NULL for binary)
 *   rock : [nz][ny][nx] rock_state (nonzero = rock; NULL = no rock)
 *   shear_sum : value from the checktopo file; nt : restored time step.
 */
int lb3dc_upload_state(lb3dc_handle *h, const double *n, const double *db, const double *rock,
                       double shear_sum, int nt);
/* Interior state after the last completed call.  Any pointer may be NULL.
 *   n, db as above; rho: [ncomp][site]; mom: [ncomp][3][site] (the
 *   reference's u_* fields hold momentum); da: [3][site]. */
int lb3dc_download_state(lb3dc_handle *h, double *n, double *db, double *rho, double *mom,
                         double *da);
/*
 * The reference's own arena: whole_N(0:nx+1,0:ny+1,0:nz+1) of type lbe_site
 * (code/lb3d_lattice.F90:35-83), sequence layout per site
 *   per component: n(19), rho, u(3), rock_colour   then (ternary) da(3),
 *   db(3)                                           then rock_state
 * i.e. 49 (binary) or 79 (ternary) doubles per site, x fastest, halo 1.
 * upload reads n, db and rock_state of the interior sites; download writes
 * n, rho, u, rock_colour, da, db and rock_state of the interior sites.
 */
int lb3dc_upload_sites(lb3dc_handle *h, const double *whole_N, double shear_sum, int nt);
int lb3dc_download_sites(lb3dc_handle *h, double *whole_N);

/* ---- the time-loop stages (asynchronous) ------------------------------ */
/* code/lb3d_force.F90:98-121: stages 6, 8, 10 are no-ops in the default
 * build; kept for call-for-call parity. */
int lb3dc_force_apply(lb3dc_handle *h, int stage);
/* code/lb3d_bc.F90:95-155.  Stage 6 advances the time step counter and,
 * under Lees-Edwards, updates shear_u, shear_sum and the plane offset and
 * builds the x-halo; stage 8 applies the inflow boundaries of the z planes
 * (lbe_invade: Zou-He flux inv_fluid 12, Zou-He density 11, recolouring 7
 * and 8, code/lb3d_invasion.F90:45-129) and rebuilds the Lees-Edwards halo
 * after streaming.  On the FP32 path, whose advection is deferred into the
 * collision's kernel passes, the inflow boundaries run inside those passes.
 * Periodic halos are an index wrap inside the kernels. */
int lb3dc_bc_apply(lb3dc_handle *h, int stage);
/* code/lb3d_advection.F90:40-151 with half-way bounce-back
 * (code/lb3d_bc_bounce.F90:53-90). */
int lb3dc_advection(lb3dc_handle *h);
/* code/lb3d_collision.F90:41-291: dipole relaxation (ternary), Shan-Chen
 * and body forces, BGK relaxation. */
int lb3dc_collision(lb3dc_handle *h);
/* nsteps full time steps (stages 6..9 each); may fuse stages.  The FP64
 * path pulls the post-stream populations inside its collision kernel where
 * nothing acts on them between advection and collision (no Lees-Edwards
 * planes, no inflow boundaries): the results, rho, psi, the momenta and the
 * dipole flux included, are those of the stage-by-stage calls bit for
 * bit. */
int lb3dc_time_loop(lb3dc_handle *h, int nsteps);
/* Waits for all work of h; reports deferred kernel errors. */
int lb3dc_sync(lb3dc_handle *h);

/* ---- launch shape of the FP32 fused kernel ------------------------------ */
/* Tile of the FP32 kernels: tx x ty sites per CTA, zc planes per work
 * item; supported (tx,ty): (32,8) (32,4) (16,16) (16,8) (64,4).  split
 * selects the strategy: 0 = one fused stream-collide pass per step (the
 * moments of the halo are recomputed on chip), 1 = a moments pass writing a
 * per-site moment field (32 B ternary, 8 B binary) and own-site moments
 * (48 B / 32 B), a dipole pass (ternary) and a collide pass that reads them
 * with their halo, 2 = as 1, but the collide pass stages each site's pulled
 * populations in shared memory with asynchronous copies one plane ahead
 * and sums the own moments itself (no own-moment field), 3 = a moments
 * pass writing halo-padded moment fields, a dipole pass (ternary) and a
 * collide pass that receive those fields as TMA boxes with a one-site halo,
 * the collide pass writing the equilibrium: offered only when every
 * component relaxes fully (tau = 1) on a lattice at least 2 sites across in
 * x and y without inflow boundaries (LB3DC_ENOTSUP otherwise); each of its
 * passes chunks z to fill its own resident grid, so zc is not used.
 * Lees-Edwards lattices (binary) run strategies 2 and 3 only.  All strategies give the same result up to FP32
 * rounding; 0, 1, 2 and 3 agree bit for bit (up to the sign of zero). */
int lb3dc_set_launch_shape(lb3dc_handle *h, int tx, int ty, int zc, int split);
int lb3dc_get_launch_shape(const lb3dc_handle *h, int *tx, int *ty, int *zc, int *split);
/* Times every supported shape and strategy on this lattice (on a saved copy
 * of the state, which is restored afterwards) and keeps the fastest.  ms_out
 * (optional, length >= 64) receives the measured ms per step of each tried
 * candidate in the order tried; returns the number tried in *ntried. */
int lb3dc_autotune(lb3dc_handle *h, double *ms_out, int *ntried);

/* ---- measurement ------------------------------------------------------ */
/* The CUDA stream of h (a cudaStream_t), for callers that record their own
 * events or order work against the handle. */
void *lb3dc_stream(const lb3dc_handle *h);
/* When enabled, every launch of the dominant kernel of a step (the fused
 * stream-collide kernel of the FP32 path, the stream and collide kernels of
 * the FP64 path) is bracketed by CUDA events on the handle's stream; the
 * accumulated device time and launch count are read (synchronising) with
 * lb3dc_kernel_stats and reset by lb3dc_set_profiling. */
int lb3dc_set_profiling(lb3dc_handle *h, int enable);
int lb3dc_kernel_stats(lb3dc_handle *h, double *ms_total, long long *launches,
                       long long *all_launches);

/* ---- Lees-Edwards bookkeeping (FP64 on the host) ---------------------- */
int lb3dc_set_lees_edwards(lb3dc_handle *h, double shear_sum, double shear_u);
int lb3dc_get_lees_edwards(const lb3dc_handle *h, double *shear_sum, double *shear_u);
int lb3dc_get_timestep(const lb3dc_handle *h, int *nt);

/* ---- observability (synchronising) ------------------------------------ */
/* FP64 sums over fluid sites: mass[c] = sum rho_c, mom[k] = sum_c sum
 * n_c g c_k (the conserved quantities of lbe_sanity_check,
 * code/lb3d_sanity.F90:130-234).  Deterministic order. */
int lb3dc_reduce_conservation(lb3dc_handle *h, double mass[3], double mom[3]);
/* Counts non-finite and negative populations (code/lb3d_sanity.F90:79-130). */
int lb3dc_sanity(lb3dc_handle *h, long long *n_nonfinite, long long *n_negative);
/* The velocity statistics of lbe_sanity_check (code/lb3d_sanity.F90:130-371):
 * for each species s and axis k (index 3*s + k), over fluid sites where
 * |rho_s| > 1e-12 with v = (sum_i n_i g_i c_i) amass_s / rho_s: maxvel = the
 * maximum |v_k|, maxpos = its site (1-based x, y, z; ties go to the site the
 * reference's x-outer, z-inner loop visits last; 0,0,0 when no site
 * qualifies), velsum = the sum of v_k (divide by the site count for the
 * reference's average), n_too_fast = sites where some species has
 * |v| > 0.1, n_fluid = fluid sites.  Any output may be NULL. */
int lb3dc_sanity_velocity(lb3dc_handle *h, double maxvel[9], int maxpos[27], double velsum[9],
                          long long *n_fluid, long long *n_too_fast);
/* Science dump fields at the current state (code/lb3d_io_dump_data.F90):
 * "od", "wd", "sur", "vel", "rock" -> [site]; "dir", "arr" -> [site][3];
 * FP64 values, site index x fastest. */
int lb3dc_dump(lb3dc_handle *h, const char *field, double *out);

/* ---- XDR files (big-endian, the reference's formats) ------------------ */
/* Checkpoint file of one rank (code/lb3d_io_checkpoint.F90:790-873,
 * 1084-1106): sites x outermost, z innermost; per site n_r(19), n_b(19),
 * [n_s(19), da(3), db(3)], rock_state as FP64. Arrays as in upload. */
int lb3dc_xdr_read_checkpoint(const char *path, int nx, int ny, int nz, int ncomp, double *n,
                              double *db, double *rock);
int lb3dc_xdr_write_checkpoint(const char *path, int nx, int ny, int nz, int ncomp,
                               const double *n, const double *da, const double *db,
                               const double *rock);
/* checktopo file (code/lb3d_io_checkpoint.F90:741-779): cdims(3),
 * ccoords(3*nprocs) as int32, then shear_sum as FP64. One rank. */
int lb3dc_xdr_read_topo(const char *path, double *shear_sum);
int lb3dc_xdr_write_topo(const char *path, double shear_sum);
/* Obstacle file (code/lb3d_io_xdrf.F90:358-479): FP32 per site, x fastest;
 * value > 0 is rock.  rock: [nz][ny][nx] 0/1. */
int lb3dc_xdr_read_rock(const char *path, int nx, int ny, int nz, double *rock);
int lb3dc_xdr_write_rock(const char *path, int nx, int ny, int nz, const double *rock);
/* Dump files (code/lb3d_io_xdrf.F90:717-754, 872-912): ncomp_per_site
 * values per site, z outermost, x fastest, FP32 (dump_double = 0) or FP64. */
int lb3dc_xdr_write_field(const char *path, const double *v, long long nsites,
                          int values_per_site, int dump_double);

/* ---- files written while the lattice keeps stepping -------------------- */
/* lb3dc_checkpoint_async reads the current state off the device (as
 * lb3dc_download_state, synchronising) into a pinned buffer of the handle
 * and returns; a host thread then writes it as lb3dc_xdr_write_checkpoint
 * does (rock sites with rock_state 1).  lb3dc_dump_async does the same for
 * one lb3dc_dump field written as lb3dc_xdr_write_field.  One write is in
 * flight per handle: a new one waits for the previous one first (and
 * returns its error if it failed); lb3dc_io_wait waits and returns the
 * status of the last write; lb3dc_destroy waits too.  Replaces the
 * download + write of lb3d_io_write_checkpoint / lb3d_io_write_data on
 * dump steps (code/lb3d_time_loop.F90:88-90,
 * code/lb3d_io_checkpoint.F90:790-873, code/lb3d_io_dump_data.F90:241-301). */
int lb3dc_checkpoint_async(lb3dc_handle *h, const char *path);
int lb3dc_dump_async(lb3dc_handle *h, const char *field, const char *path, int dump_double);
int lb3dc_io_wait(lb3dc_handle *h);

/* ---- ensembles: many lattices, one persistent kernel ------------------- */
/*
 * Parameter sweeps (many independent small lattices of uneven size) run as
 * one ensemble: every member occupies a contiguous range of one packed,
 * device-resident site space and all active members advance together in
 * the FP32 deviation path's fused kernel over one tile list, replayed from a
 * CUDA graph while the active set is unchanged.  A member's results are the
 * same alone and in any mix.  No counterpart in the reference (which runs
 * one lattice per MPI job); the per-lattice arithmetic is that of the
 * single-lattice FP32 path.
 */
typedef struct lb3dc_ensemble lb3dc_ensemble;
/* capacity_sites bounds the sum of member sizes (19*capacity < 2^32);
 * device bytes: 2*19*ncomp*4 (+24 ternary) per site of capacity. */
int lb3dc_ensemble_create(int ncomp, long long capacity_sites, int max_lattices,
                          lb3dc_ensemble **out);
int lb3dc_ensemble_destroy(lb3dc_ensemble *e);
int lb3dc_ensemble_last_error(const lb3dc_ensemble *e, char *buf, int len);
int lb3dc_ensemble_set_shape(lb3dc_ensemble *e, int tx, int ty, int zc, int split);
/* Admits one periodic lattice (p->precision is ignored: members are FP32
 * deviation) that will run nsteps steps; n, db as in lb3dc_upload_state.
 * Returns LB3DC_ENOMEM when no slot or no contiguous site range is free:
 * the caller keeps the request queued (admission by HBM footprint). */
int lb3dc_ensemble_admit(lb3dc_ensemble *e, const lb3dc_params *p, const double *n,
                         const double *db, int nsteps, int *slot_out);
/* As lb3dc_ensemble_admit, with the seeded initial state generated on the
 * device: rho_c = rho[c] + U(-amp, amp) per site from the SplitMix64
 * counter generator of lb3d_b200/ic.py, zero velocity, unit dipoles. */
int lb3dc_ensemble_admit_seeded(lb3dc_ensemble *e, const lb3dc_params *p, unsigned long long seed,
                                const double rho[3], double amp, int nsteps, int *slot_out);
/* Advances every active member by up to max_steps steps, stopping early when
 * the first member completes its steps; *steps_done receives the count.
 * Asynchronous. */
int lb3dc_ensemble_step(lb3dc_ensemble *e, int max_steps, int *steps_done);
int lb3dc_ensemble_sync(lb3dc_ensemble *e);
/* Members that completed their steps (still resident until retired). */
int lb3dc_ensemble_finished(lb3dc_ensemble *e, int *slots, int max, int *count);
/* Downloads a member's populations/dipoles (either may be NULL) and frees
 * its slot and site range (synchronising). */
int lb3dc_ensemble_retire(lb3dc_ensemble *e, int slot, double *n, double *db);
/* Asynchronous retire of a finished member: its FP64 populations (and
 * dipoles) are converted and copied to n (db) on a copy stream while the
 * other members keep stepping; n and db should be pinned host memory
 * (lb3dc_host_alloc) for the copies to overlap.  The slot and its site
 * range stay reserved until lb3dc_ensemble_poll reports the copies done. */
int lb3dc_ensemble_retire_async(lb3dc_ensemble *e, int slot, double *n, double *db);
/* *done = 1 (and the slot freed) once the asynchronous retire of slot has
 * landed on the host, else *done = 0. */
int lb3dc_ensemble_poll(lb3dc_ensemble *e, int slot, int *done);
/* Page-locked host memory for asynchronous copies. */
int lb3dc_host_alloc(long long bytes, void **ptr);
int lb3dc_host_free(void *ptr);
int lb3dc_ensemble_stats(const lb3dc_ensemble *e, long long *free_sites, int *active,
                         int *resident, long long *site_updates);
long long lb3dc_ensemble_bytes(const lb3dc_ensemble *e);

/* ---- FP64 step without device allocation ------------------------------ */
/* No counterpart in the reference.  For callers that may not call
 * cudaMalloc -- hosts that own all device memory through their own pool or
 * arrays (for instance a Fortran code keeping its lattice in its own device
 * arrays, or a server that fixes its HBM budget at start-up), or loops that
 * cannot take the synchronisation an allocation can imply.
 * Runs nsteps periodic FP64 steps (the same kernels and results as
 * lb3dc_time_loop with precision LB3DC_FP64) on device buffers the caller
 * owns:
 *   f    : [ncomp][19][nz][ny][nx] populations, in/out (rock sites must hold
 *          zeros, as after lbe_init_rock_colour)
 *   db   : [3][nz][ny][nx] dipoles, in/out (ternary; NULL for binary)
 *   rock : [nz][ny][nx] uint8 rock mask, or NULL for none
 *   stream : a cudaStream_t, or NULL for the default stream.
 * It allocates nothing: the step's intermediate fields live in one
 * file-scope device array of LB3DC_NOALLOC_SCRATCH_BYTES (32 MiB), which
 * every GPU that loads the library holds until the process exits.  That
 * bounds the lattice to 87380 binary or 55923 ternary sites (384 or 600
 * scratch bytes per site; 87152 / 55829 without a caller rock mask); larger
 * lattices are rejected with LB3DC_EINVAL and a message for
 * lb3dc_last_error(NULL, ...).  Lees-Edwards and FP32 are not offered here.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream
 * capture; the address is kept per device and context, and looked up again
 * (outside any capture, too) after a device reset.  All calls share the one array and it keeps the last call's
 * contents: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  Asynchronous on
 * `stream`; returns after enqueueing. */
#define LB3DC_NOALLOC_SCRATCH_BYTES (32ull * 1024ull * 1024ull)
int lb3dc_time_loop_fp64_noalloc(const lb3dc_params *p, double *f, double *db,
                                 const unsigned char *rock, int nsteps, void *stream);

/* ---- self-test helpers ------------------------------------------------- */
/* Evaluates the deterministic FP64 exp (fn 0), expm1 (1) or tanh (2) of
 * the FP64 path on the host (device = 0) or on the current CUDA device
 * (device = 1) for n values; used to prove host/device bit identity. */
int lb3dc_detmath_eval(int fn, int device, const double *x, double *y, long long n);
/* Library build string. */
const char *lb3dc_version(void);

#ifdef __cplusplus
}
#endif
#endif
