/*
 * lb3d_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (FP64) of LB3D's per-timestep hot path, used as the
 * checker for the CUDA kernels of lb3d_b200.  Only tests/, the smoke()
 * entry of __graft_entry__.py and bench.py's CPU-baseline leg may load
 * this library; the product never links it.
 *
 * The restatement keeps the reference's data model (an array-of-structs
 * arena with a one-site halo, code/lb3d_lattice.F90:35-83,274-287) and its
 * loop semantics and floating-point operation order, stage by stage, as
 * lb3d_time_loop calls them (code/lb3d_time_loop.F90:58-92).
 *
 * Parity pin: the reference's own golden vectors (test/gyroid,
 * test/bodyForce, test/leesEdwards, test/wettingWall: FP32 XDR dumps at
 * t=10 restored from t=0 checkpoints) are reproduced by this oracle; the
 * tests in tests/test_oracle_golden.py check it to <= 1 FP32 ulp.
 */
#ifndef LB3D_ORACLE_H
#define LB3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors the &lbe_input / &variable_input scalars the hot path reads
 * (code/lb3d_config.F90:44-297).  Component order everywhere: red, blue,
 * surfactant. */
typedef struct lb3do_params {
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
  int bdist;
  int restore; /* 1: state came from a checkpoint (init_cond = 7) */
  int inv_type; /* Zou-He closure (inv_fluid = 12) */
  double pr, pg, pb;
  double fr, fg, fb; /* Zou-He density boundaries (inv_fluid = 11) */
} lb3do_params;

/* Returns NULL on an unsupported parameter combination. */
void *lb3do_create(const lb3do_params *p);
void lb3do_destroy(void *h);
void lb3do_set_threads(int nthreads);
/* 0 (default): glibc exp/tanh; 1: the deterministic exp/tanh the device
 * FP64 path uses (lb3d_b200/csrc/detmath.h). */
void lb3do_set_math(int det);

/* Loads the restored state and runs the initialisation the reference does
 * after a restore: lbe_init_rock_colour (code/lb3d_ic_rock.F90:146-189)
 * and lb3d_bc_init(4) (code/lb3d_bc.F90:48-90).
 * n: [ncomp][19][nz][ny][nx]; db: [3][nz][ny][nx] (ternary, may be NULL);
 * rock: [nz][ny][nx] (0 fluid, nonzero rock; may be NULL).
 * shear_sum: the value read from the checktopo file; nt0: restored step. */
int lb3do_load(void *h, const double *n, const double *db, const double *rock,
               double shear_sum, int nt0);

/* One stage of lb3d_time_loop: 6 = bc_apply(6), 7 = advection,
 * 8 = bc_apply(8), 9 = collision.  lb3do_run does nsteps full steps. */
int lb3do_stage(void *h, int stage);
int lb3do_run(void *h, int nsteps);

/* Interior state; any pointer may be NULL.
 * rho: [ncomp][site]; mom (the reference's u_*, i.e. momentum):
 * [ncomp][3][site]; da, db: [3][site]; site index x fastest. */
int lb3do_get(const void *h, double *n, double *db, double *rho, double *mom, double *da);

/* Science dumps at the current state (code/lb3d_io_dump_data.F90):
 * "od", "wd", "sur", "vel", "rock" -> [site]; "dir", "arr" -> [site][3]. */
int lb3do_dump(void *h, const char *field, double *out);

/* Sum over fluid sites of rho_c and of the momentum sum_c u_c. */
int lb3do_sums(const void *h, double mass[3], double mom[3]);
/* Velocity statistics of lbe_sanity_check (code/lb3d_sanity.F90:130-229),
 * index 3*species + axis; positions 1-based x, y, z. */
int lb3do_sanity_velocity(const void *h, double maxvel[9], int maxpos[27], double velsum[9],
                          long long *n_fluid, long long *n_too_fast);

/* y-slab decomposition (code/lb3d_mpi.F90:492-596 splits the lattice over
 * ranks; here along y only).  A slab oracle is created with ny = its own
 * planes and global-coordinate parameters; lb3do_set_slab, called before
 * lb3do_load, gives its first plane's global y offset and the function that
 * fills the y-halo planes y = 0 and y = ny + 1 from the neighbouring slabs
 * at every halo exchange (with lb3do_yplane), after the x faces and before
 * the z faces.  Not for Lees-Edwards lattices. */
typedef void (*lb3do_halo_fn)(void *ctx, void *h);
int lb3do_set_slab(void *h, int y_off, lb3do_halo_fn fn, void *ctx);
/* Doubles in one y plane of whole sites, x = 0..nx+1, z = 1..nz. */
long long lb3do_yplane_doubles(const void *h);
/* Copies plane y (0..ny+1) out of (put = 0) or into (put = 1) buf. */
int lb3do_yplane(void *h, int y, double *buf, int put);

double lb3do_shear_sum(const void *h);
int lb3do_nt(const void *h);

#ifdef __cplusplus
}
#endif
#endif
