// fp32_path.h -- the FP32 deviation-storage path (LB3DC_FP32_DEV) and the
// packed multi-lattice layout it shares with the ensemble runtime.
#ifndef LB3D_FP32_PATH_H
#define LB3D_FP32_PATH_H

#include <vector>

#include <cuda.h>

#include "common.cuh"
#include "reduce.h"

namespace lb3d {

// One lattice inside the packed arrays.  Populations are stored as FP32
// deviations delta = n - w_i rho0 in f[c][q][S] with a global stride S
// (the capacity in sites); lattice sites start at `base`.
struct LatDesc {
  int nx, ny, nz, nc;
  long long base;
  int parity;     // buffer holding the current state (0/1)
  int flags;      // LAT_ROCK | LAT_BODY | LAT_ACTIVE
  float omega[3], tau[3], amass[3];
  float g_br, g_bs, g_ss;
  float wall_r, wall_b;  // -g_wr tau_wr / tau_r and -g_wb tau_wb / tau_b
  float psiw_r, psiw_b;  // psi(rock colour) seen from a fluid site
  float beta, d0, omega_d;
  float g_accn, g_accn_x, g_accn_y;
  int amin_x, amax_x, amin_y, amax_y, amin_z, amax_z, inv_fluid;
  float rho0, psi0, em0;  // psi(rho0) = 1 - exp(-rho0), em0 = exp(-rho0)
  // Lees-Edwards x-halo planes (binary single lattices; null otherwise):
  // le_h[0/1] the sheared pre-stream populations below x = 0 / above
  // x = nx - 1, [nc][19][nz][ny] deviations; le_p[0/1] the psi deviations of
  // the post-stream halo sites, [nz][ny] float2 {dpsi_r, dpsi_b}.
  // stage-8 inflow boundaries on the z planes (single lattices): kind as
  // DevParams::invk, the Zou-He closure type and the imposed values
  int invk, inv_type;
  float zh_in[2], zh_uz[3];
  float *le_h[2];
  float2 *le_p[2];
  // Lees-Edwards boundary planes, [nc][19][nz][ny] deviations: le_b[0/1] the
  // pre-stream populations at x = nx - 1 / x = 0 (written by the collide
  // pass of the previous step), le_b[2/3] the post-stream populations there
  // (written by the moments pass); the halo kernels read them coalesced
  float *le_b[4];
};
constexpr int LAT_ROCK = 1, LAT_BODY = 2, LAT_ACTIVE = 4;

// Tile: lattice id, xy origin and z range of one CTA work item.
struct Tile {
  int lat;
  short x0, y0;
  short z0, zc;
};

struct Fp32State {
  float *f[2] = {nullptr, nullptr};   // [nc][19][S]
  float *db[2] = {nullptr, nullptr};  // [3][S] (ternary)
  LatDesc *d_lat = nullptr;
  Tile *d_tiles = nullptr;
  int ntiles = 0;
  LatDesc lat{};        // host copy (single-lattice handle)
  long long S = 0;      // stride (sites)
  int tx = 32, ty = 8, zc = 16;  // launch shape (autotuned)
  int split = 0;                 // kernel strategy (autotuned)
  float4 *M = nullptr;           // stencil moment field of the split strategy
  float4 *J = nullptr;           // own-site densities and momenta (split)
  int grid = 0;
  long long bytes = 0;
  KernelTimer *timer = nullptr;  // optional, owned by the handle
  // two FP64 population planes (N sites each) for uploads and downloads: the
  // copy of one plane on the copy stream overlaps the conversion of the other
  double *stage = nullptr;
  cudaStream_t xs = nullptr;                         // copy stream
  cudaEvent_t xev[4] = {nullptr, nullptr, nullptr, nullptr};  // per plane: filled, drained
  float *le_h[2] = {nullptr, nullptr};  // Lees-Edwards halo planes (see LatDesc)
  float2 *le_p[2] = {nullptr, nullptr};
  float *le_b[4] = {nullptr, nullptr, nullptr, nullptr};
  // moment-field strategy (split 3): the halo-padded moment fields (and
  // dipole field, ternary), the plain momentum plane, the tensor maps of their
  // TMA boxes (encoded for the tile shape mf_tx x mf_ty) and the device flag
  // of a wait that gave up
  float4 *MF1 = nullptr, *MF2 = nullptr, *DD = nullptr;
  float2 *MFp = nullptr;
  float *DS = nullptr;
  int *err = nullptr;
  CUtensorMap tm1{}, tm2{}, tmd{};
  int mf_tx = 0, mf_ty = 0;
  // its tile lists, one per pass (moments, dipole, collide), each chunking z
  // so that the tiles fill the pass's resident grid: mf_ntiles[p] tiles at
  // mf_tiles + mf_off[p], launched on mf_grid[p] CTAs
  Tile *mf_tiles = nullptr;
  int mf_ntiles[3] = {0, 0, 0}, mf_off[3] = {0, 0, 0}, mf_grid[3] = {0, 0, 0};
};

// Launch configuration of the fused kernel.
struct FusedShape {
  int tx, ty, zc;
  int split = 0;  // 0: one fused pass per step; 1: moments (+ dipole) + collide passes;
                  // 2: as 1 with the asynchronously staged collide pass (no J field);
                  // 3: moment field + TMA-fed dipole/force/equilibrium pass (full
                  //    relaxation only, single lattices)
};

long long fp32_footprint(const lb3dc_params &p);
LatDesc fp32_make_desc(const DevParams &P, double rho0, long long base, bool rock);
int fp32_alloc(const DevParams &P, const lb3dc_params &p, Fp32State &s, cudaStream_t st);
void fp32_free(Fp32State &s);
int fp32_upload(const DevParams &P, const lb3dc_params &p, Fp32State &s, const double *n,
                const double *db, const uint8_t *rock, cudaStream_t st);
int fp32_download(const DevParams &P, const lb3dc_params &p, Fp32State &s, double *n,
                  double *db, double *rho, double *mom, double *da, const uint8_t *rock,
                  cudaStream_t st);
// One step; le gives this step's Lees-Edwards offset (null: periodic).
int fp32_step(const DevParams &P, Fp32State &s, const uint8_t *rock, cudaStream_t st,
              const LEStep *le = nullptr);
// nsteps steps; le (null: periodic) is applied unchanged to every step, as the
// autotuner wants; a Lees-Edwards time loop advances one step at a time.
int fp32_run(const DevParams &P, Fp32State &s, const uint8_t *rock, int nsteps, cudaStream_t st,
             const LEStep *le = nullptr);
int fp32_dump(const DevParams &P, Fp32State &s, int field, const uint8_t *rock, double *out,
              cudaStream_t st);
cudaError_t fp32_reduce_conservation(const DevParams &P, Fp32State &s, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st);
cudaError_t fp32_sanity_counts(const DevParams &P, Fp32State &s, unsigned long long *scratch,
                               unsigned long long cnt[2], cudaStream_t st);
cudaError_t fp32_sanity_velocity(const DevParams &P, Fp32State &s, const uint8_t *rock,
                                 void *scratch, SanityVelocity &out, cudaStream_t st);

// Shared with the ensemble runtime: tile list for a lattice, fused launch.
void fp32_tiles_for(const LatDesc &L, int lat_id, const FusedShape &sh, std::vector<Tile> &out);
// fin/fout select by parity inside the kernel; `flip` is applied by caller.
// Each pass runs as many CTAs as are resident at once for that kernel (at
// most ntiles); max_grid > 0 caps that number.
// With le (a binary single lattice whose LatDesc carries the halo planes,
// strategy 2 only) the step also builds the sheared x-halos: the stage-6
// populations before the moments pass and the stage-8 psi planes before the
// collide pass.
cudaError_t fp32_launch_fused(int nc, bool rock, bool body, const FusedShape &sh,
                              const LatDesc *d_lat, const Tile *d_tiles, int ntiles, int max_grid,
                              float *f0, float *f1, float *db0, float *db1, const uint8_t *rockp,
                              long long S, cudaStream_t st, float4 *M = nullptr,
                              float4 *J = nullptr, const LEStep *le = nullptr,
                              const DevParams *P = nullptr);
// FP32 deviations <-> FP64 populations of one lattice (N sites at `base`
// in arrays of stride S), on the device; rock (optional, device, N bytes)
// marks sites whose populations are zero.
cudaError_t fp32_to_fp64(const float *f, double *out, long long S, long long base, long long N,
                         int nc, double rho0, cudaStream_t st);
cudaError_t fp32_from_fp64(const double *n, float *f, long long S, long long base, long long N,
                           int nc, double rho0, const uint8_t *rock, cudaStream_t st);
// `planes` FP32 planes of stride S (lattice at base) widened to FP64 [planes][N].
cudaError_t fp32_planes_to_fp64(const float *src, double *dst, long long S, long long base,
                                long long N, int planes, cudaStream_t st);
// Bytes per site of the split strategy's moment fields.
inline long long fp32_moment_bytes(int nc) { return nc == 3 ? 32 : 8; }
inline long long fp32_own_bytes(int nc) { return nc == 3 ? 48 : 32; }
// Flips the parity of every active lattice (one tiny kernel).
cudaError_t fp32_flip_parity(LatDesc *d_lat, int nlat, cudaStream_t st);
size_t fp32_fused_smem(int nc, const FusedShape &sh);
int fp32_set_shape(const DevParams &P, Fp32State &s, const FusedShape &sh, cudaStream_t st);
// Candidate shapes of the autotuner.
std::vector<FusedShape> fp32_candidate_shapes(const DevParams &P);
int fp32_autotune(const DevParams &P, Fp32State &s, const uint8_t *rock, double *ms_out,
                  int *ntried, cudaStream_t st, const LEStep *le = nullptr);
int fp32_fused_ctas_per_sm(int nc, bool rock, bool body, const FusedShape &sh);
// The moment-field strategy applies: every component relaxes fully
// (omega = 1), periodic or walled lattice without Lees-Edwards planes or
// inflow boundaries, at least 2 sites across in x and y.
bool fp32_mf_eligible(const DevParams &P);
// Bytes of the moment and dipole fields of strategy 3.
long long fp32_mf_bytes(const DevParams &P);
// The device error flag of the handle's kernels (0, or LB3DC_ETIMEOUT when a
// bounded wait gave up), read and cleared; LB3DC_OK when no flag exists.
int fp32_take_error(Fp32State &s, cudaStream_t st);

}  // namespace lb3d
#endif
