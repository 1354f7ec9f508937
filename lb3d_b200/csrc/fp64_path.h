// fp64_path.h -- host launchers of the FP64 drop-in kernels (fp64_path.cu).
#ifndef LB3D_FP64_PATH_H
#define LB3D_FP64_PATH_H

#include "common.cuh"

namespace lb3d {

cudaError_t fp64_le_halo(const DevParams &P, const LEStep &S, const double *src, double *hlo,
                         double *hhi, double *rlo, double *rhi, double *plo, double *phi,
                         cudaStream_t st);
// Zou-He flux boundaries on the z = 1 and z = nz planes (inv_fluid 12),
// applied to the post-stream populations g and the advected dipole flux da.
cudaError_t fp64_zouhe_density(const DevParams &P, double *g, const uint8_t *rock, double fr,
                               double fb, double pr, double pb, cudaStream_t st);
cudaError_t fp64_recolour(const DevParams &P, double *g, const uint8_t *rock, double mr, double mb,
                          cudaStream_t st);
cudaError_t fp64_zouhe_flux(const DevParams &P, double *g, double *da, const double *db,
                            const uint8_t *rock, cudaStream_t st);
cudaError_t fp64_stream(const DevParams &P, const double *fin, double *fout, double *rho,
                        double *psi, double *mom, double *da, const double *db,
                        const uint8_t *rock, const double *hlo, const double *hhi,
                        cudaStream_t st);
// One time step with streaming fused into the collision (periodic lattices,
// no Lees-Edwards planes, no stage-8 boundaries): moments pass (rho, psi,
// momenta, dipole flux), dipole relaxation (ternary), pull + forces + BGK
// from fin into fout.  Every buffer ends up as after fp64_stream +
// fp64_dipole + fp64_collide, bit for bit, except that the post-stream
// populations are never stored.
cudaError_t fp64_step_pull(const DevParams &P, const double *fin, double *fout, double *rho,
                           double *psi, double *mom, double *da, double *db, const uint8_t *rock,
                           cudaStream_t st);
cudaError_t fp64_dipole(const DevParams &P, const double *rho, const double *da, double *db,
                        cudaStream_t st);
cudaError_t fp64_collide(const DevParams &P, const double *g, double *f, const double *rho,
                         const double *psi, const double *mom, const double *db,
                         const uint8_t *rock, const double *plo, const double *phi,
                         cudaStream_t st);
// field: 0 od, 1 wd, 2 sur, 3 dir, 4 vel, 5 arr, 6 rock
cudaError_t fp64_dump(const DevParams &P, int field, const double *f, const double *rho,
                      const double *psi, const double *db, const uint8_t *rock, double *out,
                      cudaStream_t st);
cudaError_t fp64_moments(const DevParams &P, const double *f, double *rho, double *psi,
                         double *mom, cudaStream_t st);
cudaError_t fp64_detmath(int fn, const double *x, double *y, long long n, cudaStream_t st);

}  // namespace lb3d

#endif
