// reduce.h -- deterministic FP64 conservation sums and sanity counters.
#ifndef LB3D_REDUCE_H
#define LB3D_REDUCE_H

#include "common.cuh"

namespace lb3d {

constexpr int kReduceBlock = 256;
constexpr int kReduceMaxBlocks = 4 * 148 * 8;  // grid-stride, fixed partition

// room for the largest per-block partials (the velocity statistics: 29 words)
inline long long reduce_scratch_bytes(long long) { return (long long)kReduceMaxBlocks * 29 * 8 + 64; }

// Velocity statistics of lbe_sanity_check; index 3*species + axis.
struct SanityVelocity {
  double vmax[9];     // max |v_k| over fluid sites with |rho| > 1e-12
  int pos[9][3];      // its site (1-based x, y, z; 0,0,0 when none qualifies)
  double vsum[9];     // sum of v_k over those sites
  long long n_fluid;  // fluid sites
  long long n_too_fast;  // sites where some species has |v| > 0.1
};

// Sums over fluid sites of rho_c and of the total momentum, from FP64
// populations f [nc][19][nsites].  Each block reduces a fixed set of sites
// in a fixed tree order and the host adds the block partials in order, so
// the result does not depend on scheduling.
cudaError_t reduce_conservation_fp64(const DevParams &P, const double *f, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st);
// cnt[0] = non-finite populations, cnt[1] = negative populations.
cudaError_t sanity_counts_fp64(const DevParams &P, const double *f, unsigned long long *scratch,
                               unsigned long long cnt[2], cudaStream_t st);

// The same on the FP32 path's deviations (stride S, lattice at base).
cudaError_t reduce_conservation_fp32(const DevParams &P, const float *f, long long S,
                                     long long base, double rho0, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st);
cudaError_t sanity_counts_fp32(const DevParams &P, const float *f, long long S, long long base,
                               double rho0, unsigned long long *scratch, unsigned long long cnt[2],
                               cudaStream_t st);
cudaError_t sanity_velocity_fp64(const DevParams &P, const double *f, const uint8_t *rock,
                                 void *scratch, SanityVelocity &out, cudaStream_t st);
cudaError_t sanity_velocity_fp32(const DevParams &P, const float *f, long long S, long long base,
                                 double rho0, const uint8_t *rock, void *scratch,
                                 SanityVelocity &out, cudaStream_t st);

// Block-partial layout shared with the FP32 path: partial[b*6 + k],
// k = mass r, b, s, mom x, y, z.
cudaError_t reduce_finish(const double *partials, int nblocks, double mass[3], double mom[3],
                          cudaStream_t st);

}  // namespace lb3d
#endif
