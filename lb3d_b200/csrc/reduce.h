// reduce.h -- deterministic FP64 conservation sums and sanity counters.
#ifndef LB3D_REDUCE_H
#define LB3D_REDUCE_H

#include "common.cuh"

namespace lb3d {

constexpr int kReduceBlock = 256;
constexpr int kReduceMaxBlocks = 4 * 148 * 8;  // grid-stride, fixed partition

inline long long reduce_scratch_bytes(long long) { return (long long)kReduceMaxBlocks * 6 * 8 + 64; }

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

// Block-partial layout shared with the FP32 path: partial[b*6 + k],
// k = mass r, b, s, mom x, y, z.
cudaError_t reduce_finish(const double *partials, int nblocks, double mass[3], double mom[3],
                          cudaStream_t st);

}  // namespace lb3d
#endif
