// reduce.cu -- FP64 conservation sums (warp shuffles + a fixed block tree)
// and sanity counters for the FP64 path.
#include <vector>

#include "reduce.h"

namespace lb3d {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NC>
__global__ void __launch_bounds__(kReduceBlock) k_conserve(DevParams P, const double *__restrict__ f,
                                                           const uint8_t *__restrict__ rock,
                                                           double *__restrict__ partial) {
  const long long N = P.nsites;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (rock[i] != 0) continue;
    for (int c = 0; c < NC; ++c) {
      double r = 0.0, m0 = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        double ng = f[(c * 19 + q) * N + i] * (double)gw(q);
        r += ng;
        m0 += ng * (double)cx(q);
        m1 += ng * (double)cy(q);
        m2 += ng * (double)cz(q);
      }
      acc[c] += r;
      acc[3] += m0;
      acc[4] += m1;
      acc[5] += m2;
    }
  }
  __shared__ double sh[6][kReduceBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < 6; ++k) {
    double v = warp_sum(acc[k]);
    if (lane == 0) sh[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0.0;
    for (int w = 0; w < kReduceBlock / 32; ++w) v += sh[threadIdx.x][w];
    partial[blockIdx.x * 6 + threadIdx.x] = v;
  }
}

template <int NC>
__global__ void k_sanity(DevParams P, const double *__restrict__ f, unsigned long long *cnt) {
  const long long M = (long long)NC * 19 * P.nsites;
  unsigned long long bad = 0, neg = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (long long)gridDim.x * blockDim.x) {
    double v = f[i];
    if (!isfinite(v)) ++bad;
    else if (v < 0.0) ++neg;
  }
  for (int o = 16; o > 0; o >>= 1) {
    bad += __shfl_down_sync(0xffffffffu, bad, o);
    neg += __shfl_down_sync(0xffffffffu, neg, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicAdd(&cnt[0], bad);
    if (neg) atomicAdd(&cnt[1], neg);
  }
}

int nblocks_for(long long n) {
  long long b = (n + kReduceBlock - 1) / kReduceBlock;
  if (b > kReduceMaxBlocks) b = kReduceMaxBlocks;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t reduce_finish(const double *partials, int nb, double mass[3], double mom[3],
                          cudaStream_t st) {
  std::vector<double> h((size_t)nb * 6);
  cudaError_t e = cudaMemcpyAsync(h.data(), partials, h.size() * 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  for (int k = 0; k < 3; ++k) mass[k] = mom[k] = 0.0;
  for (int b = 0; b < nb; ++b) {
    for (int k = 0; k < 3; ++k) mass[k] += h[(size_t)b * 6 + k];
    for (int k = 0; k < 3; ++k) mom[k] += h[(size_t)b * 6 + 3 + k];
  }
  return cudaSuccess;
}

cudaError_t reduce_conservation_fp64(const DevParams &P, const double *f, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st) {
  int nb = nblocks_for(P.nsites);
  if (P.nc == 2)
    k_conserve<2><<<nb, kReduceBlock, 0, st>>>(P, f, rock, scratch);
  else
    k_conserve<3><<<nb, kReduceBlock, 0, st>>>(P, f, rock, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return reduce_finish(scratch, nb, mass, mom, st);
}

cudaError_t sanity_counts_fp64(const DevParams &P, const double *f, unsigned long long *scratch,
                               unsigned long long cnt[2], cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(scratch, 0, 16, st);
  if (e != cudaSuccess) return e;
  long long M = (long long)P.nc * 19 * P.nsites;
  int nb = nblocks_for(M);
  if (P.nc == 2)
    k_sanity<2><<<nb, kReduceBlock, 0, st>>>(P, f, scratch);
  else
    k_sanity<3><<<nb, kReduceBlock, 0, st>>>(P, f, scratch);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, scratch, 16, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

}  // namespace lb3d
