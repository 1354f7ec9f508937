// reduce.cu -- FP64 conservation sums (warp shuffles + a fixed block tree),
// sanity counters and the velocity statistics of lbe_sanity_check, for the
// FP64 arrays and for the FP32 path's deviations (read as FP64 populations,
// rounded as its download rounds).
#include <type_traits>
#include <vector>

#include "reduce.h"

namespace lb3d {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// FP64 view of a lattice's populations [nc][19] x stride S from `base`:
// the FP64 arrays themselves, or FP32 deviations + w_q rho0.
template <typename T>
struct Pops {
  const T *f;
  long long S, base;
  double rho0;
  __device__ __forceinline__ double operator()(int c, int q, long long i) const {
    const T v = f[((long long)c * 19 + q) * S + base + i];
    if constexpr (std::is_same<T, float>::value)
      return __dadd_rn((double)v, __dmul_rn(q == 18 ? 1.0 / 3.0 : 1.0 / 36.0, rho0));
    else
      return v;
  }
};

template <int NC, typename T>
__global__ void __launch_bounds__(kReduceBlock) k_conserve(DevParams P, Pops<T> pop,
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
        double ng = pop(c, q, i) * (double)gw(q);
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

template <int NC, typename T>
__global__ void k_sanity(DevParams P, Pops<T> pop, unsigned long long *cnt) {
  const long long N = P.nsites;
  unsigned long long bad = 0, neg = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q) {
        const double v = pop(c, q, i);
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

// lbe_sanity_check's velocity statistics (code/lb3d_sanity.F90:130-229):
// over fluid sites, for each species with |rho| > 1e-12, the velocity
// v = (sum_q n_q g_q c_q) amass / rho; per species and axis the maximum
// |v_k| and the site holding it (ties go to the later site of the
// reference's x-outer, z-inner loop, as its `>=` does), the sum of v, and
// the count of sites where some species has |v| > 0.1.  Per block: the
// (|v|, loop index) maxima, the sums in a fixed tree order and the counts;
// the host combines the blocks in order.
constexpr int kVelSlots = 9;
struct VelPartial {
  double vmax[kVelSlots];
  long long loc[kVelSlots];
  double vsum[kVelSlots];
  unsigned long long n_fluid, n_fast;
};

__device__ __forceinline__ void keep_max(double &v, long long &l, double v2, long long l2) {
  if (v2 > v || (v2 == v && l2 > l)) v = v2, l = l2;
}

template <int NC, typename T>
__global__ void __launch_bounds__(kReduceBlock) k_sanity_vel(DevParams P, Pops<T> pop,
                                                             const uint8_t *__restrict__ rock,
                                                             VelPartial *__restrict__ out) {
  const long long N = P.nsites;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  double vmax[kVelSlots], vsum[kVelSlots];
  long long loc[kVelSlots];
  for (int k = 0; k < kVelSlots; ++k) vmax[k] = -1.0, loc[k] = -1, vsum[k] = 0.0;
  unsigned long long n_fluid = 0, n_fast = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if (rock[i] != 0) continue;
    ++n_fluid;
    const long long t = i / nx;
    const int x = (int)(i - t * nx), z = (int)(t / ny), y = (int)(t - (long long)z * ny);
    const long long L = ((long long)x * ny + y) * nz + z;  // reference loop order
    bool fast = false;
    for (int c = 0; c < NC; ++c) {
      double r = 0.0, m0 = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        const double ng = pop(c, q, i) * (double)gw(q);
        r = r + ng;
        m0 = m0 + ng * (double)cx(q);
        m1 = m1 + ng * (double)cy(q);
        m2 = m2 + ng * (double)cz(q);
      }
      if (fabs(r) > 1.0e-12) {
        const double v[3] = {m0 * P.amass[c] / r, m1 * P.amass[c] / r, m2 * P.amass[c] / r};
        for (int k = 0; k < 3; ++k) {
          vsum[3 * c + k] = vsum[3 * c + k] + v[k];
          keep_max(vmax[3 * c + k], loc[3 * c + k], fabs(v[k]), L);
        }
        if (sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) > 0.1) fast = true;
      }
    }
    if (fast) ++n_fast;
  }
  __shared__ double shv[kReduceBlock / 32];
  __shared__ long long shl[kReduceBlock / 32];
  __shared__ unsigned long long shc[2][kReduceBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < kVelSlots; ++k) {
    double v = vmax[k];
    long long l = loc[k];
    for (int o = 16; o > 0; o >>= 1)
      keep_max(v, l, __shfl_down_sync(0xffffffffu, v, o), __shfl_down_sync(0xffffffffu, l, o));
    double sm = warp_sum(vsum[k]);
    __syncthreads();
    if (lane == 0) shv[wid] = v, shl[wid] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
      double bv = -1.0;
      long long bl = -1;
      for (int w = 0; w < kReduceBlock / 32; ++w) keep_max(bv, bl, shv[w], shl[w]);
      out[blockIdx.x].vmax[k] = bv;
      out[blockIdx.x].loc[k] = bl;
    }
    __syncthreads();
    if (lane == 0) shv[wid] = sm;
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0;
      for (int w = 0; w < kReduceBlock / 32; ++w) a += shv[w];
      out[blockIdx.x].vsum[k] = a;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    n_fluid += __shfl_down_sync(0xffffffffu, n_fluid, o);
    n_fast += __shfl_down_sync(0xffffffffu, n_fast, o);
  }
  if (lane == 0) shc[0][wid] = n_fluid, shc[1][wid] = n_fast;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long a = 0, b = 0;
    for (int w = 0; w < kReduceBlock / 32; ++w) a += shc[0][w], b += shc[1][w];
    out[blockIdx.x].n_fluid = a;
    out[blockIdx.x].n_fast = b;
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

template <typename T>
static cudaError_t conservation(const DevParams &P, Pops<T> pop, const uint8_t *rock,
                                double *scratch, double mass[3], double mom[3], cudaStream_t st) {
  int nb = nblocks_for(P.nsites);
  if (P.nc == 2)
    k_conserve<2, T><<<nb, kReduceBlock, 0, st>>>(P, pop, rock, scratch);
  else
    k_conserve<3, T><<<nb, kReduceBlock, 0, st>>>(P, pop, rock, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return reduce_finish(scratch, nb, mass, mom, st);
}

template <typename T>
static cudaError_t counts(const DevParams &P, Pops<T> pop, unsigned long long *scratch,
                          unsigned long long cnt[2], cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(scratch, 0, 16, st);
  if (e != cudaSuccess) return e;
  int nb = nblocks_for(P.nsites);
  if (P.nc == 2)
    k_sanity<2, T><<<nb, kReduceBlock, 0, st>>>(P, pop, scratch);
  else
    k_sanity<3, T><<<nb, kReduceBlock, 0, st>>>(P, pop, scratch);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, scratch, 16, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

template <typename T>
static cudaError_t velocity(const DevParams &P, Pops<T> pop, const uint8_t *rock, void *scratch,
                            SanityVelocity &out, cudaStream_t st) {
  int nb = nblocks_for(P.nsites);
  VelPartial *part = (VelPartial *)scratch;
  if (P.nc == 2)
    k_sanity_vel<2, T><<<nb, kReduceBlock, 0, st>>>(P, pop, rock, part);
  else
    k_sanity_vel<3, T><<<nb, kReduceBlock, 0, st>>>(P, pop, rock, part);
  cudaError_t e = cudaGetLastError();
  std::vector<VelPartial> h(nb);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, nb * sizeof(VelPartial), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  double vmax[kVelSlots];
  long long loc[kVelSlots];
  for (int k = 0; k < kVelSlots; ++k) vmax[k] = -1.0, loc[k] = -1, out.vsum[k] = 0.0;
  out.n_fluid = out.n_too_fast = 0;
  for (int b = 0; b < nb; ++b) {
    for (int k = 0; k < kVelSlots; ++k) {
      if (h[b].vmax[k] > vmax[k] || (h[b].vmax[k] == vmax[k] && h[b].loc[k] > loc[k]))
        vmax[k] = h[b].vmax[k], loc[k] = h[b].loc[k];
      out.vsum[k] += h[b].vsum[k];
    }
    out.n_fluid += (long long)h[b].n_fluid;
    out.n_too_fast += (long long)h[b].n_fast;
  }
  for (int k = 0; k < kVelSlots; ++k) {
    // no qualifying site: maximum 0 at position (0, 0, 0), the reference's initial values
    out.vmax[k] = loc[k] < 0 ? 0.0 : vmax[k];
    int x = 0, y = 0, z = 0;
    if (loc[k] >= 0) {
      z = (int)(loc[k] % P.nz);
      const long long t = loc[k] / P.nz;
      y = (int)(t % P.ny);
      x = (int)(t / P.ny);
      ++x, ++y, ++z;  // 1-based, as the reference reports them
    }
    out.pos[k][0] = x, out.pos[k][1] = y, out.pos[k][2] = z;
  }
  return cudaSuccess;
}

cudaError_t reduce_conservation_fp64(const DevParams &P, const double *f, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st) {
  return conservation(P, Pops<double>{f, P.nsites, 0, 0.0}, rock, scratch, mass, mom, st);
}
cudaError_t reduce_conservation_fp32(const DevParams &P, const float *f, long long S,
                                     long long base, double rho0, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st) {
  return conservation(P, Pops<float>{f, S, base, rho0}, rock, scratch, mass, mom, st);
}
cudaError_t sanity_counts_fp64(const DevParams &P, const double *f, unsigned long long *scratch,
                               unsigned long long cnt[2], cudaStream_t st) {
  return counts(P, Pops<double>{f, P.nsites, 0, 0.0}, scratch, cnt, st);
}
cudaError_t sanity_counts_fp32(const DevParams &P, const float *f, long long S, long long base,
                               double rho0, unsigned long long *scratch, unsigned long long cnt[2],
                               cudaStream_t st) {
  return counts(P, Pops<float>{f, S, base, rho0}, scratch, cnt, st);
}
cudaError_t sanity_velocity_fp64(const DevParams &P, const double *f, const uint8_t *rock,
                                 void *scratch, SanityVelocity &out, cudaStream_t st) {
  return velocity(P, Pops<double>{f, P.nsites, 0, 0.0}, rock, scratch, out, st);
}
cudaError_t sanity_velocity_fp32(const DevParams &P, const float *f, long long S, long long base,
                                 double rho0, const uint8_t *rock, void *scratch,
                                 SanityVelocity &out, cudaStream_t st) {
  return velocity(P, Pops<float>{f, S, base, rho0}, rock, scratch, out, st);
}

}  // namespace lb3d
