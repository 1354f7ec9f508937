// fp32_path.h -- the FP32 deviation-storage path (LB3DC_FP32_DEV).
#ifndef LB3D_FP32_PATH_H
#define LB3D_FP32_PATH_H

#include "common.cuh"

namespace lb3d {

struct Fp32State {
  float *fa = nullptr, *fb = nullptr;  // deviation populations, ping-pong [nc][19][N]
  float *da_ = nullptr, *db_a = nullptr, *db_b = nullptr;
  double rho0 = 0.7;
  int cur = 0;
  long long bytes = 0;
  void *aux = nullptr;
};

long long fp32_footprint(const lb3dc_params &p);
int fp32_alloc(const DevParams &P, const lb3dc_params &p, Fp32State &s, cudaStream_t st);
void fp32_free(Fp32State &s);
int fp32_upload(const DevParams &P, const lb3dc_params &p, Fp32State &s, const double *n,
                const double *db, const uint8_t *rock, cudaStream_t st);
int fp32_download(const DevParams &P, const lb3dc_params &p, Fp32State &s, double *n,
                  double *db, double *rho, double *mom, double *da, double *scratch,
                  cudaStream_t st);
int fp32_step(const DevParams &P, Fp32State &s, const uint8_t *rock, cudaStream_t st);
int fp32_run(const DevParams &P, Fp32State &s, const uint8_t *rock, int nsteps, cudaStream_t st);
int fp32_dump(const DevParams &P, Fp32State &s, int field, const uint8_t *rock, double *out,
              cudaStream_t st);
cudaError_t fp32_reduce_conservation(const DevParams &P, Fp32State &s, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st);
cudaError_t fp32_sanity_counts(const DevParams &P, Fp32State &s, unsigned long long *scratch,
                               unsigned long long cnt[2], cudaStream_t st);

}  // namespace lb3d
#endif
