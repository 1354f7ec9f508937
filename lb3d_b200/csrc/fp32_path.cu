// fp32_path.cu -- the FP32 deviation-storage path (LB3DC_FP32_DEV).
#include "fp32_path.h"

namespace lb3d {

long long fp32_footprint(const lb3dc_params &p) {
  const long long N = (long long)p.nx * p.ny * p.nz;
  return 2LL * p.ncomp * 19 * N * 4 + (p.ncomp == 3 ? 6LL * N * 4 : 0);
}
int fp32_alloc(const DevParams &, const lb3dc_params &, Fp32State &, cudaStream_t) {
  return LB3DC_ENOTSUP;
}
void fp32_free(Fp32State &) {}
int fp32_upload(const DevParams &, const lb3dc_params &, Fp32State &, const double *,
                const double *, const uint8_t *, cudaStream_t) {
  return LB3DC_ENOTSUP;
}
int fp32_download(const DevParams &, const lb3dc_params &, Fp32State &, double *, double *,
                  double *, double *, double *, double *, cudaStream_t) {
  return LB3DC_ENOTSUP;
}
int fp32_step(const DevParams &, Fp32State &, const uint8_t *, cudaStream_t) { return LB3DC_ENOTSUP; }
int fp32_run(const DevParams &, Fp32State &, const uint8_t *, int, cudaStream_t) { return LB3DC_ENOTSUP; }
int fp32_dump(const DevParams &, Fp32State &, int, const uint8_t *, double *, cudaStream_t) {
  return LB3DC_ENOTSUP;
}
cudaError_t fp32_reduce_conservation(const DevParams &, Fp32State &, const uint8_t *, double *,
                                     double *, double *, cudaStream_t) {
  return cudaErrorNotSupported;
}
cudaError_t fp32_sanity_counts(const DevParams &, Fp32State &, unsigned long long *,
                               unsigned long long *, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace lb3d
