// noalloc.cu -- the FP64 time step for callers that cannot allocate device
// memory.
//
// Some callers may not call cudaMalloc: hosts that own every device byte
// through their own pool or allocator (a Fortran code holding its lattice in
// its own device arrays, a server that fixes its HBM budget at start-up) and
// loops that cannot afford the device-wide synchronisation an allocation can
// imply.  For them,
// lb3dc_time_loop_fp64_noalloc runs the FP64 drop-in step on buffers the
// caller owns and keeps its intermediate fields (the post-stream populations
// and moments) in a file-scope device array of fixed size instead of
// allocating them.
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda.h>

#include "../../include/lb3dc.h"
#include "common.cuh"
#include "fp64_path.h"
#include "params.h"

namespace {

// The scratch array.  Every GPU that loads the library holds these bytes
// until the process exits.  Its name is only a host-side stand-in in host
// code: host code must use the device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LB3DC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 256;
std::mutex g_mu;
unsigned char *g_addr[kMaxDevices] = {nullptr};
// The context each cached address belongs to: a device reset (or any
// teardown of the primary context) reloads the module in a new context
// with a new unique id, and the address is looked up again.
unsigned long long g_ctx_id[kMaxDevices] = {0};

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context (0 if none or if the
// driver offers no id), through the runtime's driver entry points.
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<CtxGetCurrentFn>(a);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(b);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

inline size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// Scratch bytes of one step for n sites: post-stream populations g
// [nc][19][n], rho and psi [nc][n], mom [nc][3][n], da [3][n] (ternary),
// plus a zero rock mask [n] when the caller passes none.
size_t scratch_need(int nc, long long n, bool own_rock) {
  size_t b = up256((size_t)nc * 19 * n * 8);
  b += 2 * up256((size_t)nc * n * 8);
  b += up256((size_t)nc * 3 * n * 8);
  if (nc == 3) b += up256((size_t)3 * n * 8);
  if (own_rock) b += up256((size_t)n);
  return b;
}

int err(int code, const std::string &m) { return lb3d::set_global_error(code, m.c_str()); }

}  // namespace

extern "C" int lb3dc_time_loop_fp64_noalloc(const lb3dc_params *p, double *f, double *db,
                                            const unsigned char *rock, int nsteps, void *stream) {
  std::string why;
  int rc = lb3d::validate_params(p, why);
  if (rc != LB3DC_OK) return err(rc, why);
  if (p->precision != LB3DC_FP64) return err(LB3DC_ENOTSUP, "the no-alloc step is the FP64 path only");
  if (p->boundary_cond != 0) return err(LB3DC_ENOTSUP, "the no-alloc step is periodic (boundary_cond = 0) only");
  if (!f || (p->ncomp == 3 && !db) || nsteps < 0) return err(LB3DC_EINVAL, "NULL populations/dipoles or nsteps < 0");
  const long long n = (long long)p->nx * p->ny * p->nz;
  const size_t need = scratch_need(p->ncomp, n, rock == nullptr);
  if (need > (size_t)LB3DC_NOALLOC_SCRATCH_BYTES) {
    char m[256];
    std::snprintf(m, sizeof(m),
                  "lattice of %lld sites needs %zu scratch bytes; the no-alloc step holds %llu "
                  "(at most 87380 binary or 55923 ternary sites with a rock mask)",
                  n, need, (unsigned long long)LB3DC_NOALLOC_SCRATCH_BYTES);
    return err(LB3DC_EINVAL, m);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return err(LB3DC_ECUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return err(LB3DC_EINVAL, "device ordinal out of range");
  unsigned char *base;
  {
    // Set-up, once per device (and again after the device's context was
    // torn down and recreated) with that device current: the device
    // address of the scratch array.
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long id = current_ctx_id();
    if (!g_addr[dev] || id == 0 || id != g_ctx_id[dev]) {
      void *ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) return err(LB3DC_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[dev] = (unsigned char *)ptr;
      g_ctx_id[dev] = current_ctx_id();  // the lookup made the context current
    }
    base = g_addr[dev];
  }
  const int nc = p->ncomp;
  unsigned char *cur = base;
  auto take = [&](size_t bytes) {
    unsigned char *r = cur;
    cur += up256(bytes);
    return r;
  };
  double *g = (double *)take((size_t)nc * 19 * n * 8);
  double *rho = (double *)take((size_t)nc * n * 8);
  double *psi = (double *)take((size_t)nc * n * 8);
  double *mom = (double *)take((size_t)nc * 3 * n * 8);
  double *da = nc == 3 ? (double *)take((size_t)3 * n * 8) : nullptr;
  const uint8_t *rk = rock;
  cudaStream_t st = (cudaStream_t)stream;
  if (!rk) {
    // The kernels read a rock mask; without one from the caller, a cleared
    // part of the scratch serves (the array keeps the last call's bytes).
    uint8_t *zero = (uint8_t *)take((size_t)n);
    e = cudaMemsetAsync(zero, 0, (size_t)n, st);
    if (e != cudaSuccess) return err(LB3DC_ECUDA, cudaGetErrorString(e));
    rk = zero;
  }
  lb3d::DevParams P = lb3d::dev_params_from(*p);
  P.any_rock = rock ? 1 : 0;  // a caller's mask may hold rock
  for (int s = 0; s < nsteps; ++s) {
    // Every scratch field is written by the stream kernel before the dipole
    // and collide kernels read it, so nothing else needs clearing.
    e = lb3d::fp64_stream(P, f, g, rho, psi, mom, da, db, rk, nullptr, nullptr, st);
    if (e == cudaSuccess && nc == 3) e = lb3d::fp64_dipole(P, rho, da, db, st);
    if (e == cudaSuccess)
      e = lb3d::fp64_collide(P, g, f, rho, psi, mom, db, rk, nullptr, nullptr, st);
    if (e != cudaSuccess) return err(LB3DC_ECUDA, cudaGetErrorString(e));
  }
  return LB3DC_OK;
}
