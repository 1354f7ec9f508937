// capi.cu -- the C ABI (include/lb3dc.h): handles, state transfer, the
// time-loop stages and the host-side FP64 bookkeeping of the boundary
// conditions.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/lb3dc.h"
#include "common.cuh"
#include "detmath.h"
#include "fp32_path.h"
#include "fp64_path.h"
#include "params.h"
#include "reduce.h"

using namespace lb3d;

struct lb3dc_handle {
  lb3dc_params p;
  DevParams P;
  int device = 0;
  cudaStream_t stream = nullptr;
  // FP64 path
  double *f = nullptr, *g = nullptr, *rho = nullptr, *psi = nullptr, *mom = nullptr;
  double *da = nullptr, *db = nullptr;
  double *hlo = nullptr, *hhi = nullptr, *rlo = nullptr, *rhi = nullptr, *plo = nullptr,
         *phi = nullptr;
  // FP32 deviation path
  Fp32State s32;
  // shared
  uint8_t *rock = nullptr;
  double *scratch = nullptr;  // dump output / reduction partials
  long long scratch_bytes = 0;
  long long bytes = 0;
  // host bookkeeping
  int nt = 0;
  bool le = false, loaded = false;
  double shear_u = 0.0, shear_tmp = 0.0, shear_sum = 0.0, lefrac = 0.0;
  int lelo = 0;
  bool pending_advection = false;  // FP32 path: advection deferred into collision
  KernelTimer timer;
  std::string err;
  int errcode = 0;
  // asynchronous file writers: a pinned host copy of what is being written
  // and the thread that converts it to XDR and writes the file
  void *io_pin = nullptr;
  size_t io_pin_bytes = 0;
  std::thread io_thread;
  int io_status = 0;
};

namespace {

std::string g_create_err;
int g_create_code = 0;

int fail(lb3dc_handle *h, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) {
    h->err = buf;
    h->errcode = code;
  } else {
    g_create_err = buf;
    g_create_code = code;
  }
  return code;
}

#define CK(h, call)                                                                      \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail((h), LB3DC_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

template <typename T>
int dalloc(lb3dc_handle *h, T **ptr, size_t count) {
  if (count == 0) {
    *ptr = nullptr;
    return 0;
  }
  cudaError_t e = cudaMalloc((void **)ptr, count * sizeof(T));
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return fail(h, LB3DC_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T),
                cudaGetErrorString(e));
  }
  h->bytes += (long long)(count * sizeof(T));
  cudaMemsetAsync(*ptr, 0, count * sizeof(T), h->stream);
  return 0;
}

// Clears the populations (ncq arrays of n sites) and, when given, the
// dipole arrays of rock sites.
__global__ void k_clear_rock(double *f, int ncq, double *db, double *da, const uint8_t *rock,
                             long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || rock[i] == 0) return;
  for (int cq = 0; cq < ncq; ++cq) f[cq * n + i] = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (db) db[k * n + i] = 0.0;
    if (da) da[k * n + i] = 0.0;
  }
}

int validate(const lb3dc_params *p, std::string &why) {
  if (!p) return (why = "params is NULL", LB3DC_EINVAL);
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return (why = "lattice sizes must be >= 1", LB3DC_EINVAL);
  if ((long long)p->nx * p->ny * p->nz > (1LL << 34))
    return (why = "lattice too large", LB3DC_EINVAL);
  if (p->ncomp != 2 && p->ncomp != 3) return (why = "ncomp must be 2 or 3", LB3DC_EINVAL);
  if (p->bdist != 2) return (why = "only bdist = 2 is implemented", LB3DC_ENOTSUP);
  bool le = p->boundary_cond != 0 && (p->inv_fluid == 5 || p->inv_fluid == 6);
  if (p->ncomp == 3 && le)
    return (why = "FATAL: Lees Edwards BC are not supported for ternary mixtures", LB3DC_EINVAL);
  const bool zouhe = p->boundary_cond != 0 && p->inv_fluid == 12;
  if (zouhe && p->nz < 2)
    return (why = "the Zou-He flux boundaries need two distinct z planes (nz >= 2)", LB3DC_EINVAL);
  if (zouhe && p->inv_type != 0 && p->inv_type != 1 && p->inv_type != -1)
    return (why = "inv_type must be 0, 1 or -1 for the Zou-He flux boundaries", LB3DC_EINVAL);
  // recolouring inflow, lbe_invade_binary: binary builds only
  // (code/lb3d_invasion.F90:80-85)
  const bool recolour = p->boundary_cond != 0 && (p->inv_fluid == 7 || p->inv_fluid == 8);
  if (recolour && p->ncomp != 2)
    return (why = "Illegal value: inv_fluid 7/8 (recolouring) exists in binary builds only", LB3DC_EINVAL);
  if (recolour && p->nz < 2)
    return (why = "the recolouring boundaries need two z planes (nz >= 2)", LB3DC_EINVAL);
  const bool zh_density = p->boundary_cond != 0 && p->inv_fluid == 11;
  if (zh_density && p->nz < 2)
    return (why = "the Zou-He density boundaries need two distinct z planes (nz >= 2)", LB3DC_EINVAL);
  if (p->boundary_cond != 0 && p->inv_fluid >= 0 && !le && !zouhe && !recolour && !zh_density)
    return (why = "invasion boundaries are not implemented", LB3DC_ENOTSUP);
  if (p->boundary_cond > 0) return (why = "boundary_cond > 0 is not implemented", LB3DC_ENOTSUP);
  if (p->tau_r <= 0 || p->tau_b <= 0 || (p->ncomp == 3 && (p->tau_s <= 0 || p->tau_d <= 0)))
    return (why = "relaxation times must be positive", LB3DC_EINVAL);
  if (p->amass_r <= 0 || p->amass_b <= 0 || (p->ncomp == 3 && p->amass_s <= 0))
    return (why = "amass must be positive", LB3DC_EINVAL);
  if (p->precision != LB3DC_FP64 && p->precision != LB3DC_FP32_DEV)
    return (why = "precision must be LB3DC_FP64 or LB3DC_FP32_DEV", LB3DC_EINVAL);
  if (p->precision == LB3DC_FP64 &&
      (long long)p->nx * p->ny * p->nz + 2LL * p->ny * p->nz >= (1LL << 31))
    return (why = "FP64 lattices are limited to 2^31 sites including the Lees-Edwards planes",
            LB3DC_EINVAL);
  // FP32 population offsets within a component are unsigned 32-bit
  if (p->precision == LB3DC_FP32_DEV && 19LL * p->nx * p->ny * p->nz >= (1LL << 32))
    return (why = "FP32 lattices are limited to 19*sites < 2^32 (226,050,910 sites)", LB3DC_EINVAL);

  return LB3DC_OK;
}

DevParams make_dev_params(const lb3dc_params &p) {
  DevParams P{};
  P.nx = p.nx;
  P.ny = p.ny;
  P.nz = p.nz;
  P.nc = p.ncomp;
  P.nsites = (long long)p.nx * p.ny * p.nz;
  P.tau[0] = p.tau_r;
  P.tau[1] = p.tau_b;
  P.tau[2] = p.tau_s;
  P.amass[0] = p.amass_r;
  P.amass[1] = p.amass_b;
  P.amass[2] = p.amass_s;
  // omega = 1/tau (code/lb3d_config.F90:886-889); the surfactant slot of a
  // binary mixture is unused.
  for (int c = 0; c < 3; ++c) P.omega[c] = 1.0 / P.tau[c];
  P.omega_d = 1.0 / p.tau_d;
  P.g_br = p.g_br;
  P.g_bs = p.g_bs;
  P.g_ss = p.g_ss;
  P.g_wr = p.g_wr;
  P.g_wb = p.g_wb;
  P.tau_wr = p.tau_wr;
  P.tau_wb = p.tau_wb;
  P.beta = p.beta;
  P.d_0 = p.d_0;
  P.g_accn = p.g_accn;
  P.g_accn_x = p.g_accn_x;
  P.g_accn_y = p.g_accn_y;
  P.g_accn_min = p.g_accn_min;
  P.g_accn_max = p.g_accn_max;
  P.g_accn_min_x = p.g_accn_min_x;
  P.g_accn_max_x = p.g_accn_max_x;
  P.g_accn_min_y = p.g_accn_min_y;
  P.g_accn_max_y = p.g_accn_max_y;
  P.inv_fluid = p.inv_fluid;
  // lbe_init_rock_colour colours rock sites only with positive colours
  // (code/lb3d_ic_rock.F90:176-183).
  P.rc_r = p.rock_colour_r > 0 ? p.rock_colour_r : 0.0;
  P.rc_b = p.rock_colour_b > 0 ? p.rock_colour_b : 0.0;
  P.psi_rc[0] = 1.0 - lb3d_detmath::det_exp(-(0.0 + P.rc_r));
  P.psi_rc[1] = 1.0 - lb3d_detmath::det_exp(-(0.0 + P.rc_b));
  P.le = (p.boundary_cond != 0 && (p.inv_fluid == 5 || p.inv_fluid == 6)) ? 1 : 0;
  P.any_rock = 1;  // until a state without rock is uploaded
  P.zouhe = (p.boundary_cond != 0 && p.inv_fluid == 12) ? 1 : 0;
  P.inv_type = p.inv_type;
  P.zh_uz[0] = p.pr;
  P.zh_uz[1] = p.pb;
  P.zh_uz[2] = p.pg;
  P.invk = p.boundary_cond == 0 ? 0
           : (p.inv_fluid == 7 || p.inv_fluid == 8) ? 1
           : p.inv_fluid == 11 ? 2 : p.inv_fluid == 12 ? 3 : 0;
  P.zh_in[0] = p.fr;
  P.zh_in[1] = p.fb;
  return P;
}

long long footprint_bytes(const lb3dc_params &p) {
  const long long N = (long long)p.nx * p.ny * p.nz, nc = p.ncomp;
  const long long np = (long long)p.ny * p.nz;
  long long b = N;  // rock
  if (p.precision == LB3DC_FP64) {
    b += 2 * nc * 19 * N * 8;           // f, g
    b += 2 * nc * N * 8 + nc * 3 * N * 8;  // rho, psi, mom
    if (nc == 3) b += 6 * N * 8;        // da, db
    bool le = p.boundary_cond != 0 && (p.inv_fluid == 5 || p.inv_fluid == 6);
    if (le) b += 2 * nc * 19 * np * 8 + 4 * nc * np * 8;
  } else {
    b += fp32_footprint(p);
  }
  return b;
}

// le_neighbours, code/lb3d_bc_leesedwards.F90:86-140 (one rank).
void le_neighbours(lb3dc_handle *h) {
  if (h->p.inv_fluid == 6) {
    h->shear_u = 0.0;
    h->lelo = h->p.nz / 2 + 1;
    h->lefrac = 0.0;
  } else {
    h->shear_sum = h->shear_sum + h->shear_u;
    h->lelo = ((int)(2.0 * h->shear_sum)) % h->p.nz;
    double s = 2.0 * h->shear_sum;
    h->lefrac = std::fabs(s - std::trunc(s));
  }
}

LEStep le_step(const lb3dc_handle *h) {
  LEStep S;
  S.shear_u = h->shear_u;
  S.lefrac = h->lefrac;
  S.eoff = h->lelo >= 0 ? h->lelo : h->lelo - 1;
  return S;
}

int need_loaded(lb3dc_handle *h) {
  if (!h) return LB3DC_EINVAL;
  if (!h->loaded) return fail(h, LB3DC_ESTATE, "no state loaded (call lb3dc_upload_state first)");
  cudaSetDevice(h->device);
  return LB3DC_OK;
}

// The FP64 time loop streams inside the collision (fp64_step_pull) unless
// something runs between the two: the Lees-Edwards stage-8 halo or an
// invasion boundary on the post-stream populations.
bool fp64_pull_ok(const lb3dc_handle *h) {
  if (h->p.precision != LB3DC_FP64 || h->le || h->P.zouhe) return false;
  const int k = h->p.inv_fluid;
  return !(h->p.boundary_cond != 0 && (k == 11 || k == 7 || k == 8));
}

int ensure_scratch(lb3dc_handle *h, long long bytes) {
  if (h->scratch_bytes >= bytes) return 0;
  if (h->scratch) {
    cudaFree(h->scratch);
    h->bytes -= h->scratch_bytes;
  }
  h->scratch = nullptr;
  h->scratch_bytes = 0;
  int rc = dalloc(h, (unsigned char **)&h->scratch, (size_t)bytes);
  if (rc) return rc;
  h->scratch_bytes = bytes;
  return 0;
}

}  // namespace

namespace lb3d {
int validate_params(const lb3dc_params *p, std::string &why) { return validate(p, why); }
DevParams dev_params_from(const lb3dc_params &p) { return make_dev_params(p); }
int set_global_error(int code, const char *msg) { return fail(nullptr, code, "%s", msg); }
}  // namespace lb3d

extern "C" {

const char *lb3dc_version(void) { return "lb3d_b200 0.1 (sm_100a)"; }

long long lb3dc_footprint(const lb3dc_params *p) {
  std::string why;
  if (validate(p, why) != LB3DC_OK) return -1;
  return footprint_bytes(*p);
}

int lb3dc_create(const lb3dc_params *p, lb3dc_handle **out) {
  if (!out) return fail(nullptr, LB3DC_EINVAL, "out is NULL");
  *out = nullptr;
  std::string why;
  int rc = validate(p, why);
  if (rc != LB3DC_OK) return fail(nullptr, rc, "%s", why.c_str());
  lb3dc_handle *h = new lb3dc_handle();
  h->p = *p;
  h->P = make_dev_params(*p);
  h->le = h->P.le != 0;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    int code = fail(nullptr, LB3DC_ECUDA, "CUDA device unavailable: %s", cudaGetErrorString(e));
    delete h;
    return code;
  }
  const size_t N = (size_t)h->P.nsites, nc = (size_t)p->ncomp;
  const size_t np = (size_t)p->ny * p->nz;
  rc = dalloc(h, &h->rock, N);
  if (!rc && p->precision == LB3DC_FP64) {
    rc = rc ? rc : dalloc(h, &h->f, nc * 19 * N);
    rc = rc ? rc : dalloc(h, &h->g, nc * 19 * N);
    rc = rc ? rc : dalloc(h, &h->rho, nc * N);
    rc = rc ? rc : dalloc(h, &h->psi, nc * N);
    rc = rc ? rc : dalloc(h, &h->mom, nc * 3 * N);
    if (nc == 3) {
      rc = rc ? rc : dalloc(h, &h->da, 3 * N);
      rc = rc ? rc : dalloc(h, &h->db, 3 * N);
    }
    if (h->le) {
      rc = rc ? rc : dalloc(h, &h->hlo, nc * 19 * np);
      rc = rc ? rc : dalloc(h, &h->hhi, nc * 19 * np);
      rc = rc ? rc : dalloc(h, &h->rlo, nc * np);
      rc = rc ? rc : dalloc(h, &h->rhi, nc * np);
      rc = rc ? rc : dalloc(h, &h->plo, nc * np);
      rc = rc ? rc : dalloc(h, &h->phi, nc * np);
    }
  } else if (!rc) {
    rc = fp32_alloc(h->P, *p, h->s32, h->stream);
    if (rc) fail(h, rc, "FP32 state allocation failed");
    h->bytes += h->s32.bytes;
  }
  if (!rc) {
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(h, LB3DC_ECUDA, "%s", cudaGetErrorString(e));
  }
  if (rc) {
    g_create_err = h->err;
    g_create_code = rc;
    lb3dc_destroy(h);
    return rc;
  }
  h->shear_u = p->shear_u;
  *out = h;
  return LB3DC_OK;
}

int lb3dc_destroy(lb3dc_handle *h) {
  if (!h) return LB3DC_OK;
  if (h->io_thread.joinable()) h->io_thread.join();
  cudaSetDevice(h->device);
  if (h->io_pin) cudaFreeHost(h->io_pin);
  if (h->stream) cudaStreamSynchronize(h->stream);
  double *bufs[] = {h->f, h->g, h->rho, h->psi, h->mom, h->da, h->db, h->hlo, h->hhi,
                    h->rlo, h->rhi, h->plo, h->phi, h->scratch};
  for (double *b : bufs)
    if (b) cudaFree(b);
  if (h->rock) cudaFree(h->rock);
  fp32_free(h->s32);
  h->timer.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return LB3DC_OK;
}

int lb3dc_last_error(const lb3dc_handle *h, char *buf, int len) {
  const std::string &m = h ? h->err : g_create_err;
  if (buf && len > 0) {
    std::strncpy(buf, m.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return h ? h->errcode : g_create_code;
}

long long lb3dc_device_bytes(const lb3dc_handle *h) { return h ? h->bytes : 0; }

int lb3dc_upload_state(lb3dc_handle *h, const double *n, const double *db, const double *rock,
                       double shear_sum, int nt) {
  if (!h || !n) return h ? fail(h, LB3DC_EINVAL, "n is NULL") : LB3DC_EINVAL;
  if (h->p.ncomp == 3 && !db) return fail(h, LB3DC_EINVAL, "ternary state needs db");
  cudaSetDevice(h->device);
  const size_t N = (size_t)h->P.nsites, nc = (size_t)h->p.ncomp;
  // lbe_init_rock_colour (code/lb3d_ic_rock.F90:146-189): populations and
  // dipoles of rock sites are cleared -- on the device, so the caller's
  // (possibly pinned) arrays are copied as they are.
  bool any = false;
  if (rock) {
    std::vector<uint8_t> rk(N, 0);
    for (size_t i = 0; i < N; ++i)
      if (rock[i] != 0.0) rk[i] = 1, any = true;
    CK(h, cudaMemcpyAsync(h->rock, rk.data(), N, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));  // rk is released at the end of this block
  } else {
    CK(h, cudaMemsetAsync(h->rock, 0, N, h->stream));
  }
  h->P.any_rock = any ? 1 : 0;
  if (h->p.precision == LB3DC_FP64) {
    CK(h, cudaMemcpyAsync(h->f, n, nc * 19 * N * 8, cudaMemcpyHostToDevice, h->stream));
    if (nc == 3) {
      CK(h, cudaMemcpyAsync(h->db, db, 3 * N * 8, cudaMemcpyHostToDevice, h->stream));
      CK(h, cudaMemcpyAsync(h->da, db, 3 * N * 8, cudaMemcpyHostToDevice, h->stream));
    }
    if (any) {
      k_clear_rock<<<(unsigned)((N + 255) / 256), 256, 0, h->stream>>>(
          h->f, (int)(nc * 19), nc == 3 ? h->db : nullptr, nc == 3 ? h->da : nullptr, h->rock,
          (long long)N);
      CK(h, cudaGetLastError());
    }
    CK(h, fp64_moments(h->P, h->f, h->rho, h->psi, h->mom, h->stream));
  } else {
    int rc = fp32_upload(h->P, h->p, h->s32, n, nc == 3 ? db : nullptr, h->rock, h->stream);
    if (rc) return fail(h, rc, "FP32 upload failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  CK(h, cudaStreamSynchronize(h->stream));
  h->nt = nt;
  h->shear_sum = shear_sum;
  h->shear_u = h->p.shear_u;
  h->pending_advection = false;
  // lb3d_bc_init(4), code/lb3d_bc.F90:48-90
  if (h->le) {
    h->shear_u = ((double)h->p.nx / ((double)h->p.nx - 1.0)) * h->p.shear_u;
    h->shear_tmp = h->shear_u;
    if (h->p.restore) h->shear_sum = h->shear_sum - h->shear_u;
    le_neighbours(h);
  }
  h->loaded = true;
  return LB3DC_OK;
}

int lb3dc_download_state(lb3dc_handle *h, double *n, double *db, double *rho, double *mom,
                         double *da) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (h->pending_advection)
    return fail(h, LB3DC_ESTATE, "state is mid-step (advection deferred into collision)");
  const size_t N = (size_t)h->P.nsites, nc = (size_t)h->p.ncomp;
  if (h->p.precision == LB3DC_FP64) {
    if (n) CK(h, cudaMemcpyAsync(n, h->f, nc * 19 * N * 8, cudaMemcpyDeviceToHost, h->stream));
    if (rho) CK(h, cudaMemcpyAsync(rho, h->rho, nc * N * 8, cudaMemcpyDeviceToHost, h->stream));
    if (mom) CK(h, cudaMemcpyAsync(mom, h->mom, nc * 3 * N * 8, cudaMemcpyDeviceToHost, h->stream));
    if (nc == 3) {
      if (db) CK(h, cudaMemcpyAsync(db, h->db, 3 * N * 8, cudaMemcpyDeviceToHost, h->stream));
      if (da) CK(h, cudaMemcpyAsync(da, h->da, 3 * N * 8, cudaMemcpyDeviceToHost, h->stream));
    } else {
      if (db) std::memset(db, 0, 3 * N * 8);
      if (da) std::memset(da, 0, 3 * N * 8);
    }
    CK(h, cudaStreamSynchronize(h->stream));
  } else {
    rc = fp32_download(h->P, h->p, h->s32, n, db, rho, mom, da, h->rock, h->stream);
    if (rc) return fail(h, rc, "FP32 download failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  return LB3DC_OK;
}

int lb3dc_upload_sites(lb3dc_handle *h, const double *whole_N, double shear_sum, int nt) {
  if (!h || !whole_N) return h ? fail(h, LB3DC_EINVAL, "whole_N is NULL") : LB3DC_EINVAL;
  const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz, nc = h->p.ncomp;
  const size_t N = (size_t)nx * ny * nz;
  const int sd = nc == 3 ? 79 : 49;
  std::vector<double> n(nc * 19 * N), db(nc == 3 ? 3 * N : 0), rock(N);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
        size_t a = ((size_t)(x + 1) + (size_t)(nx + 2) * ((size_t)(y + 1) + (size_t)(ny + 2) * (z + 1))) * sd;
        const double *s = whole_N + a;
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) n[((size_t)c * 19 + q) * N + i] = s[24 * c + q];
        if (nc == 3)
          for (int k = 0; k < 3; ++k) db[(size_t)k * N + i] = s[72 + 3 + k];
        rock[i] = s[sd - 1];
      }
  return lb3dc_upload_state(h, n.data(), nc == 3 ? db.data() : nullptr, rock.data(), shear_sum, nt);
}

int lb3dc_download_sites(lb3dc_handle *h, double *whole_N) {
  if (!h || !whole_N) return h ? fail(h, LB3DC_EINVAL, "whole_N is NULL") : LB3DC_EINVAL;
  const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz, nc = h->p.ncomp;
  const size_t N = (size_t)nx * ny * nz;
  const int sd = nc == 3 ? 79 : 49;
  std::vector<double> n(nc * 19 * N), rho(nc * N), mom(nc * 3 * N), da(3 * N), db(3 * N), rk(N);
  int rc = lb3dc_download_state(h, n.data(), db.data(), rho.data(), mom.data(), da.data());
  if (rc) return rc;
  rc = lb3dc_dump(h, "rock", rk.data());
  if (rc) return rc;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
        size_t a = ((size_t)(x + 1) + (size_t)(nx + 2) * ((size_t)(y + 1) + (size_t)(ny + 2) * (z + 1))) * sd;
        double *s = whole_N + a;
        for (int c = 0; c < nc; ++c) {
          for (int q = 0; q < 19; ++q) s[24 * c + q] = n[((size_t)c * 19 + q) * N + i];
          s[24 * c + 19] = rho[(size_t)c * N + i];
          for (int k = 0; k < 3; ++k) s[24 * c + 20 + k] = mom[((size_t)c * 3 + k) * N + i];
          double rcol = 0.0;
          if (rk[i] != 0.0) rcol = (c == 0) ? h->P.rc_r : (c == 1) ? h->P.rc_b : 0.0;
          s[24 * c + 23] = rcol;
        }
        if (nc == 3)
          for (int k = 0; k < 3; ++k) {
            s[72 + k] = da[(size_t)k * N + i];
            s[75 + k] = db[(size_t)k * N + i];
          }
        s[sd - 1] = rk[i];
      }
  return LB3DC_OK;
}

int lb3dc_force_apply(lb3dc_handle *h, int stage) {
  if (!h) return LB3DC_EINVAL;
  if (stage != 6 && stage != 8 && stage != 10) return fail(h, LB3DC_EINVAL, "bad stage %d", stage);
  return LB3DC_OK;
}

int lb3dc_bc_apply(lb3dc_handle *h, int stage) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (stage == 6) {
    h->nt += 1;
    if (h->le) {
      h->shear_u = h->shear_tmp * std::cos(h->p.shear_omega * (double)h->nt);
      le_neighbours(h);
      if (h->p.precision == LB3DC_FP64) {
        CK(h, fp64_le_halo(h->P, le_step(h), h->f, h->hlo, h->hhi, nullptr, nullptr, nullptr,
                           nullptr, h->stream));
        h->timer.launches += 1;
      }
    }
    return LB3DC_OK;
  }
  if (stage == 8) {
    if (h->P.zouhe && h->p.precision == LB3DC_FP64) {
      // code/lb3d_bc.F90:125-133: the invasion boundaries come first
      CK(h, fp64_zouhe_flux(h->P, h->g, h->da, h->db, h->rock, h->stream));
      h->timer.launches += 1;
    }
    if (h->p.boundary_cond != 0 && h->p.inv_fluid == 11 && h->p.precision == LB3DC_FP64) {
      CK(h, fp64_zouhe_density(h->P, h->g, h->rock, h->p.fr, h->p.fb, h->p.pr, h->p.pb, h->stream));
      h->timer.launches += 1;
    }
    if (h->p.boundary_cond != 0 && (h->p.inv_fluid == 7 || h->p.inv_fluid == 8) &&
        h->p.precision == LB3DC_FP64) {
      const double mr = h->p.inv_fluid == 7 ? 1.0 : 0.0;
      CK(h, fp64_recolour(h->P, h->g, h->rock, mr, 1.0 - mr, h->stream));
      h->timer.launches += 1;
    }
    if (h->le && h->p.precision == LB3DC_FP64) {
      CK(h, fp64_le_halo(h->P, le_step(h), h->g, nullptr, nullptr, h->rlo, h->rhi, h->plo,
                         h->phi, h->stream));
      h->timer.launches += 1;
    }
    return LB3DC_OK;
  }
  if (stage == 10) return LB3DC_OK;
  return fail(h, LB3DC_EINVAL, "bad stage %d", stage);
}

int lb3dc_advection(lb3dc_handle *h) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (h->p.precision == LB3DC_FP64) {
    h->timer.start(h->stream);
    CK(h, fp64_stream(h->P, h->f, h->g, h->rho, h->psi, h->mom, h->da, h->db, h->rock, h->hlo,
                      h->hhi, h->stream));
    h->timer.stop(h->stream);
    h->timer.launches += h->P.nc;
  } else {
    // The FP32 path streams inside its fused stream-collide kernel.
    h->pending_advection = true;
  }
  return LB3DC_OK;
}

int lb3dc_collision(lb3dc_handle *h) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (h->p.precision == LB3DC_FP64) {
    if (h->p.ncomp == 3) {
      CK(h, fp64_dipole(h->P, h->rho, h->da, h->db, h->stream));
      h->timer.launches += 1;
    }
    h->timer.start(h->stream);
    CK(h, fp64_collide(h->P, h->g, h->f, h->rho, h->psi, h->mom, h->db, h->rock, h->plo,
                       h->phi, h->stream));
    h->timer.stop(h->stream);
    h->timer.launches += 1;
  } else {
    if (!h->pending_advection)
      return fail(h, LB3DC_ESTATE, "collision without a preceding advection");
    LEStep S;
    if (h->le) S = le_step(h);
    rc = fp32_step(h->P, h->s32, h->rock, h->stream, h->le ? &S : nullptr);
    if (rc) return fail(h, LB3DC_ECUDA, "FP32 step failed: %s", cudaGetErrorString(cudaGetLastError()));
    h->pending_advection = false;
  }
  return LB3DC_OK;
}

int lb3dc_time_loop(lb3dc_handle *h, int nsteps) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (nsteps < 0) return fail(h, LB3DC_EINVAL, "nsteps < 0");
  if (h->p.precision == LB3DC_FP32_DEV && !h->le) {
    h->nt += nsteps;
    rc = fp32_run(h->P, h->s32, h->rock, nsteps, h->stream);
    if (rc) return fail(h, LB3DC_ECUDA, "FP32 run failed: %s", cudaGetErrorString(cudaGetLastError()));
    return LB3DC_OK;
  }
  if (fp64_pull_ok(h)) {
    // stages 6 and 8 have nothing to do here; each step is the moments
    // pass, the dipole relaxation and the pulling collision, f -> g, after
    // which f and g trade places
    for (int s = 0; s < nsteps; ++s) {
      h->nt += 1;
      h->timer.start(h->stream);
      CK(h, fp64_step_pull(h->P, h->f, h->g, h->rho, h->psi, h->mom, h->da, h->db, h->rock,
                           h->stream));
      h->timer.stop(h->stream);
      h->timer.launches += h->P.nc + (h->p.ncomp == 3 ? 1 : 0) + 1;
      std::swap(h->f, h->g);
    }
    return LB3DC_OK;
  }
  for (int s = 0; s < nsteps; ++s) {
    if ((rc = lb3dc_force_apply(h, 6)) || (rc = lb3dc_bc_apply(h, 6)) || (rc = lb3dc_advection(h)) ||
        (rc = lb3dc_bc_apply(h, 8)) || (rc = lb3dc_force_apply(h, 8)) || (rc = lb3dc_collision(h)))
      return rc;
  }
  return LB3DC_OK;
}

int lb3dc_sync(lb3dc_handle *h) {
  if (!h) return LB3DC_EINVAL;
  cudaSetDevice(h->device);
  CK(h, cudaStreamSynchronize(h->stream));
  CK(h, cudaGetLastError());
  if (h->p.precision == LB3DC_FP32_DEV) {
    const int rc = fp32_take_error(h->s32, h->stream);
    if (rc) return fail(h, rc, "a bounded device-side wait of the FP32 path gave up");
  }
  return LB3DC_OK;
}

void *lb3dc_stream(const lb3dc_handle *h) { return h ? (void *)h->stream : nullptr; }

int lb3dc_set_profiling(lb3dc_handle *h, int enable) {
  if (!h) return LB3DC_EINVAL;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  h->timer.reset();
  h->timer.on = enable != 0;
  h->s32.timer = &h->timer;
  return LB3DC_OK;
}

int lb3dc_kernel_stats(lb3dc_handle *h, double *ms_total, long long *launches,
                       long long *all_launches) {
  if (!h) return LB3DC_EINVAL;
  cudaSetDevice(h->device);
  long long n = 0;
  double ms = h->timer.collect(&n);
  if (ms_total) *ms_total = ms;
  if (launches) *launches = n;
  if (all_launches) *all_launches = h->timer.launches;
  return LB3DC_OK;
}

int lb3dc_set_launch_shape(lb3dc_handle *h, int tx, int ty, int zc, int split) {
  if (!h) return LB3DC_EINVAL;
  if (h->p.precision != LB3DC_FP32_DEV) return fail(h, LB3DC_ENOTSUP, "launch shape applies to the FP32 path");
  cudaSetDevice(h->device);
  int rc = fp32_set_shape(h->P, h->s32, FusedShape{tx, ty, zc, split}, h->stream);
  return rc ? fail(h, rc, "unsupported launch shape %dx%dx%d split %d", tx, ty, zc, split) : LB3DC_OK;
}

int lb3dc_get_launch_shape(const lb3dc_handle *h, int *tx, int *ty, int *zc, int *split) {
  if (!h) return LB3DC_EINVAL;
  if (split) *split = h->s32.split;
  if (tx) *tx = h->s32.tx;
  if (ty) *ty = h->s32.ty;
  if (zc) *zc = h->s32.zc;
  return LB3DC_OK;
}

int lb3dc_autotune(lb3dc_handle *h, double *ms_out, int *ntried) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (h->p.precision != LB3DC_FP32_DEV) return fail(h, LB3DC_ENOTSUP, "autotune applies to the FP32 path");
  LEStep S;
  if (h->le) S = le_step(h);  // tune on this step's offset (the state is restored)
  rc = fp32_autotune(h->P, h->s32, h->rock, ms_out, ntried, h->stream, h->le ? &S : nullptr);
  return rc ? fail(h, rc, "autotune failed: %s", cudaGetErrorString(cudaGetLastError())) : LB3DC_OK;
}

int lb3dc_set_lees_edwards(lb3dc_handle *h, double shear_sum, double shear_u) {
  if (!h) return LB3DC_EINVAL;
  h->shear_sum = shear_sum;
  h->shear_u = shear_u;
  h->shear_tmp = shear_u;
  return LB3DC_OK;
}

int lb3dc_get_lees_edwards(const lb3dc_handle *h, double *shear_sum, double *shear_u) {
  if (!h) return LB3DC_EINVAL;
  if (shear_sum) *shear_sum = h->shear_sum;
  if (shear_u) *shear_u = h->shear_u;
  return LB3DC_OK;
}

int lb3dc_get_timestep(const lb3dc_handle *h, int *nt) {
  if (!h || !nt) return LB3DC_EINVAL;
  *nt = h->nt;
  return LB3DC_OK;
}

int lb3dc_reduce_conservation(lb3dc_handle *h, double mass[3], double mom[3]) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (!mass || !mom) return fail(h, LB3DC_EINVAL, "NULL output");
  rc = ensure_scratch(h, reduce_scratch_bytes(h->P.nsites));
  if (rc) return rc;
  cudaError_t e;
  if (h->p.precision == LB3DC_FP64)
    e = reduce_conservation_fp64(h->P, h->f, h->rock, h->scratch, mass, mom, h->stream);
  else
    e = fp32_reduce_conservation(h->P, h->s32, h->rock, h->scratch, mass, mom, h->stream);
  CK(h, e);
  return LB3DC_OK;
}

int lb3dc_sanity(lb3dc_handle *h, long long *n_nonfinite, long long *n_negative) {
  int rc = need_loaded(h);
  if (rc) return rc;
  rc = ensure_scratch(h, 64);
  if (rc) return rc;
  unsigned long long cnt[2] = {0, 0};
  cudaError_t e;
  if (h->p.precision == LB3DC_FP64)
    e = sanity_counts_fp64(h->P, h->f, (unsigned long long *)h->scratch, cnt, h->stream);
  else
    e = fp32_sanity_counts(h->P, h->s32, (unsigned long long *)h->scratch, cnt, h->stream);
  CK(h, e);
  if (n_nonfinite) *n_nonfinite = (long long)cnt[0];
  if (n_negative) *n_negative = (long long)cnt[1];
  return cnt[0] ? fail(h, LB3DC_ENAN, "%llu non-finite populations", cnt[0]) : LB3DC_OK;
}

int lb3dc_sanity_velocity(lb3dc_handle *h, double maxvel[9], int maxpos[27], double velsum[9],
                          long long *n_fluid, long long *n_too_fast) {
  int rc = need_loaded(h);
  if (rc) return rc;
  rc = ensure_scratch(h, reduce_scratch_bytes(h->P.nsites));
  if (rc) return rc;
  SanityVelocity v;
  cudaError_t e;
  if (h->p.precision == LB3DC_FP64)
    e = sanity_velocity_fp64(h->P, h->f, h->rock, h->scratch, v, h->stream);
  else
    e = fp32_sanity_velocity(h->P, h->s32, h->rock, h->scratch, v, h->stream);
  CK(h, e);
  for (int k = 0; k < 9; ++k) {
    if (maxvel) maxvel[k] = v.vmax[k];
    if (velsum) velsum[k] = v.vsum[k];
    if (maxpos)
      for (int a = 0; a < 3; ++a) maxpos[3 * k + a] = v.pos[k][a];
  }
  if (n_fluid) *n_fluid = v.n_fluid;
  if (n_too_fast) *n_too_fast = v.n_too_fast;
  return LB3DC_OK;
}

int lb3dc_dump(lb3dc_handle *h, const char *field, double *out) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (!field || !out) return fail(h, LB3DC_EINVAL, "NULL argument");
  static const char *names[] = {"od", "wd", "sur", "dir", "vel", "arr", "rock"};
  int fid = -1;
  for (int k = 0; k < 7; ++k)
    if (std::strcmp(field, names[k]) == 0) fid = k;
  if (fid < 0) return fail(h, LB3DC_EINVAL, "unknown dump field '%s'", field);
  const long long N = h->P.nsites;
  const int vps = (fid == 3 || fid == 5) ? 3 : 1;
  if (h->p.precision == LB3DC_FP64) {
    rc = ensure_scratch(h, N * vps * 8);
    if (rc) return rc;
    CK(h, fp64_dump(h->P, fid, h->f, h->rho, h->psi, h->db, h->rock, h->scratch, h->stream));
  } else {
    rc = ensure_scratch(h, N * vps * 8);
    if (rc) return rc;
    rc = fp32_dump(h->P, h->s32, fid, h->rock, h->scratch, h->stream);
    if (rc) return fail(h, rc, "FP32 dump failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  CK(h, cudaMemcpyAsync(out, h->scratch, (size_t)N * vps * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return LB3DC_OK;
}

// ---- asynchronous checkpoint and dump files --------------------------------
// The state (or field) is read off the device into a pinned host buffer
// owned by the handle, synchronously; the big-endian conversion and the
// file write run on a host thread while the caller keeps stepping.  One
// write is in flight per handle: a new one first waits for the previous one
// and, if that failed, returns its error instead of starting.
static int io_join(lb3dc_handle *h) {
  if (h->io_thread.joinable()) h->io_thread.join();
  const int s = h->io_status;
  h->io_status = LB3DC_OK;
  return s;
}

static int io_pinned(lb3dc_handle *h, size_t bytes) {
  if (h->io_pin_bytes >= bytes) return LB3DC_OK;
  if (h->io_pin) cudaFreeHost(h->io_pin);
  h->io_pin = nullptr;
  h->io_pin_bytes = 0;
  if (cudaHostAlloc(&h->io_pin, bytes, cudaHostAllocDefault) != cudaSuccess) {
    h->io_pin = nullptr;
    cudaGetLastError();
    return fail(h, LB3DC_ENOMEM, "pinned host buffer of %zu bytes for the file writer", bytes);
  }
  h->io_pin_bytes = bytes;
  return LB3DC_OK;
}

int lb3dc_checkpoint_async(lb3dc_handle *h, const char *path) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (!path) return fail(h, LB3DC_EINVAL, "path is NULL");
  if ((rc = io_join(h))) return fail(h, rc, "the previous asynchronous write failed");
  const size_t N = (size_t)h->P.nsites, nc = (size_t)h->p.ncomp;
  const size_t nn = nc * 19 * N, n3 = nc == 3 ? 3 * N : 0;
  if ((rc = io_pinned(h, (nn + 2 * n3 + N) * 8 + N))) return rc;
  double *n = (double *)h->io_pin, *da = n + nn, *db = da + n3, *rk = db + n3;
  uint8_t *rb = (uint8_t *)(rk + N);
  rc = lb3dc_download_state(h, n, nc == 3 ? db : nullptr, nullptr, nullptr, nc == 3 ? da : nullptr);
  if (rc) return rc;
  CK(h, cudaMemcpyAsync(rb, h->rock, N, cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  const std::string file(path);
  const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
  h->io_thread = std::thread([h, file, nx, ny, nz, nc, N, n, da, db, rk, rb]() {
    // rock sites are written with rock_state 1
    for (size_t i = 0; i < N; ++i) rk[i] = rb[i] ? 1.0 : 0.0;
    h->io_status = lb3dc_xdr_write_checkpoint(file.c_str(), nx, ny, nz, (int)nc, n,
                                              nc == 3 ? da : nullptr, nc == 3 ? db : nullptr, rk);
  });
  return LB3DC_OK;
}

int lb3dc_dump_async(lb3dc_handle *h, const char *field, const char *path, int dump_double) {
  int rc = need_loaded(h);
  if (rc) return rc;
  if (!field || !path) return fail(h, LB3DC_EINVAL, "NULL argument");
  if ((rc = io_join(h))) return fail(h, rc, "the previous asynchronous write failed");
  const long long N = h->P.nsites;
  const int vps = (std::strcmp(field, "dir") == 0 || std::strcmp(field, "arr") == 0) ? 3 : 1;
  if ((rc = io_pinned(h, (size_t)N * vps * 8))) return rc;
  double *v = (double *)h->io_pin;
  if ((rc = lb3dc_dump(h, field, v))) return rc;
  const std::string file(path);
  h->io_thread = std::thread([h, file, v, N, vps, dump_double]() {
    h->io_status = lb3dc_xdr_write_field(file.c_str(), v, N, vps, dump_double);
  });
  return LB3DC_OK;
}

int lb3dc_io_wait(lb3dc_handle *h) {
  if (!h) return LB3DC_EINVAL;
  const int rc = io_join(h);
  return rc ? fail(h, rc, "asynchronous file write failed") : LB3DC_OK;
}

int lb3dc_detmath_eval(int fn, int device, const double *x, double *y, long long n) {
  if (!x || !y || n < 0 || fn < 0 || fn > 2) return LB3DC_EINVAL;
  if (!device) {
    for (long long i = 0; i < n; ++i)
      y[i] = fn == 0 ? lb3d_detmath::det_exp(x[i])
                     : fn == 1 ? lb3d_detmath::det_expm1(x[i]) : lb3d_detmath::det_tanh(x[i]);
    return LB3DC_OK;
  }
  double *dx = nullptr, *dy = nullptr;
  if (cudaMalloc(&dx, (size_t)n * 8 + 8) != cudaSuccess) return LB3DC_ENOMEM;
  if (cudaMalloc(&dy, (size_t)n * 8 + 8) != cudaSuccess) {
    cudaFree(dx);
    return LB3DC_ENOMEM;
  }
  cudaError_t e = cudaMemcpy(dx, x, (size_t)n * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = fp64_detmath(fn, dx, dy, n, 0);
  if (e == cudaSuccess) e = cudaMemcpy(y, dy, (size_t)n * 8, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dy);
  return e == cudaSuccess ? LB3DC_OK : LB3DC_ECUDA;
}

}  // extern "C"
