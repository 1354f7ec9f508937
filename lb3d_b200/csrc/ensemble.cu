// ensemble.cu -- many independent lattices advanced by one persistent
// kernel over a packed site index (the batched FP32 deviation path).
//
// Every lattice occupies a contiguous range [base, base + N) of one packed
// site space of capacity S; its populations live at f[(c*19+q)*S + base + i]
// like a single lattice's.  A lattice table (LatDesc: size, parameters,
// parity) and a tile list covering every active lattice drive the same fused
// stream-collide kernel as the single-lattice path, so a lattice advances
// exactly as it would alone (the per-site arithmetic does not depend on which
// tiles or lattices share a launch).  Site ranges are handed out first-fit;
// admission fails with LB3DC_ENOMEM when no range fits, which is how the
// caller's scheduler admits by HBM footprint.  Steps between changes of the
// active set are replayed from a captured CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/lb3dc.h"
#include "fp32_path.h"
#include "params.h"

using namespace lb3d;

struct Member {
  bool used = false;
  long long base = 0, n = 0;
  int remaining = 0;   // steps still to run
  int done_steps = 0;
  bool finished = false;
  bool retiring = false;             // results on their way to the host (async retire)
  cudaEvent_t copied = nullptr;      // recorded on the copy stream after the last copy
  LatDesc desc{};
  lb3dc_params p{};
};

struct lb3dc_ensemble {
  int nc = 3;
  long long S = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  float *f[2] = {nullptr, nullptr};
  float *db[2] = {nullptr, nullptr};
  uint8_t *rock = nullptr;
  LatDesc *d_lat = nullptr;
  Tile *d_tiles = nullptr;
  int max_lat = 0, tile_cap = 0, ntiles = 0, grid = 0;
  std::vector<Member> members;
  std::map<long long, long long> free_ranges;  // base -> length
  FusedShape shape{32, 4, 8, 2};  // fastest measured on the parameter-sweep stream
  float4 *M = nullptr, *J = nullptr;
  double *stage = nullptr;  // FP64 staging of one member's populations (admit / retire)
  size_t stage_bytes = 0;
  cudaStream_t copy_stream = nullptr;  // asynchronous retires
  double *cstage = nullptr;            // their FP64 staging (populations, then dipoles)
  size_t cstage_bytes = 0;
  bool dirty = true;  // tile list must be rebuilt
  bool body = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_steps = 0;
  long long bytes = 0;
  long long steps_launched = 0, site_updates = 0;
  std::string err;
};

namespace {

int efail(lb3dc_ensemble *e, int code, const std::string &m) {
  if (e) e->err = m;
  else set_global_error(code, m.c_str());
  return code;
}

// Device staging for a member's FP64 populations, grown on demand and kept.
bool ensure_stage(lb3dc_ensemble *e, size_t bytes) {
  if (e->stage_bytes >= bytes) return true;
  if (e->stage) cudaFree(e->stage);
  e->stage = nullptr;
  e->stage_bytes = 0;
  if (cudaMalloc(&e->stage, bytes) != cudaSuccess) return false;
  e->stage_bytes = bytes;
  return true;
}

void drop_graph(lb3dc_ensemble *e) {
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->gexec = nullptr;
  e->graph = nullptr;
  e->graph_steps = 0;
}

bool take_range(lb3dc_ensemble *e, long long n, long long *base) {
  for (auto it = e->free_ranges.begin(); it != e->free_ranges.end(); ++it) {
    if (it->second >= n) {
      *base = it->first;
      long long rest = it->second - n;
      long long nb = it->first + n;
      e->free_ranges.erase(it);
      if (rest > 0) e->free_ranges[nb] = rest;
      return true;
    }
  }
  return false;
}

void give_range(lb3dc_ensemble *e, long long base, long long n) {
  auto it = e->free_ranges.emplace(base, n).first;
  auto nx = std::next(it);
  if (nx != e->free_ranges.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    e->free_ranges.erase(nx);
  }
  if (it != e->free_ranges.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      e->free_ranges.erase(it);
    }
  }
}

int rebuild(lb3dc_ensemble *e) {
  std::vector<Tile> tiles;
  e->body = false;
  for (int i = 0; i < (int)e->members.size(); ++i) {
    Member &m = e->members[i];
    if (!m.used || m.remaining <= 0) continue;
    fp32_tiles_for(m.desc, i, e->shape, tiles);
    if (m.desc.flags & LAT_BODY) e->body = true;
  }
  if ((int)tiles.size() > e->tile_cap) {
    if (e->d_tiles) cudaFree(e->d_tiles);
    e->tile_cap = (int)tiles.size() * 2 + 64;
    if (cudaMalloc(&e->d_tiles, (size_t)e->tile_cap * sizeof(Tile)) != cudaSuccess)
      return efail(e, LB3DC_ENOMEM, "tile list allocation failed");
  }
  e->ntiles = (int)tiles.size();
  if (e->ntiles)
    cudaMemcpyAsync(e->d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                    e->stream);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device);
  int per = fp32_fused_ctas_per_sm(e->nc, false, e->body, e->shape);
  if (per < 1) return efail(e, LB3DC_EINVAL, "launch shape does not fit");
  e->grid = std::max(1, std::min(e->ntiles, per * nsm));
  drop_graph(e);
  e->dirty = false;
  return LB3DC_OK;
}

// One step of every active lattice: the fused kernel, then the parity flip.
cudaError_t launch_step(lb3dc_ensemble *e) {
  cudaError_t r = fp32_launch_fused(e->nc, false, e->body, e->shape, e->d_lat, e->d_tiles, e->ntiles,
                                    0, e->f[0], e->f[1], e->db[0], e->db[1], e->rock, e->S,
                                    e->stream, e->M, e->J);
  if (r != cudaSuccess) return r;
  return fp32_flip_parity(e->d_lat, e->max_lat, e->stream);
}

// Seeded initial state on the device, the generator of lb3d_b200/ic.py:
// SplitMix64 of a counter (seed, stream, index); densities rho_c + U(-amp,
// amp); populations n = w_i rho (rest state at zero velocity); unit dipoles
// uniform on the sphere.  Written as FP32 deviations from w_i rho0.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  unsigned long long z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(unsigned long long seed, unsigned long long stream,
                                            unsigned long long idx) {
  unsigned long long key = (idx + (stream << 40)) ^ (seed * 0xD1B54A32D192ED03ull);
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void k_seed_state(float *f, float *db, long long S, long long base, long long N, int nc,
                             unsigned long long seed, double r0, double r1, double r2, double amp,
                             double rho0) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double rb[3] = {r0, r1, r2};
  for (int c = 0; c < nc; ++c) {
    const double rho = rb[c] + (uniform01(seed, 1 + c, i) * (2.0 * amp) - amp);
    for (int q = 0; q < 19; ++q) {
      const double w = q == 18 ? 1.0 / 3.0 : 1.0 / 36.0;
      // rounded step by step (no contraction), as the host generator computes it
      f[((long long)c * 19 + q) * S + base + i] = (float)__dsub_rn(__dmul_rn(rho, w), __dmul_rn(w, rho0));
    }
  }
  if (nc == 3) {
    const double z = 2.0 * uniform01(seed, 11, i) - 1.0;
    const double phi = 2.0 * 3.141592653589793 * uniform01(seed, 12, i);
    const double r = sqrt(fmax(0.0, 1.0 - z * z));
    db[base + i] = (float)(r * cos(phi));
    db[S + base + i] = (float)(r * sin(phi));
    db[2 * S + base + i] = (float)z;
  }
}

int place(lb3dc_ensemble *e, const lb3dc_params *p, int nsteps, int *slot_out, long long *base_out) {
  std::string why;
  int rc = validate_params(p, why);
  if (rc) return efail(e, rc, why);
  if (p->ncomp != e->nc) return efail(e, LB3DC_EINVAL, "ncomp differs from the ensemble's");
  if (p->boundary_cond != 0) return efail(e, LB3DC_ENOTSUP, "ensemble members are periodic");
  if (nsteps < 0) return efail(e, LB3DC_EINVAL, "nsteps < 0");
  int slot = -1;
  for (int i = 0; i < e->max_lat; ++i)
    if (!e->members[i].used) {
      slot = i;
      break;
    }
  if (slot < 0) return efail(e, LB3DC_ENOMEM, "no free lattice slot");
  const long long N = (long long)p->nx * p->ny * p->nz;
  long long base;
  if (!take_range(e, N, &base)) return efail(e, LB3DC_ENOMEM, "no free site range large enough");
  Member &m = e->members[slot];
  m = Member();
  m.used = true;
  m.base = base;
  m.n = N;
  m.remaining = nsteps;
  m.p = *p;
  DevParams P = dev_params_from(*p);
  m.desc = fp32_make_desc(P, p->rho0 > 0 ? p->rho0 : 0.7, base, false);
  m.desc.parity = 0;
  if (nsteps == 0) m.desc.flags &= ~LAT_ACTIVE;
  *slot_out = slot;
  *base_out = base;
  return LB3DC_OK;
}

}  // namespace

extern "C" {

int lb3dc_ensemble_admit_seeded(lb3dc_ensemble *e, const lb3dc_params *p, unsigned long long seed,
                                const double rho[3], double amp, int nsteps, int *slot_out) {
  if (!e || !p || !rho || !slot_out) return efail(e, LB3DC_EINVAL, "NULL argument");
  cudaSetDevice(e->device);
  int slot;
  long long base;
  int rc = place(e, p, nsteps, &slot, &base);
  if (rc) return rc;
  Member &m = e->members[slot];
  k_seed_state<<<(unsigned)((m.n + 255) / 256), 256, 0, e->stream>>>(
      e->f[0], e->db[0], e->S, base, m.n, e->nc, seed, rho[0], rho[1], e->nc == 3 ? rho[2] : 0.0,
      amp, (double)m.desc.rho0);
  if (cudaGetLastError() != cudaSuccess) return efail(e, LB3DC_ECUDA, "seed kernel failed");
  if (cudaMemcpyAsync(e->d_lat + slot, &m.desc, sizeof(LatDesc), cudaMemcpyHostToDevice, e->stream) !=
      cudaSuccess)
    return efail(e, LB3DC_ECUDA, "descriptor upload failed");
  e->dirty = true;
  *slot_out = slot;
  return LB3DC_OK;
}

int lb3dc_ensemble_create(int ncomp, long long capacity_sites, int max_lattices,
                          lb3dc_ensemble **out) {
  if (!out) return efail(nullptr, LB3DC_EINVAL, "out is NULL");
  *out = nullptr;
  if (ncomp != 2 && ncomp != 3) return efail(nullptr, LB3DC_EINVAL, "ncomp must be 2 or 3");
  if (capacity_sites < 1 || capacity_sites * 19 >= (1LL << 32))
    return efail(nullptr, LB3DC_EINVAL, "capacity must satisfy 19*capacity < 2^32 sites");
  if (max_lattices < 1) return efail(nullptr, LB3DC_EINVAL, "max_lattices must be >= 1");
  lb3dc_ensemble *e = new lb3dc_ensemble();
  e->nc = ncomp;
  e->S = capacity_sites;
  e->max_lat = max_lattices;
  cudaGetDevice(&e->device);
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete e;
    return efail(nullptr, LB3DC_ECUDA, "stream creation failed");
  }
  const size_t pop = (size_t)ncomp * 19 * capacity_sites * sizeof(float);
  bool ok = true;
  for (int b = 0; b < 2; ++b) {
    ok = ok && cudaMalloc(&e->f[b], pop) == cudaSuccess;
    if (ncomp == 3) ok = ok && cudaMalloc(&e->db[b], 3 * (size_t)capacity_sites * 4) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&e->rock, (size_t)capacity_sites) == cudaSuccess;
  ok = ok && cudaMalloc(&e->M, (size_t)capacity_sites * fp32_moment_bytes(ncomp)) == cudaSuccess;
  ok = ok && cudaMalloc(&e->d_lat, (size_t)max_lattices * sizeof(LatDesc)) == cudaSuccess;
  if (!ok) {
    lb3dc_ensemble_destroy(e);
    return efail(nullptr, LB3DC_ENOMEM, "ensemble allocation failed");
  }
  cudaMemsetAsync(e->rock, 0, (size_t)capacity_sites, e->stream);
  cudaMemsetAsync(e->d_lat, 0, (size_t)max_lattices * sizeof(LatDesc), e->stream);
  e->bytes = 2 * (long long)pop + (ncomp == 3 ? 24LL * capacity_sites : 0) + capacity_sites +
             capacity_sites * fp32_moment_bytes(ncomp) +
             (long long)max_lattices * sizeof(LatDesc);
  e->members.resize(max_lattices);
  e->free_ranges[0] = capacity_sites;
  cudaStreamSynchronize(e->stream);
  *out = e;
  return LB3DC_OK;
}

int lb3dc_ensemble_destroy(lb3dc_ensemble *e) {
  if (!e) return LB3DC_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graph(e);
  for (int b = 0; b < 2; ++b) {
    if (e->f[b]) cudaFree(e->f[b]);
    if (e->db[b]) cudaFree(e->db[b]);
  }
  if (e->rock) cudaFree(e->rock);
  if (e->M) cudaFree(e->M);
  if (e->J) cudaFree(e->J);
  if (e->d_lat) cudaFree(e->d_lat);
  if (e->d_tiles) cudaFree(e->d_tiles);
  if (e->stage) cudaFree(e->stage);
  if (e->copy_stream) {
    cudaStreamSynchronize(e->copy_stream);
    cudaStreamDestroy(e->copy_stream);
  }
  for (auto &m : e->members)
    if (m.copied) cudaEventDestroy(m.copied);
  if (e->cstage) cudaFree(e->cstage);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return LB3DC_OK;
}

int lb3dc_ensemble_last_error(const lb3dc_ensemble *e, char *buf, int len) {
  if (!e || !buf || len < 1) return LB3DC_EINVAL;
  std::strncpy(buf, e->err.c_str(), (size_t)len - 1);
  buf[len - 1] = 0;
  return LB3DC_OK;
}

int lb3dc_ensemble_set_shape(lb3dc_ensemble *e, int tx, int ty, int zc, int split) {
  if (!e) return LB3DC_EINVAL;
  if (split < 0 || split > 2) return efail(e, LB3DC_EINVAL, "split must be 0, 1 or 2");
  FusedShape sh{tx, ty, zc, split};
  if (fp32_fused_ctas_per_sm(e->nc, false, false, sh) < 1 || zc < 1)
    return efail(e, LB3DC_EINVAL, "unsupported launch shape");
  // the own-moment field is read by the plain split strategy only; it is
  // allocated the first time that strategy is chosen
  if (split == 1 && !e->J) {
    cudaSetDevice(e->device);
    if (cudaMalloc(&e->J, (size_t)e->S * fp32_own_bytes(e->nc)) != cudaSuccess) {
      e->J = nullptr;
      cudaGetLastError();
      return efail(e, LB3DC_ENOMEM, "own-moment field allocation failed");
    }
    e->bytes += e->S * fp32_own_bytes(e->nc);
  }
  e->shape = sh;
  e->dirty = true;
  return LB3DC_OK;
}

int lb3dc_ensemble_admit(lb3dc_ensemble *e, const lb3dc_params *p, const double *n, const double *db,
                         int nsteps, int *slot_out) {
  if (!e || !p || !n || !slot_out) return efail(e, LB3DC_EINVAL, "NULL argument");
  if (e->nc == 3 && !db) return efail(e, LB3DC_EINVAL, "ternary member needs dipoles");
  cudaSetDevice(e->device);
  int slot;
  long long base;
  int rc = place(e, p, nsteps, &slot, &base);
  if (rc) return rc;
  Member &m = e->members[slot];
  const long long N = m.n;
  const double rho0 = m.desc.rho0;
  // FP64 populations to the device, converted there into deviations in the
  // parity-0 buffer's range
  const size_t nb = (size_t)e->nc * 19 * N * sizeof(double);
  if (!ensure_stage(e, nb)) return efail(e, LB3DC_ENOMEM, "staging allocation failed");
  if (cudaMemcpyAsync(e->stage, n, nb, cudaMemcpyHostToDevice, e->stream) != cudaSuccess ||
      fp32_from_fp64(e->stage, e->f[0], e->S, base, N, e->nc, rho0, nullptr, e->stream) != cudaSuccess)
    return efail(e, LB3DC_ECUDA, "upload failed");
  if (e->nc == 3) {
    std::vector<float> d(3 * N);
    for (long long i = 0; i < 3 * N; ++i) d[i] = (float)db[i];
    for (int k = 0; k < 3; ++k)
      if (cudaMemcpyAsync(e->db[0] + (size_t)k * e->S + base, d.data() + (size_t)k * N, N * 4,
                          cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
        return efail(e, LB3DC_ECUDA, "upload failed");
    cudaStreamSynchronize(e->stream);
  }
  if (cudaMemcpyAsync(e->d_lat + slot, &m.desc, sizeof(LatDesc), cudaMemcpyHostToDevice, e->stream) !=
      cudaSuccess)
    return efail(e, LB3DC_ECUDA, "descriptor upload failed");
  cudaStreamSynchronize(e->stream);
  e->dirty = true;
  *slot_out = slot;
  return LB3DC_OK;
}

int lb3dc_ensemble_step(lb3dc_ensemble *e, int max_steps, int *steps_done) {
  if (!e || max_steps < 0) return efail(e, LB3DC_EINVAL, "bad argument");
  cudaSetDevice(e->device);
  if (steps_done) *steps_done = 0;
  // run until max_steps or until the first member finishes
  int chunk = max_steps;
  bool any = false;
  for (auto &m : e->members)
    if (m.used && m.remaining > 0) {
      chunk = std::min(chunk, m.remaining);
      any = true;
    }
  if (!any || chunk == 0) return LB3DC_OK;
  if (e->dirty) {
    int rc = rebuild(e);
    if (rc) return rc;
  }
  // steps are replayed from a graph of `chunk` steps when the same chunk
  // length repeats for an unchanged active set
  if (chunk >= 4) {
    if (!e->gexec || e->graph_steps != chunk) {
      drop_graph(e);
      cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed);
      cudaError_t r = cudaSuccess;
      for (int s = 0; s < chunk && r == cudaSuccess; ++s) r = launch_step(e);
      cudaStreamEndCapture(e->stream, &e->graph);
      if (r != cudaSuccess || !e->graph) return efail(e, LB3DC_ECUDA, "graph capture failed");
      if (cudaGraphInstantiate(&e->gexec, e->graph, 0) != cudaSuccess)
        return efail(e, LB3DC_ECUDA, "graph instantiation failed");
      e->graph_steps = chunk;
    }
    if (cudaGraphLaunch(e->gexec, e->stream) != cudaSuccess) return efail(e, LB3DC_ECUDA, "graph launch failed");
  } else {
    for (int s = 0; s < chunk; ++s)
      if (launch_step(e) != cudaSuccess) return efail(e, LB3DC_ECUDA, "launch failed");
  }
  long long active_sites = 0;
  for (auto &m : e->members) {
    if (!m.used || m.remaining <= 0) continue;
    active_sites += m.n;
    m.remaining -= chunk;
    m.done_steps += chunk;
    m.desc.parity ^= (chunk & 1);
    if (m.remaining == 0) {
      m.finished = true;
      e->dirty = true;
    }
  }
  // finished members stop: clear their ACTIVE flag on the device so that
  // later flips leave their parity alone
  if (e->dirty) {
    for (int i = 0; i < e->max_lat; ++i) {
      Member &m = e->members[i];
      if (m.used && m.remaining == 0 && (m.desc.flags & LAT_ACTIVE)) {
        m.desc.flags &= ~LAT_ACTIVE;
        cudaMemcpyAsync(e->d_lat + i, &m.desc, sizeof(LatDesc), cudaMemcpyHostToDevice, e->stream);
      }
    }
  }
  e->steps_launched += chunk;
  e->site_updates += active_sites * chunk;
  if (steps_done) *steps_done = chunk;
  return LB3DC_OK;
}

int lb3dc_ensemble_sync(lb3dc_ensemble *e) {
  if (!e) return LB3DC_EINVAL;
  cudaSetDevice(e->device);
  cudaError_t r = cudaStreamSynchronize(e->stream);
  return r == cudaSuccess ? LB3DC_OK : efail(e, LB3DC_ECUDA, cudaGetErrorString(r));
}

int lb3dc_ensemble_finished(lb3dc_ensemble *e, int *slots, int max, int *count) {
  if (!e || !count) return LB3DC_EINVAL;
  int k = 0;
  for (int i = 0; i < e->max_lat; ++i)
    if (e->members[i].used && e->members[i].finished) {
      if (slots && k < max) slots[k] = i;
      ++k;
    }
  *count = k;
  return LB3DC_OK;
}

int lb3dc_ensemble_retire(lb3dc_ensemble *e, int slot, double *n, double *db) {
  if (!e || slot < 0 || slot >= e->max_lat || !e->members[slot].used)
    return efail(e, LB3DC_EINVAL, "bad slot");
  cudaSetDevice(e->device);
  Member &m = e->members[slot];
  if (m.retiring) return efail(e, LB3DC_ESTATE, "member is being retired asynchronously");
  const long long N = m.n;
  const int cur = m.desc.parity;
  cudaStreamSynchronize(e->stream);
  if (n) {
    // deviations -> FP64 populations on the device, one copy back
    const size_t nb = (size_t)e->nc * 19 * N * sizeof(double);
    if (!ensure_stage(e, nb)) return efail(e, LB3DC_ENOMEM, "staging allocation failed");
    if (fp32_to_fp64(e->f[cur], e->stage, e->S, m.base, N, e->nc, m.desc.rho0, e->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(n, e->stage, nb, cudaMemcpyDeviceToHost, e->stream) != cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
      return efail(e, LB3DC_ECUDA, "download failed");
  }
  if (db && e->nc == 3) {
    std::vector<float> d(3 * N);
    for (int k = 0; k < 3; ++k)
      cudaMemcpyAsync(d.data() + (size_t)k * N, e->db[cur] + (size_t)k * e->S + m.base, N * 4,
                      cudaMemcpyDeviceToHost, e->stream);
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return efail(e, LB3DC_ECUDA, "download failed");
    for (long long i = 0; i < 3 * N; ++i) db[i] = d[i];
  }
  // free the slot and its range
  LatDesc off{};
  cudaMemcpyAsync(e->d_lat + slot, &off, sizeof(LatDesc), cudaMemcpyHostToDevice, e->stream);
  cudaStreamSynchronize(e->stream);
  give_range(e, m.base, m.n);
  cudaEvent_t keep = m.copied;
  m = Member();
  m.copied = keep;
  e->dirty = true;
  return LB3DC_OK;
}

int lb3dc_ensemble_retire_async(lb3dc_ensemble *e, int slot, double *n, double *db) {
  if (!e || slot < 0 || slot >= e->max_lat || !e->members[slot].used)
    return efail(e, LB3DC_EINVAL, "bad slot");
  Member &m = e->members[slot];
  if (!m.finished || m.retiring) return efail(e, LB3DC_ESTATE, "member is not finished");
  cudaSetDevice(e->device);
  if (!e->copy_stream && cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return efail(e, LB3DC_ECUDA, "copy stream creation failed");
  const long long N = m.n;
  const int cur = m.desc.parity;
  const size_t nb = (size_t)e->nc * 19 * N * sizeof(double), dbb = 3 * (size_t)N * sizeof(double);
  if (e->cstage_bytes < nb + dbb) {
    // the staging is reused in stream order; grow it only when no copy is in flight
    cudaStreamSynchronize(e->copy_stream);
    if (e->cstage) cudaFree(e->cstage);
    e->cstage = nullptr;
    e->cstage_bytes = 0;
    if (cudaMalloc(&e->cstage, nb + dbb) != cudaSuccess) return efail(e, LB3DC_ENOMEM, "staging allocation failed");
    e->cstage_bytes = nb + dbb;
  }
  // the member's last step is queued on the main stream before this point;
  // later steps do not touch it (it is no longer active)
  cudaEvent_t after;
  if (cudaEventCreateWithFlags(&after, cudaEventDisableTiming) != cudaSuccess)
    return efail(e, LB3DC_ECUDA, "event creation failed");
  cudaEventRecord(after, e->stream);
  cudaStreamWaitEvent(e->copy_stream, after, 0);
  cudaEventDestroy(after);
  cudaError_t r = cudaSuccess;
  if (n) {
    r = fp32_to_fp64(e->f[cur], e->cstage, e->S, m.base, N, e->nc, m.desc.rho0, e->copy_stream);
    if (r == cudaSuccess) r = cudaMemcpyAsync(n, e->cstage, nb, cudaMemcpyDeviceToHost, e->copy_stream);
  }
  if (r == cudaSuccess && db && e->nc == 3) {
    double *dst = e->cstage + (size_t)e->nc * 19 * N;
    r = fp32_planes_to_fp64(e->db[cur], dst, e->S, m.base, N, 3, e->copy_stream);
    if (r == cudaSuccess) r = cudaMemcpyAsync(db, dst, dbb, cudaMemcpyDeviceToHost, e->copy_stream);
  }
  if (r == cudaSuccess && !m.copied) r = cudaEventCreateWithFlags(&m.copied, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventRecord(m.copied, e->copy_stream);
  if (r != cudaSuccess) return efail(e, LB3DC_ECUDA, std::string("asynchronous retire: ") + cudaGetErrorString(r));
  m.finished = false;
  m.retiring = true;
  return LB3DC_OK;
}

int lb3dc_ensemble_poll(lb3dc_ensemble *e, int slot, int *done) {
  if (!e || !done || slot < 0 || slot >= e->max_lat || !e->members[slot].used ||
      !e->members[slot].retiring)
    return efail(e, LB3DC_EINVAL, "bad slot");
  Member &m = e->members[slot];
  *done = 0;
  cudaError_t q = cudaEventQuery(m.copied);
  if (q == cudaErrorNotReady) return LB3DC_OK;
  if (q != cudaSuccess) return efail(e, LB3DC_ECUDA, std::string("asynchronous retire: ") + cudaGetErrorString(q));
  // the copies have landed: free the slot and its range
  cudaSetDevice(e->device);
  LatDesc off{};
  cudaMemcpyAsync(e->d_lat + slot, &off, sizeof(LatDesc), cudaMemcpyHostToDevice, e->stream);
  give_range(e, m.base, m.n);
  cudaEvent_t keep = m.copied;
  m = Member();
  m.copied = keep;  // reused by the slot's next retire
  e->dirty = true;
  *done = 1;
  return LB3DC_OK;
}

int lb3dc_host_alloc(long long bytes, void **ptr) {
  if (!ptr || bytes <= 0) return LB3DC_EINVAL;
  *ptr = nullptr;
  return cudaMallocHost(ptr, (size_t)bytes) == cudaSuccess ? LB3DC_OK : LB3DC_ENOMEM;
}

int lb3dc_host_free(void *ptr) {
  if (ptr) cudaFreeHost(ptr);
  return LB3DC_OK;
}

int lb3dc_ensemble_stats(const lb3dc_ensemble *e, long long *free_sites, int *active, int *resident,
                         long long *site_updates) {
  if (!e) return LB3DC_EINVAL;
  long long fs = 0;
  for (auto &r : e->free_ranges) fs += r.second;
  int a = 0, res = 0;
  for (auto &m : e->members) {
    if (m.used) ++res;
    if (m.used && m.remaining > 0) ++a;
  }
  if (free_sites) *free_sites = fs;
  if (active) *active = a;
  if (resident) *resident = res;
  if (site_updates) *site_updates = e->site_updates;
  return LB3DC_OK;
}

long long lb3dc_ensemble_bytes(const lb3dc_ensemble *e) { return e ? e->bytes : 0; }

}  // extern "C"
