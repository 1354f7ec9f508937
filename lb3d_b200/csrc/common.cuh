// common.cuh -- D3Q19 tables, device parameter block and index helpers.
#ifndef LB3D_COMMON_CUH
#define LB3D_COMMON_CUH

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/lb3dc.h"

#define LB3D_HDI __host__ __device__ __forceinline__

namespace lb3d {

// D3Q19 lattice of code/lb3d_lattice.F90:137-187 (0-based).  The tables are
// packed into integer constants so that, inside fully unrolled loops, every
// lookup folds to an immediate on the device.
//   q : 0..5 = +-x, +-y, +-z; 6..17 = the 12 diagonals; 18 = rest.
LB3D_HDI constexpr int cx(int q) { return (int)((0x15500aa552ull >> (2 * q)) & 3) - 1; }
LB3D_HDI constexpr int cy(int q) { return (int)((0x10a5252525ull >> (2 * q)) & 3) - 1; }
LB3D_HDI constexpr int cz(int q) { return (int)((0x1222525255ull >> (2 * q)) & 3) - 1; }
// Degeneracy g (2 on the axes, 1 elsewhere); equal to the Shan-Chen weights
// g_sc of code/lb3d_force_shanchen.F90:148-152.
LB3D_HDI constexpr int gw(int q) { return q < 6 ? 2 : 1; }
// Opposite direction, code/lb3d_lattice.F90:173-187.
LB3D_HDI constexpr int bounce(int q) {
  return q == 0 ? 1 : q == 1 ? 0 : q == 2 ? 3 : q == 3 ? 2 : q == 4 ? 5 : q == 5 ? 4
       : q == 6 ? 11 : q == 7 ? 10 : q == 8 ? 13 : q == 9 ? 12 : q == 10 ? 7 : q == 11 ? 6
       : q == 12 ? 9 : q == 13 ? 8 : q == 14 ? 17 : q == 15 ? 16 : q == 16 ? 15
       : q == 17 ? 14 : 18;
}
constexpr int NQ = 19;
constexpr int NMOV = 18;
constexpr int REST = 18;

// Parameter block shared by all kernels (passed by value).
struct DevParams {
  int nx, ny, nz, nc;
  long long nsites;
  double omega[3], tau[3], amass[3];
  double omega_d;
  double g_br, g_bs, g_ss, g_wr, g_wb, tau_wr, tau_wb;
  double beta, d_0;
  double g_accn, g_accn_x, g_accn_y;
  int g_accn_min, g_accn_max, g_accn_min_x, g_accn_max_x, g_accn_min_y, g_accn_max_y;
  int inv_fluid;
  double rc_r, rc_b;  // rock colour at rock sites (0 where not set)
  double psi_rc[2];   // 1 - exp(-rc) (detmath.h), the psi of a rock site whose density is 0
  int le;             // Lees-Edwards on the x-planes
  int any_rock;       // some site is rock (0: the stream kernel skips the rock tests)
  int zouhe;          // Zou-He flux boundaries on the z planes (inv_fluid 12)
  int inv_type;       // their closure: 0, 1 or -1 (flux / density)
  double zh_uz[3];    // their inflow per component: red pr, blue pb, surfactant pg
  // stage-8 inflow kind (boundary_cond != 0): 0 none, 1 recolouring
  // (inv_fluid 7, 8), 2 Zou-He density (11), 3 Zou-He flux (12); the density
  // boundaries impose fr, fb at z = 1 (zh_in) and pr, pb at z = nz (zh_uz)
  int invk;
  double zh_in[2];
};

// Per-step Lees-Edwards values, computed on the host in FP64 exactly as
// le_neighbours does (code/lb3d_bc_leesedwards.F90:86-140).
struct LEStep {
  double shear_u;
  double lefrac;
  int eoff;  // z offset of the bottom halo source: lelo (>= 0) or lelo-1
};

// Optional CUDA-event bracketing of the dominant kernel launches.
struct KernelTimer {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // pairs: start, stop
  long long launches = 0;       // all kernel launches issued by the handle
  void start(cudaStream_t st) {
    if (!on) return;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
    ev.push_back(a);
    ev.push_back(b);
  }
  void stop(cudaStream_t st) {
    if (on && !ev.empty()) cudaEventRecord(ev.back(), st);
  }
  double collect(long long *n) {
    double ms = 0;
    for (size_t i = 0; i + 1 < ev.size(); i += 2) {
      float t = 0;
      cudaEventSynchronize(ev[i + 1]);
      cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      ms += t;
    }
    if (n) *n = (long long)ev.size() / 2;
    return ms;
  }
  void reset() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    ev.clear();
    launches = 0;
  }
};

LB3D_HDI int wrap(int v, int n) {
  v = (v < 0) ? v + n : v;
  return (v >= n) ? v - n : v;
}

LB3D_HDI long long sidx(int x, int y, int z, int nx, int ny) {
  return (long long)x + (long long)nx * ((long long)y + (long long)ny * (long long)z);
}

// Body-force region, code/lb3d_collision.F90:431-460 (1-based global
// coordinates; one rank).
LB3D_HDI bool applyforce(const DevParams &P, int x1, int y1, int z1) {
  if (P.inv_fluid == 9) return (z1 == 1) || (z1 == P.nz);
  if (P.inv_fluid == 20 || P.inv_fluid == 21) return z1 == 1;
  return (z1 >= P.g_accn_min) && (z1 <= P.g_accn_max) && (x1 >= P.g_accn_min_x) &&
         (x1 <= P.g_accn_max_x) && (y1 >= P.g_accn_min_y) && (y1 <= P.g_accn_max_y);
}
LB3D_HDI bool in_accn_box(const DevParams &P, int x1, int y1, int z1) {
  return (z1 >= P.g_accn_min) && (z1 <= P.g_accn_max) && (x1 >= P.g_accn_min_x) &&
         (x1 <= P.g_accn_max_x) && (y1 >= P.g_accn_min_y) && (y1 <= P.g_accn_max_y);
}

}  // namespace lb3d

#endif
