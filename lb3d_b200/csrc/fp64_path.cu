// fp64_path.cu -- the FP64 drop-in path (LB3DC_FP64).
//
// Stage-by-stage kernels whose arithmetic is, expression for expression,
// the FP64 restatement of the reference (the oracle): the same operation
// order, no FMA contraction (this file is compiled with --fmad=false) and
// the deterministic exp/tanh of detmath.h, so that the device reproduces
// the host restatement bit for bit.  The 1e-12-after-1000-steps parity
// target is below the chaotic amplification of a single rounding
// difference, which is why bit identity is the design goal here.
//
// Layout in HBM (structure of arrays, site index x fastest):
//   f, g   : [nc][19][nsites]  pre-stream state / post-stream populations
//   rho    : [nc][nsites]      post-stream densities
//   psi    : [nc][nsites]      1 - exp(-rho), evaluated once per site
//   mom    : [nc][3][nsites]   post-stream momenta (the reference's u_*)
//   da, db : [3][nsites]       advected dipole flux / dipoles (ternary)
//   rock   : [nsites] uint8
// Lees-Edwards x-halo planes (binary): [nc][19][nz][ny] pre-stream, and
// [nc][nz][ny] densities after streaming.

#include <cstdio>

#include "common.cuh"
#include "detmath.h"
#include "fp64_path.h"
#include "inflow.cuh"
#include "le_common.cuh"

namespace lb3d {
namespace fp64 {

using lb3d_detmath::det_exp;
using lb3d_detmath::det_tanh;

__device__ __forceinline__ double get_psi(double rho) { return 1.0 - det_exp(-rho); }

__device__ __forceinline__ void site_xyz(long long i, int nx, int ny, int &x, int &y, int &z) {
  long long t = i / nx;
  x = (int)(i - t * nx);
  z = (int)(t / ny);
  y = (int)(t - (long long)z * ny);
}

// src: populations [NC][19][nsites].  Writes the halo planes and, when
// rho_out is given, their densities and psi (for the force stencil).
template <int NC>
__global__ void k_le_halo(DevParams P, LEStep S, const double *__restrict__ src,
                          double *__restrict__ hlo, double *__restrict__ hhi,
                          double *__restrict__ rlo, double *__restrict__ rhi,
                          double *__restrict__ plo, double *__restrict__ phi) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ny * nz) return;
  const int y = t % ny, z = t / ny;
  const long long N = P.nsites;
  const double f = S.lefrac;
  double hb[NC][19], ht[NC][19];
  {
    long long ia = sidx(nx - 1, y, ((z + S.eoff) % nz + nz) % nz, nx, ny);
    long long ib = sidx(nx - 1, y, ((z + S.eoff + 1) % nz + nz) % nz, nx, ny);
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q)
        hb[c][q] = (1.0 - f) * src[(c * 19 + q) * N + ia] + f * src[(c * 19 + q) * N + ib];
    le_adjust<NC>(P, hb, hb, S.shear_u, -1.0);
  }
  {
    long long ia = sidx(0, y, ((z - S.eoff - 1) % nz + nz) % nz, nx, ny);
    long long ib = sidx(0, y, ((z - S.eoff) % nz + nz) % nz, nx, ny);
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q)
        ht[c][q] = f * src[(c * 19 + q) * N + ia] + (1.0 - f) * src[(c * 19 + q) * N + ib];
    le_adjust<NC>(P, ht, hb, S.shear_u, +1.0);
  }
  const long long NP = (long long)ny * nz;
  if (hlo) {
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q) {
        hlo[(c * 19 + q) * NP + t] = hb[c][q];
        hhi[(c * 19 + q) * NP + t] = ht[c][q];
      }
  }
  if (rlo) {
    for (int c = 0; c < NC; ++c) {
      double a = 0.0, b = 0.0;
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        a = a + hb[c][q] * (double)gw(q);
        b = b + ht[c][q] * (double)gw(q);
      }
      rlo[c * NP + t] = a;
      rhi[c * NP + t] = b;
      plo[c * NP + t] = get_psi(a);
      phi[c * NP + t] = get_psi(b);
    }
  }
}

// ---------------------------------------------------------------------------
// Advection: pull streaming with half-way bounce-back, the advected dipole
// flux and the post-stream moments (code/lb3d_advection.F90:54-151,
// code/lb3d_bc_bounce.F90:53-90, code/lb3d_analysis.F90:64-102).
// ---------------------------------------------------------------------------
// One launch per component c (components are independent here; the
// advected dipole flux uses the surfactant only), which keeps one
// component's 19 pulls live per thread; FLUX marks the surfactant launch,
// which also accumulates the dipole flux.  STORE writes the post-stream
// populations to fout and MOM the momenta: the moments pass of the pulling
// step (k_collide with PULL) writes the moments only.
template <int NC, bool LE, bool FLUX, bool ROCK, bool STORE = true, bool MOM = true>
__global__ void __launch_bounds__(256, 2) k_stream(DevParams P, const double *__restrict__ fin,
                                                double *__restrict__ fout, double *__restrict__ rho,
                                                double *__restrict__ psi, double *__restrict__ mom,
                                                double *__restrict__ da,
                                                const double *__restrict__ db,
                                                const uint8_t *__restrict__ rock,
                                                const double *__restrict__ hlo,
                                                const double *__restrict__ hhi, int c) {
  const long long N = P.nsites;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int x, y, z;
  site_xyz(i, nx, ny, x, y, z);
  // without rock every site is fluid and the pulls do not wait on rock loads
  const bool fluid = !ROCK || rock[i] == 0;
  const long long NP = (long long)ny * nz;

  // upstream site of each moving direction (32-bit: the FP64 path bounds a
  // lattice at 2^31 sites); negative values mark the LE halo planes
  int up[18];
  bool upf[18];
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    int xu = x - cx(q), yu = wrap(y - cy(q), ny), zu = wrap(z - cz(q), nz);
    if (LE && xu < 0) {
      up[q] = -1 - (yu + ny * zu);  // bottom halo
      upf[q] = true;
    } else if (LE && xu >= nx) {
      up[q] = -1 - (int)NP - (yu + ny * zu);  // top halo
      upf[q] = true;
    } else {
      up[q] = (int)sidx(wrap(xu, nx), yu, zu, nx, ny);
      upf[q] = !ROCK || rock[up[q]] == 0;
    }
  }
  auto pulled = [&](int c, int q) -> double {
    long long j = up[q];
    if (LE && j < 0) {
      long long h = -1 - j;
      if (h < NP) return hlo[(c * 19 + q) * NP + h];
      return hhi[(c * 19 + q) * NP + (h - NP)];
    }
    return fin[(c * 19 + q) * N + j];
  };

  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
  {
    double n[19];
#pragma unroll
    for (int q = 0; q < 18; ++q) {
      if (fluid)
        n[q] = upf[q] ? pulled(c, q) : fin[(c * 19 + bounce(q)) * N + i];
      else
        n[q] = fin[(c * 19 + q) * N + i];
    }
    n[REST] = fin[(c * 19 + REST) * N + i];
    if (FLUX) {
      // advected dipole flux: bounce-back terms first (lb3d_bc_bounce_back_hw
      // runs before lb3d_advection_step), then the pulls, then the rest
      // population (code/lb3d_advection.F90:137-148).
      if (fluid) {
        if (ROCK) {
#pragma unroll
          for (int s = 0; s < 18; ++s) {
            long long ja = sidx(wrap(x + cx(s), nx), wrap(y + cy(s), ny), wrap(z + cz(s), nz), nx, ny);
            if (rock[ja] != 0) {
              double ng = fin[(2 * 19 + s) * N + i] * (double)gw(s);
              d0 = d0 + ng * db[ja];
              d1 = d1 + ng * db[N + ja];
              d2 = d2 + ng * db[2 * N + ja];
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 18; ++q) {
          if (upf[q]) {
            long long j = up[q];
            double ng = n[q] * (double)gw(q);
            d0 = d0 + ng * db[j];
            d1 = d1 + ng * db[N + j];
            d2 = d2 + ng * db[2 * N + j];
          }
        }
      }
      double ng = n[REST] * (double)gw(REST);
      d0 = d0 + ng * db[i];
      d1 = d1 + ng * db[N + i];
      d2 = d2 + ng * db[2 * N + i];
    }
    double r = 0.0, u0 = 0.0, u1 = 0.0, u2 = 0.0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      if (STORE) fout[(c * 19 + q) * N + i] = n[q];
      r = r + n[q] * (double)gw(q);
    }
    rho[c * N + i] = r;
    psi[c * N + i] = get_psi(r);
    if (MOM) {
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        double ng = n[q] * (double)gw(q);
        u0 = u0 + ng * (double)cx(q);
        u1 = u1 + ng * (double)cy(q);
        u2 = u2 + ng * (double)cz(q);
      }
      mom[(c * 3 + 0) * N + i] = u0;
      mom[(c * 3 + 1) * N + i] = u1;
      mom[(c * 3 + 2) * N + i] = u2;
    }
  }
  if (FLUX) {
    da[i] = d0;
    da[N + i] = d1;
    da[2 * N + i] = d2;
  }
}

// ---------------------------------------------------------------------------
// Zou-He flux boundaries, code/lb3d_invasion.F90:2143-2457 (one rank: both
// z planes are boundary planes).  One thread per site of the z = 1 and
// z = nz planes; per component (surfactant, red, blue) the populations
// entering the lattice are closed from the known ones and the inflow uz
// (divided by the density for inv_type < 0), in the expression order of
// the reference; the surfactant's advected dipole flux is recomputed from
// its new populations and the dipoles of the upstream sites (periodic
// images across the planes, as the stage-6 halo holds them).  Densities
// and velocities keep their advection values, as in the reference.
// F(i) is the reference's 1-based direction i.
// ---------------------------------------------------------------------------
template <int NC>
__global__ void k_zouhe_flux(DevParams P, double *__restrict__ g, double *__restrict__ da,
                             const double *__restrict__ db, const uint8_t *__restrict__ rock) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const long long N = P.nsites;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nx * ny) return;
  const bool bottom = t < nx * ny;
  const int xy = bottom ? t : t - nx * ny;
  const int x = xy % nx, y = xy / nx, z = bottom ? 0 : nz - 1;
  const long long i = sidx(x, y, z, nx, ny);
  if (rock[i] != 0) return;
  const int order[3] = {2, 0, 1};  // surfactant, red, blue
  for (int k = 0; k < 3; ++k) {
    const int c = order[k];
    if (c >= NC) continue;
    double F[19];
    for (int q = 0; q < 19; ++q) F[q] = g[(c * 19 + q) * N + i] * (double)gw(q);
    zouhe_flux_site(F, P.zh_uz[c], bottom, P.inv_type);
    for (int q = 0; q < 19; ++q) g[(c * 19 + q) * N + i] = F[q] / (double)gw(q);
    if (NC == 3 && c == 2) {
      double d0 = 0.0, d1 = 0.0, d2 = 0.0;
      for (int q = 0; q < 19; ++q) {
        const long long j =
            sidx(wrap(x - cx(q), nx), wrap(y - cy(q), ny), wrap(z - cz(q), nz), nx, ny);
        const double ng = g[(2 * 19 + q) * N + i] * (double)gw(q);
        d0 = d0 + ng * db[j];
        d1 = d1 + ng * db[N + j];
        d2 = d2 + ng * db[2 * N + j];
      }
      da[i] = d0;
      da[N + i] = d1;
      da[2 * N + i] = d2;
    }
  }
}

// Zou-He density boundaries, lbe_invade_zouandhe
// (code/lb3d_invasion.F90:1459-1796): the red and blue populations of the
// fluid sites of z = 0 take the densities fr, fb, those of z = nz - 1 the
// densities pr, pb, through the five-population density closure of the
// non-SINGLEFLUID build (Shan-Chen terms zero).  The velocity closure the
// reference runs first writes only populations that this closure
// overwrites, and reads none of them.  F(i) is the reference's 1-based
// direction i; the blue F(13) at z = 0 divides by amass_r as the reference
// writes it (:1567).
__global__ void k_zouhe_density(DevParams P, double *__restrict__ g, const uint8_t *__restrict__ rock,
                                double fr, double fb, double pr, double pb) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const long long N = P.nsites;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nx * ny) return;
  const bool bottom = t < nx * ny;
  const int xy = bottom ? t : t - nx * ny;
  const int x = xy % nx, y = xy / nx, z = bottom ? 0 : nz - 1;
  const long long i = sidx(x, y, z, nx, ny);
  if (rock[i] != 0) return;
  const double rho_c[2] = {bottom ? fr : pr, bottom ? fb : pb};
  for (int c = 0; c < 2; ++c) {
    double F[19];
    for (int q = 0; q < 19; ++q) F[q] = g[(c * 19 + q) * N + i] * (double)gw(q);
    zouhe_density_site(F, rho_c[c], P.amass[c], bottom ? P.amass[0] : P.amass[c], P.tau[c], bottom);
    for (int q = 0; q < 19; ++q) g[(c * 19 + q) * N + i] = F[q] / (double)gw(q);
  }
}

// ---------------------------------------------------------------------------
// Recolouring inflow of binary mixtures, lbe_invade_binary
// (code/lb3d_invasion.F90:1257-1358): on the post-stream populations, the
// bottom planes z = 0, 1 become red = a * (n_r + n_b), blue = b * (n_r + n_b)
// with (a, b) = (mr, mb), then the top planes z = nz - 2, nz - 1 with
// (a, b) = (mb, mr); rock sites are left alone.  One thread per (x, y)
// column runs the four planes in that order, so lattices with nz < 4, whose
// bottom and top planes coincide, are recoloured as the reference does.
// ---------------------------------------------------------------------------
__global__ void k_recolour(DevParams P, double *__restrict__ g, const uint8_t *__restrict__ rock,
                           double mr, double mb) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const long long N = P.nsites;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny) return;
  const int x = t % nx, y = t / nx;
  const int zs[4] = {0, 1, nz - 2, nz - 1};
  for (int k = 0; k < 4; ++k) {
    const long long i = sidx(x, y, zs[k], nx, ny);
    if (rock[i] != 0) continue;
    const double a = k < 2 ? mr : mb, b = k < 2 ? mb : mr;
    for (int q = 0; q < 19; ++q) {
      const double pop = g[q * N + i] + g[(19 + q) * N + i];
      g[q * N + i] = a * pop;
      g[(19 + q) * N + i] = b * pop;
    }
  }
}

// ---------------------------------------------------------------------------
// Dipole relaxation, code/lb3d_collision.F90:296-403 (ternary, periodic).
// Reads rho and da of the 18 neighbours; writes db in place (no neighbour
// reads db in this pass).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dipole(DevParams P, const double *__restrict__ rho,
                                                const double *__restrict__ da,
                                                double *__restrict__ db) {
  const long long N = P.nsites;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int x, y, z;
  site_xyz(i, nx, ny, x, y, z);
  double h_c[3] = {0.0, 0.0, 0.0};
  double h_s[3] = {da[i], da[N + i], da[2 * N + i]};
  double sN_tmp = fmaxf_(rho[2 * N + i], CLIP_RHO_S);
  double sd_tmp[3];
  for (int k = 0; k < 3; ++k) sd_tmp[k] = h_s[k] / sN_tmp;
  const double sgn = (P.g_bs >= 0.0) ? 1.0 : -1.0;
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    long long j = sidx(wrap(x + cx(q), nx), wrap(y + cy(q), ny), wrap(z + cz(q), nz), nx, ny);
    double psi_r = 0.0 + rho[j];
    double psi_b = 0.0 + rho[N + j];
    double pas[3] = {da[j], da[N + j], da[2 * N + j]};
    double hc_m = -(sgn * (psi_b - psi_r) * (double)gw(q));
    const double c[3] = {(double)cx(q), (double)cy(q), (double)cz(q)};
    for (int k = 0; k < 3; ++k) h_c[k] = h_c[k] + hc_m * c[k];
    double hs_dot = 2.0 * ((c[0] * pas[0] + c[1] * pas[1]) + c[2] * pas[2]);
    for (int k = 0; k < 3; ++k) h_s[k] = h_s[k] + (pas[k] - c[k] * hs_dot) * (double)gw(q);
  }
  double h[3];
  for (int k = 0; k < 3; ++k) h[k] = h_c[k] + h_s[k];
  double h_m = P.beta * sqrt((h[0] * h[0] + h[1] * h[1]) + h[2] * h[2]);
  double sd_eq[3];
  const double third = 1.0 / 3.0;
  for (int k = 0; k < 3; ++k) sd_eq[k] = (third * P.beta) * h[k];
  if (h_m > 10.0e-3) {
    double exh = 1.0 / det_tanh(h_m);
    double sd_mag = exh - 1.0 / h_m;
    for (int k = 0; k < 3; ++k) sd_eq[k] = ((P.beta * h[k]) / h_m) * sd_mag;
  }
  for (int k = 0; k < 3; ++k) sd_eq[k] = sd_eq[k] * P.d_0;
  for (int k = 0; k < 3; ++k) db[k * N + i] = P.omega_d * sd_eq[k] + (1.0 - P.omega_d) * sd_tmp[k];
}

// ---------------------------------------------------------------------------
// Shan-Chen forces (code/lb3d_force_shanchen.F90:127-330).  LE selects the
// Lees-Edwards neighbourhood: x-halo sites from the halo planes (never
// rock), and rock neighbours reached through the y/z halo without their
// rock colour (the Lees-Edwards y/z swaps do not copy it, :1079-1308).
// ---------------------------------------------------------------------------
template <bool LE>
__device__ __forceinline__ void sc_force_binary(const DevParams &P, int x, int y, int z, long long i,
                                                const double *__restrict__ rho,
                                                const double *__restrict__ psi,
                                                const uint8_t *__restrict__ rock,
                                                const double *__restrict__ plo,
                                                const double *__restrict__ phi, double *fr,
                                                double *fb) {
  const long long N = P.nsites;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const long long NP = (long long)ny * nz;
  double f_br[3] = {0, 0, 0}, f_rb[3] = {0, 0, 0}, f_wr[3] = {0, 0, 0}, f_wb[3] = {0, 0, 0};
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    const double c[3] = {(double)cx(q), (double)cy(q), (double)cz(q)};
    int xn = x + cx(q), yn = y + cy(q), zn = z + cz(q);
    double psi_r, psi_b;
    bool rk = false;
    if (LE && (xn < 0 || xn >= nx)) {
      long long h = wrap(yn, ny) + (long long)ny * wrap(zn, nz);
      const double *pp = (xn < 0) ? plo : phi;
      psi_r = pp[h];
      psi_b = pp[NP + h];
    } else {
      long long j = sidx(wrap(xn, nx), wrap(yn, ny), wrap(zn, nz), nx, ny);
      if (rock[j] != 0) {
        rk = true;
        bool through_halo = (yn < 0 || yn >= ny || zn < 0 || zn >= nz || xn < 0 || xn >= nx);
        double rcr = (LE && through_halo) ? 0.0 : P.rc_r;
        double rcb = (LE && through_halo) ? 0.0 : P.rc_b;
        // rock sites hold no populations, so their density is 0 and their
        // psi is that of the rock colour alone (evaluated once on the host
        // by the same detmath routine: the same bits)
        const double rj = rho[j], bj = rho[N + j];
        const bool coloured = !(LE && through_halo);
        psi_r = (coloured && rj == 0.0) ? P.psi_rc[0] : get_psi(rj + rcr);
        psi_b = (coloured && bj == 0.0) ? P.psi_rc[1] : get_psi(bj + rcb);
      } else {
        psi_r = psi[j];
        psi_b = psi[N + j];
      }
    }
    double green_r = psi_b * (double)gw(q);
    double green_b = psi_r * (double)gw(q);
    if (rk) {
      for (int k = 0; k < 3; ++k) {
        f_wb[k] = f_wb[k] + green_r * c[k];
        f_wr[k] = f_wr[k] + green_b * c[k];
      }
    } else {
      for (int k = 0; k < 3; ++k) {
        f_rb[k] = f_rb[k] + green_r * c[k];
        f_br[k] = f_br[k] + green_b * c[k];
      }
    }
  }
  double pb = psi[N + i], prr = psi[i];
  for (int k = 0; k < 3; ++k) {
    double br = -(P.g_br * f_br[k]);
    double rb = -(P.g_br * f_rb[k]);
    double wr = -(P.g_wr * f_wr[k]);
    double wb = -(P.g_wb * f_wb[k]);
    fb[k] = (br + ((wb / P.tau[1]) * P.tau_wb)) * pb;
    fr[k] = (rb + ((wr / P.tau[0]) * P.tau_wr)) * prr;
  }
}

__device__ __forceinline__ void sc_force_ternary(const DevParams &P, int x, int y, int z, long long i,
                                                 const double *__restrict__ psi,
                                                 const double *__restrict__ db, double *fr,
                                                 double *fb, double *fs) {
  const long long N = P.nsites;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  double f_br[3] = {0, 0, 0}, f_rb[3] = {0, 0, 0}, f_cs[3] = {0, 0, 0}, f_sc[3] = {0, 0, 0},
         f_ss[3] = {0, 0, 0};
  const double dbx[3] = {db[i], db[N + i], db[2 * N + i]};
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    long long j = sidx(wrap(x + cx(q), nx), wrap(y + cy(q), ny), wrap(z + cz(q), nz), nx, ny);
    const double c[3] = {(double)cx(q), (double)cy(q), (double)cz(q)};
    const double g = (double)gw(q);
    double psi_r = psi[j];
    double psi_b = psi[N + j];
    double green_r = psi_b * g;
    double green_b = psi_r * g;
    for (int k = 0; k < 3; ++k) {
      f_rb[k] = f_rb[k] + green_r * c[k];
      f_br[k] = f_br[k] + green_b * c[k];
    }
    double pss = psi[2 * N + j];
    double dd[3] = {db[j] * pss, db[N + j] * pss, db[2 * N + j] * pss};
    double d_dotc = (dd[0] * c[0] + dd[1] * c[1]) + dd[2] * c[2];
    for (int k = 0; k < 3; ++k) f_cs[k] = f_cs[k] + (dd[k] - (2.0 * d_dotc) * c[k]) * g;
    double di_dotc = (dbx[0] * c[0] + dbx[1] * c[1]) + dbx[2] * c[2];
    double greenc_s = (psi_b - psi_r) * g;
    for (int k = 0; k < 3; ++k) f_sc[k] = f_sc[k] + greenc_s * (dbx[k] - (2.0 * di_dotc) * c[k]);
    double di_dot_d = (dd[0] * dbx[0] + dd[1] * dbx[1]) + dd[2] * dbx[2];
    double green_ss = 8.0 * g;
    for (int k = 0; k < 3; ++k)
      f_ss[k] = f_ss[k] +
                green_ss * (((di_dot_d - (2.0 * di_dotc) * d_dotc) * c[k] + dd[k] * di_dotc) +
                            d_dotc * dbx[k]);
  }
  double pb = psi[N + i], prr = psi[i], ps = psi[2 * N + i];
  for (int k = 0; k < 3; ++k) {
    double br = -(P.g_br * f_br[k]);
    double rb = -(P.g_br * f_rb[k]);
    double sc = (2.0 * P.g_bs) * f_sc[k];
    double cs = -((2.0 * P.g_bs) * f_cs[k]);
    double ss = -(P.g_ss * f_ss[k]);
    fb[k] = (br + cs) * pb;
    fr[k] = (rb - cs) * prr;
    fs[k] = (sc + ss) * ps;
  }
}

template <int NC, bool LE>
__device__ __forceinline__ void sc_forces(const DevParams &P, int x, int y, int z, long long i,
                                          const double *rho, const double *psi, const double *db,
                                          const uint8_t *rock, const double *plo,
                                          const double *phi, double F[NC][3]) {
  for (int c = 0; c < NC; ++c) F[c][0] = F[c][1] = F[c][2] = 0.0;
  if (rock[i] != 0) return;
  if (NC == 2)
    sc_force_binary<LE>(P, x, y, z, i, rho, psi, rock, plo, phi, F[0], F[1]);
  else
    sc_force_ternary(P, x, y, z, i, psi, db, F[0], F[1], F[NC - 1]);
}

// ---------------------------------------------------------------------------
// Forces + BGK, code/lb3d_collision.F90:151-289.  With PULL (periodic
// lattices without stage-8 boundaries) g is the pre-stream state and each
// post-stream population is pulled from it as k_stream pulls it
// (code/lb3d_advection.F90:109-151, bounce-back from a rock upstream site,
// rock sites unmoved): the moments pass before (k_stream without STORE)
// wrote rho, psi and the momenta, and the post-stream populations never go
// to HBM.  The values are those k_stream would have stored, so f comes out
// the same bit for bit.  Occupancy (measured): the pulling variants run 2
// CTAs of 256 threads per SM, the binary one with rock 3 (faster despite
// its spills: 8.4 against 9.2 ms per step on a 256^3 porous lattice, where
// the ternary one at 3 ran 15 % slower), the staged binary ones 4.
// ---------------------------------------------------------------------------
template <int NC, bool LE, bool PULL = false, bool ROCK = true>
__global__ void __launch_bounds__(256, (PULL && ROCK && NC == 2) ? 3 : ((PULL || NC == 3) ? 2 : 4)) k_collide(DevParams P, const double *__restrict__ g,
                                                 double *__restrict__ f,
                                                 const double *__restrict__ rho,
                                                 const double *__restrict__ psi,
                                                 const double *__restrict__ mom,
                                                 const double *__restrict__ db,
                                                 const uint8_t *__restrict__ rock,
                                                 const double *__restrict__ plo,
                                                 const double *__restrict__ phi) {
  const long long N = P.nsites;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int x, y, z;
  site_xyz(i, P.nx, P.ny, x, y, z);
  double F[NC][3];
  sc_forces<NC, LE>(P, x, y, z, i, rho, psi, db, rock, plo, phi, F);
  double r[NC];
  for (int c = 0; c < NC; ++c) r[c] = rho[c * N + i];
  if (applyforce(P, x + 1, y + 1, z + 1)) {
    for (int c = 0; c < NC; ++c) {
      double mass = P.amass[c] * r[c];
      F[c][2] = F[c][2] + mass * P.g_accn;
      F[c][1] = F[c][1] + mass * P.g_accn_y;
      F[c][0] = F[c][0] + mass * P.g_accn_x;
    }
  }
  double pt[3];
  for (int k = 0; k < 3; ++k) pt[k] = (P.amass[0] * P.omega[0]) * mom[k * N + i];
  for (int c = 1; c < NC; ++c)
    for (int k = 0; k < 3; ++k) pt[k] = pt[k] + (P.amass[c] * P.omega[c]) * mom[(c * 3 + k) * N + i];
  double rho_tilde = (P.amass[0] * r[0]) * P.omega[0];
  for (int c = 1; c < NC; ++c) rho_tilde = rho_tilde + (P.amass[c] * r[c]) * P.omega[c];
  double rt = fmaxf_(rho_tilde, CLIP_RHO);
  double ut[3];
  for (int k = 0; k < 3; ++k) ut[k] = pt[k] / rt;
  auto bgk = [&](int c) {
    double pon = 1.0 / fmaxf_(r[c], CLIP_RHO);
    double du[3];
    for (int k = 0; k < 3; ++k) du[k] = ((P.tau[c] * pon) * F[c][k]) / P.amass[c];
    double b[19];
    boltz2(ut[0], ut[1], ut[2], du[0], du[1], du[2], b);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      double nq;
      if (q == REST || (ROCK && rock[i] != 0)) {
        nq = g[(c * 19 + q) * N + i];
      } else {
        const long long j =
            sidx(wrap(x - cx(q), P.nx), wrap(y - cy(q), P.ny), wrap(z - cz(q), P.nz), P.nx, P.ny);
        nq = (ROCK && rock[j] != 0) ? g[(c * 19 + bounce(q)) * N + i] : g[(c * 19 + q) * N + j];
      }
      double eq = r[c] * b[q];
      f[(c * 19 + q) * N + i] = nq - P.omega[c] * (nq - eq);
    }
  };
  // unrolled over the components where the pulls fill the loop (keeps r and
  // F in registers)
  if constexpr (PULL) {
#pragma unroll
    for (int c = 0; c < NC; ++c) bgk(c);
  } else {
    for (int c = 0; c < NC; ++c) {
      double pon = 1.0 / fmaxf_(r[c], CLIP_RHO);
      double du[3];
      for (int k = 0; k < 3; ++k) du[k] = ((P.tau[c] * pon) * F[c][k]) / P.amass[c];
      double b[19];
      boltz2(ut[0], ut[1], ut[2], du[0], du[1], du[2], b);
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        double nq = g[(c * 19 + q) * N + i];
        double eq = r[c] * b[q];
        f[(c * 19 + q) * N + i] = nq - P.omega[c] * (nq - eq);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Science dumps (code/lb3d_io_dump_data.F90:922-1460).  The XDR dump path
// gathers the lattice into a fresh arena with a plain periodic halo
// (code/lb3d_io.F90:387-442, code/lb3d_mpi.F90:783-859), so the dump-time
// forces always use the periodic neighbourhood.
// ---------------------------------------------------------------------------
template <int NC>
__global__ void k_dump(DevParams P, int field, const double *__restrict__ f,
                       const double *__restrict__ rho, const double *__restrict__ psi,
                       const double *__restrict__ db, const uint8_t *__restrict__ rock,
                       double *__restrict__ out) {
  const long long N = P.nsites;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int x, y, z;
  site_xyz(i, P.nx, P.ny, x, y, z);
  const bool fluid = rock[i] == 0;
  auto sumg = [&](int c, int dir) {
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      double cc = dir == 0 ? (double)cx(q) : dir == 1 ? (double)cy(q) : dir == 2 ? (double)cz(q) : 1.0;
      acc = acc + (f[(c * 19 + q) * N + i] * (double)gw(q)) * cc;
    }
    return acc;
  };
  switch (field) {
    case 0:  // od
      out[i] = fluid ? P.amass[0] * sumg(0, 3) : 0.0;
      break;
    case 1:  // wd
      out[i] = fluid ? P.amass[1] * sumg(1, 3) : 0.0;
      break;
    case 2:  // sur
      out[i] = (NC == 3) ? P.amass[NC - 1] * sumg(NC - 1, 3) : 0.0;
      break;
    case 3:  // dir
      for (int k = 0; k < 3; ++k) out[3 * i + k] = (NC == 3) ? db[k * N + i] : 0.0;
      break;
    case 4: {  // vel
      if (fluid) {
        double v = 0.0, den = 0.0;
        for (int c = 0; c < NC; ++c) {
          double term = (sumg(c, 2) * P.amass[c]) * P.omega[c];
          v = (c == 0) ? term : v + term;
          double dterm = (sumg(c, 3) * P.amass[c]) * P.omega[c];
          den = (c == 0) ? dterm : den + dterm;
        }
        v = v / fmaxf_(10.0e-9, den);
        if (in_accn_box(P, x + 1, y + 1, z + 1)) v = v - P.g_accn / 2.0;
        out[i] = v;
      } else {
        out[i] = 0.0;
      }
      break;
    }
    case 5: {  // arr
      double F[NC][3];
      sc_forces<NC, false>(P, x, y, z, i, rho, psi, db, rock, nullptr, nullptr, F);
      double den = 0.0;
      for (int c = 0; c < NC; ++c) {
        double t = sumg(c, 3) * P.amass[c];
        den = (c == 0) ? t : den + t;
      }
      float dd = (float)den;
      float denf = (1.0e-8f < dd) ? dd : 1.0e-8f;
      for (int k = 0; k < 3; ++k) {
        double v = 0.0;
        for (int c = 0; c < NC; ++c) {
          double m = sumg(c, k) * P.amass[c];
          double corr = ((F[c][k] / 2.0) * sumg(c, 3)) * P.amass[c];
          v = (c == 0) ? (m - corr) : ((v + m) - corr);
        }
        out[3 * i + k] = v / (double)denf;
      }
      if (in_accn_box(P, x + 1, y + 1, z + 1) && fluid) {
        out[3 * i + 0] = out[3 * i + 0] - P.g_accn_x / 2.0;
        out[3 * i + 1] = out[3 * i + 1] - P.g_accn_y / 2.0;
        out[3 * i + 2] = out[3 * i + 2] - P.g_accn / 2.0;
      }
      break;
    }
    case 6:  // rock
      out[i] = fluid ? 0.0 : 1.0;
      break;
  }
}

// Moments of the current state (used by downloads after a collision: the
// reference's rho/u fields then still hold the post-stream moments, which
// the stream kernel stored; this kernel is for states loaded by upload).
template <int NC>
__global__ void k_moments(DevParams P, const double *__restrict__ f, double *__restrict__ rho,
                          double *__restrict__ psi, double *__restrict__ mom) {
  const long long N = P.nsites;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int c = 0; c < NC; ++c) {
    double r = 0.0, u0 = 0.0, u1 = 0.0, u2 = 0.0;
#pragma unroll
    for (int q = 0; q < 19; ++q) r = r + f[(c * 19 + q) * N + i] * (double)gw(q);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      double ng = f[(c * 19 + q) * N + i] * (double)gw(q);
      u0 = u0 + ng * (double)cx(q);
      u1 = u1 + ng * (double)cy(q);
      u2 = u2 + ng * (double)cz(q);
    }
    rho[c * N + i] = r;
    psi[c * N + i] = get_psi(r);
    mom[(c * 3 + 0) * N + i] = u0;
    mom[(c * 3 + 1) * N + i] = u1;
    mom[(c * 3 + 2) * N + i] = u2;
  }
}

__global__ void k_detmath(int fn, const double *x, double *y, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = x[i];
  y[i] = fn == 0 ? det_exp(v) : fn == 1 ? lb3d_detmath::det_expm1(v) : det_tanh(v);
}

static inline unsigned grid_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace fp64

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
using namespace fp64;

cudaError_t fp64_le_halo(const DevParams &P, const LEStep &S, const double *src, double *hlo,
                         double *hhi, double *rlo, double *rhi, double *plo, double *phi,
                         cudaStream_t st) {
  int n = P.ny * P.nz;
  if (P.nc == 2)
    k_le_halo<2><<<grid_for(n, 128), 128, 0, st>>>(P, S, src, hlo, hhi, rlo, rhi, plo, phi);
  else
    k_le_halo<3><<<grid_for(n, 128), 128, 0, st>>>(P, S, src, hlo, hhi, rlo, rhi, plo, phi);
  return cudaGetLastError();
}

cudaError_t fp64_zouhe_flux(const DevParams &P, double *g, double *da, const double *db,
                            const uint8_t *rock, cudaStream_t st) {
  const int n = 2 * P.nx * P.ny;
  if (P.nc == 2)
    k_zouhe_flux<2><<<grid_for(n, 128), 128, 0, st>>>(P, g, da, db, rock);
  else
    k_zouhe_flux<3><<<grid_for(n, 128), 128, 0, st>>>(P, g, da, db, rock);
  return cudaGetLastError();
}

cudaError_t fp64_zouhe_density(const DevParams &P, double *g, const uint8_t *rock, double fr,
                               double fb, double pr, double pb, cudaStream_t st) {
  const int n = 2 * P.nx * P.ny;
  k_zouhe_density<<<grid_for(n, 128), 128, 0, st>>>(P, g, rock, fr, fb, pr, pb);
  return cudaGetLastError();
}

cudaError_t fp64_recolour(const DevParams &P, double *g, const uint8_t *rock, double mr, double mb,
                          cudaStream_t st) {
  const int n = P.nx * P.ny;
  k_recolour<<<grid_for(n, 128), 128, 0, st>>>(P, g, rock, mr, mb);
  return cudaGetLastError();
}

cudaError_t fp64_stream(const DevParams &P, const double *fin, double *fout, double *rho,
                        double *psi, double *mom, double *da, const double *db,
                        const uint8_t *rock, const double *hlo, const double *hhi,
                        cudaStream_t st) {
  unsigned gr = grid_for(P.nsites, 256);
#define LB3D_STREAM(NC_, LE_, FLUX_)                                                           \
  (P.any_rock ? k_stream<NC_, LE_, FLUX_, true><<<gr, 256, 0, st>>>(P, fin, fout, rho, psi, mom, da, \
                                                                    db, rock, hlo, hhi, c)        \
              : k_stream<NC_, LE_, FLUX_, false><<<gr, 256, 0, st>>>(P, fin, fout, rho, psi, mom, da, \
                                                                     db, rock, hlo, hhi, c))
  for (int c = 0; c < P.nc; ++c) {
    if (P.nc == 2) {
      if (P.le)
        LB3D_STREAM(2, true, false);
      else
        LB3D_STREAM(2, false, false);
    } else if (c < 2) {
      LB3D_STREAM(3, false, false);
    } else {
      LB3D_STREAM(3, false, true);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
#undef LB3D_STREAM
  return cudaSuccess;
}

cudaError_t fp64_step_pull(const DevParams &P, const double *fin, double *fout, double *rho,
                           double *psi, double *mom, double *da, double *db, const uint8_t *rock,
                           cudaStream_t st) {
  if (P.le || P.zouhe) return cudaErrorInvalidValue;
  unsigned gr = grid_for(P.nsites, 256);
  const bool rk = P.any_rock != 0;
  // moments pass: densities, psi and (surfactant) the advected dipole flux
  for (int c = 0; c < P.nc; ++c) {
#define LB3D_MOMENTS(NC_, FLUX_, ROCK_)                                                  \
  k_stream<NC_, false, FLUX_, ROCK_, false, true><<<gr, 256, 0, st>>>(P, fin, nullptr, rho, psi, \
                                                                      mom, da, db, rock, nullptr, \
                                                                      nullptr, c)
    if (P.nc == 2) {
      if (rk)
        LB3D_MOMENTS(2, false, true);
      else
        LB3D_MOMENTS(2, false, false);
    } else if (c < 2) {
      if (rk)
        LB3D_MOMENTS(3, false, true);
      else
        LB3D_MOMENTS(3, false, false);
    } else {
      if (rk)
        LB3D_MOMENTS(3, true, true);
      else
        LB3D_MOMENTS(3, true, false);
    }
#undef LB3D_MOMENTS
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (P.nc == 3) {
    k_dipole<<<grid_for(P.nsites, 256), 256, 0, st>>>(P, rho, da, db);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (P.nc == 2) {
    if (rk)
      k_collide<2, false, true, true><<<gr, 256, 0, st>>>(P, fin, fout, rho, psi, mom, db, rock, nullptr,
                                                           nullptr);
    else
      k_collide<2, false, true, false><<<gr, 256, 0, st>>>(P, fin, fout, rho, psi, mom, db, rock, nullptr,
                                                            nullptr);
  } else {
    if (rk)
      k_collide<3, false, true, true><<<gr, 256, 0, st>>>(P, fin, fout, rho, psi, mom, db, rock, nullptr,
                                                           nullptr);
    else
      k_collide<3, false, true, false><<<gr, 256, 0, st>>>(P, fin, fout, rho, psi, mom, db, rock, nullptr,
                                                            nullptr);
  }
  return cudaGetLastError();
}

cudaError_t fp64_dipole(const DevParams &P, const double *rho, const double *da, double *db,
                        cudaStream_t st) {
  k_dipole<<<grid_for(P.nsites, 256), 256, 0, st>>>(P, rho, da, db);
  return cudaGetLastError();
}

cudaError_t fp64_collide(const DevParams &P, const double *g, double *f, const double *rho,
                         const double *psi, const double *mom, const double *db,
                         const uint8_t *rock, const double *plo, const double *phi,
                         cudaStream_t st) {
  unsigned gr = grid_for(P.nsites, 256);
  if (P.nc == 2) {
    if (P.le)
      k_collide<2, true><<<gr, 256, 0, st>>>(P, g, f, rho, psi, mom, db, rock, plo, phi);
    else
      k_collide<2, false><<<gr, 256, 0, st>>>(P, g, f, rho, psi, mom, db, rock, plo, phi);
  } else {
    k_collide<3, false><<<gr, 256, 0, st>>>(P, g, f, rho, psi, mom, db, rock, plo, phi);
  }
  return cudaGetLastError();
}

cudaError_t fp64_dump(const DevParams &P, int field, const double *f, const double *rho,
                      const double *psi, const double *db, const uint8_t *rock, double *out,
                      cudaStream_t st) {
  unsigned gr = grid_for(P.nsites, 256);
  if (P.nc == 2)
    k_dump<2><<<gr, 256, 0, st>>>(P, field, f, rho, psi, db, rock, out);
  else
    k_dump<3><<<gr, 256, 0, st>>>(P, field, f, rho, psi, db, rock, out);
  return cudaGetLastError();
}

cudaError_t fp64_moments(const DevParams &P, const double *f, double *rho, double *psi,
                         double *mom, cudaStream_t st) {
  unsigned gr = grid_for(P.nsites, 256);
  if (P.nc == 2)
    k_moments<2><<<gr, 256, 0, st>>>(P, f, rho, psi, mom);
  else
    k_moments<3><<<gr, 256, 0, st>>>(P, f, rho, psi, mom);
  return cudaGetLastError();
}

cudaError_t fp64_detmath(int fn, const double *x, double *y, long long n, cudaStream_t st) {
  k_detmath<<<grid_for(n, 256), 256, 0, st>>>(fn, x, y, n);
  return cudaGetLastError();
}

}  // namespace lb3d
