// lb3d_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// FP64 CPU restatement of LB3D's per-timestep hot path.  Every routine
// cites the reference routine it restates; the operation order inside each
// expression follows the Fortran source (left-to-right evaluation, explicit
// parentheses kept).  Build with -O2 -ffp-contract=off (no FMA contraction,
// no reassociation); see oracle/Makefile.
//
// Data model: an array-of-structs arena with a one-site halo, the
// equivalent of whole_N(0:nx+1,0:ny+1,0:nz+1) of type lbe_site
// (code/lb3d_lattice.F90:35-83,274-287); site index x fastest as in
// Fortran's column-major N(x,y,z).
//
// Single-rank semantics: the MPI halo exchange becomes a periodic copy of
// the whole site (code/lb3d_mpi.F90:222-236 lbe_halo_exchange_local, the
// one-rank case of code/lb3d_bc_periodic.F90:36-56), and the Lees-Edwards
// exchange (code/lb3d_bc_leesedwards.F90:147-1315) is restated through the
// buffer mapping its one-rank send/receive pattern produces.

#include "lb3d_oracle.h"

// The deterministic exp/tanh of the product's FP64 path (a published
// method, see the header); selectable so that the oracle can be run with
// either glibc's libm or the same transcendental results as the device.
#include "../lb3d_b200/csrc/detmath.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// D3Q19 tables, code/lb3d_lattice.F90:137-187 (0-based here).
const int CX[19] = {1, -1, 0, 0, 0, 0, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0, 0};
const int CY[19] = {0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0};
const int CZ[19] = {0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, 0};
const int G[19] = {2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
const int BOUNCE[19] = {1, 0, 3, 2, 5, 4, 11, 10, 13, 12, 7, 6, 9, 8, 17, 16, 15, 14, 18};
const int NNONREST = 18;
const int REST = 18;

// Shan-Chen force weights g_sc, code/lb3d_force_shanchen.F90:148-152.
const int GSC[19] = {2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};

// The Fortran literals 10.e-5 and 10.e-9 are default-real (FP32) constants
// widened to FP64 (code/lb3d_collision.F90:345,546,586).
const double CLIP_RHO_S = (double)1.0e-4f;
const double CLIP_RHO = (double)1.0e-8f;

struct Site {
  double n[3][19];
  double rho[3];
  double u[3][3];  // momentum, not velocity (code/lb3d_analysis.F90:80-102)
  double rc[3];    // rock_colour_r, rock_colour_b, rock_colour_s
  double da[3];
  double db[3];
  double rock;
};

inline double fmax_f(double a, double b) { return (a < b) ? b : a; }  // Fortran max(a,b)

int g_detmath = 0;  // 0: glibc exp/tanh, 1: lb3d_detmath
inline double m_exp(double x) { return g_detmath ? lb3d_detmath::det_exp(x) : std::exp(x); }
inline double m_tanh(double x) { return g_detmath ? lb3d_detmath::det_tanh(x) : std::tanh(x); }

// psi(rho) = 1 - exp(-rho), code/lb3d_force_shanchen.F90:334-353 (psifunc 2).
inline double get_psi(double rho) { return 1.0 - m_exp(-rho); }

// boltz_dist, bdist = 2 (COMPAT_BDIST default), code/lb3d_bdist.F90:301-370.
void boltz_dist2(double ux, double uy, double uz, double dux, double duy, double duz,
                 double *boltz) {
  const double T = 1.0 / 3.0;
  const double holdit = 1.0 / T;
  const double w1 = 1.0 / 36.0;  // weight(1) = weight(7) = 1/36
  const double w0 = 1.0 / 3.0;   // weight(restvec)
  double tux = ux + dux, tuy = uy + duy, tuz = uz + duz;
  double tuxt = tux * holdit, tuyt = tuy * holdit, tuzt = tuz * holdit;
  double uke = 0.5 * (tux * tuxt + tuy * tuyt + tuz * tuzt);
  double cst = 1.0 - uke;
  double const1 = w1 * cst;
  double const2 = w1 * cst;
  double weight1by2 = w1 / 2.0, weight2by2 = w1 / 2.0;
  double weight1by6 = w1 / 6.0, weight2by6 = w1 / 6.0;
  auto pr = [&](double cdotu, double c, double wb2, double wb6, int i, int j) {
    double even = c + wb2 * (cdotu * cdotu);
    double odd = c * cdotu + wb6 * (cdotu * cdotu * cdotu);
    boltz[i] = even + odd;
    boltz[j] = even - odd;
  };
  pr(tuxt, const1, weight1by2, weight1by6, 0, 1);
  pr(tuyt, const1, weight1by2, weight1by6, 2, 3);
  pr(tuzt, const1, weight1by2, weight1by6, 4, 5);
  pr(tuxt + tuyt, const2, weight2by2, weight2by6, 6, 11);
  pr(tuxt - tuyt, const2, weight2by2, weight2by6, 7, 10);
  pr(tuxt + tuzt, const2, weight2by2, weight2by6, 8, 13);
  pr(tuxt - tuzt, const2, weight2by2, weight2by6, 9, 12);
  pr(tuyt + tuzt, const2, weight2by2, weight2by6, 14, 17);
  pr(tuyt - tuzt, const2, weight2by2, weight2by6, 15, 16);
  boltz[REST] = w0 * cst;
}

struct Oracle {
  lb3do_params p;
  int nx, ny, nz, nc;
  // y-slab of a decomposed lattice: its first plane's global y offset and
  // the exchange that fills the y-halo planes from the neighbouring slabs
  // (null: this lattice is periodic in y, as one rank is)
  int y_off = 0;
  lb3do_halo_fn yhook = nullptr;
  void *yctx = nullptr;
  double omega[3], omega_d, amass[3], tau[3];
  std::vector<Site> N, Nbuf;
  std::vector<double> F;  // forces [interior site][comp][3]
  int nt;
  bool le;
  double shear_u, shear_tmp, shear_sum, lefrac;
  int lelo;

  size_t idx(int x, int y, int z) const {
    return (size_t)x + (size_t)(nx + 2) * ((size_t)y + (size_t)(ny + 2) * (size_t)z);
  }
  size_t iidx(int x, int y, int z) const {  // interior, 1-based coordinates
    return (size_t)(x - 1) + (size_t)nx * ((size_t)(y - 1) + (size_t)ny * (size_t)(z - 1));
  }
  Site &at(int x, int y, int z) { return N[idx(x, y, z)]; }

  // ---- moments, code/lb3d_analysis.F90:64-102 -----------------------------
  void update_density(Site &s) {
    for (int c = 0; c < nc; ++c) {
      double acc = 0.0;
      for (int q = 0; q < 19; ++q) acc = acc + s.n[c][q] * (double)G[q];
      s.rho[c] = acc;
    }
  }
  void update_velocity(Site &s) {
    for (int c = 0; c < nc; ++c) {
      double u0 = 0.0, u1 = 0.0, u2 = 0.0;
      for (int q = 0; q < 19; ++q) {
        double ng = s.n[c][q] * (double)G[q];
        u0 = u0 + ng * (double)CX[q];
        u1 = u1 + ng * (double)CY[q];
        u2 = u2 + ng * (double)CZ[q];
      }
      s.u[c][0] = u0;
      s.u[c][1] = u1;
      s.u[c][2] = u2;
    }
  }
  // lb3d_update_density_loop / lb3d_update_velocity_loop, whole box incl. halo
  // (code/lb3d_analysis.F90:106-153).
  void update_loops() {
    for (size_t i = 0; i < N.size(); ++i) {
      update_density(N[i]);
      update_velocity(N[i]);
    }
  }

  // ---- periodic halo, code/lb3d_mpi.F90:222-236 ---------------------------
  void halo_periodic() {
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y) {
        at(0, y, z) = at(nx, y, z);
        at(nx + 1, y, z) = at(1, y, z);
      }
    if (yhook) {
      // the y neighbours are other ranks' slabs (code/lb3d_mpi.F90:492-596
      // exchanges the y faces after the x faces and before the z faces, so
      // the planes sent carry their x halo and the z faces copy the y halo)
      yhook(yctx, this);
    } else {
      for (int z = 1; z <= nz; ++z)
        for (int x = 0; x <= nx + 1; ++x) {
          at(x, 0, z) = at(x, ny, z);
          at(x, ny + 1, z) = at(x, 1, z);
        }
    }
    for (int y = 0; y <= ny + 1; ++y)
      for (int x = 0; x <= nx + 1; ++x) {
        at(x, y, 0) = at(x, y, nz);
        at(x, y, nz + 1) = at(x, y, 1);
      }
  }

  // ---- Lees-Edwards, code/lb3d_bc_leesedwards.F90 -------------------------
  // le_neighbours, :86-140 (one rank: only the offset bookkeeping matters).
  void le_neighbours() {
    if (p.inv_fluid == 6) {
      shear_u = 0.0;
      lelo = nz / 2 + 1;
      lefrac = 0.0;
    } else {
      shear_sum = shear_sum + shear_u;
      lelo = ((int)(2.0 * shear_sum)) % nz;  // mod(int(2.*shear_sum),nz)
      double s = 2.0 * shear_sum;
      lefrac = std::fabs(s - std::trunc(s));
    }
  }
  int wz(int z) const {  // wrap into 1..nz
    int r = (z - 1) % nz;
    if (r < 0) r += nz;
    return r + 1;
  }
  // Velocity adjustment of one x-halo site, :680-825 (bottom, sign=-1)
  // and :866-1002 (top, sign=+1).  For the top halo the clipping branch
  // reads the bottom-halo site N(0,y,z) (:951-986), which is reproduced.
  void le_adjust(Site &h, const Site &clipref, double sign) {
    double p[3][3] = {{0}}, ns[3] = {0, 0, 0};
    for (int q = 0; q < 19; ++q)
      for (int c = 0; c < nc; ++c) {
        ns[c] = ns[c] + h.n[c][q] * (double)G[q];
        double ng = h.n[c][q] * (double)G[q];
        p[c][0] = p[c][0] + ng * (double)CX[q];
        p[c][1] = p[c][1] + ng * (double)CY[q];
        p[c][2] = p[c][2] + ng * (double)CZ[q];
      }
    double pt[3], rho_tilde;
    for (int k = 0; k < 3; ++k) pt[k] = (amass[0] * omega[0]) * p[0][k];
    double rho_c = amass[0] * ns[0];
    rho_tilde = rho_c * omega[0];
    for (int c = 1; c < nc; ++c) {
      for (int k = 0; k < 3; ++k) pt[k] = pt[k] + (amass[c] * omega[c]) * p[c][k];
      rho_c = amass[c] * ns[c];
      rho_tilde = rho_tilde + rho_c * omega[c];
    }
    double rho_tmp = fmax_f(rho_tilde, CLIP_RHO);
    double ut[3];
    for (int k = 0; k < 3; ++k) ut[k] = pt[k] / rho_tmp;
    double b_udu[19], b_u[19], bdu[19];
    double uz2 = (sign < 0) ? ((ut[2] - shear_u) - shear_u) : ((ut[2] + shear_u) + shear_u);
    boltz_dist2(ut[0], ut[1], uz2, 0.0, 0.0, 0.0, b_udu);
    boltz_dist2(ut[0], ut[1], ut[2], 0.0, 0.0, 0.0, b_u);
    for (int q = 0; q < 19; ++q) bdu[q] = b_udu[q] - b_u[q];
    double df[3][19], fnew[3][19];
    bool neg = false;
    for (int c = 0; c < nc; ++c)
      for (int q = 0; q < 19; ++q) {
        df[c][q] = ns[c] * bdu[q];
        fnew[c][q] = h.n[c][q] + df[c][q];
        if (fnew[c][q] < 0.0) neg = true;
      }
    if (neg) {
      double mn = clipref.n[0][0];
      for (int c = 0; c < nc; ++c)
        for (int q = 0; q < 19; ++q) mn = std::min(mn, clipref.n[c][q]);
      double df_scale;
      if (mn > 0.0) {
        df_scale = -df[0][0] / clipref.n[0][0];
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) df_scale = fmax_f(df_scale, -df[c][q] / clipref.n[c][q]);
      } else {
        df_scale = 0.0;
      }
      if (std::fabs(df_scale) > 1.0) {
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) fnew[c][q] = clipref.n[c][q] + df[c][q] / df_scale;
      } else {
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) fnew[c][q] = clipref.n[c][q];
      }
    }
    for (int c = 0; c < nc; ++c)
      for (int q = 0; q < 19; ++q) h.n[c][q] = fnew[c][q];
  }

  // le_halo_exchange for one rank, :147-1315.  The one-rank receive
  // buffers map to pinbuf(k) = N(nx, wrap(k-1+e)) and
  // minbuf(k) = N(1, wrap(k-1-e-1)) with e = lelo (lelo >= 0) or lelo-1
  // (lelo < 0), from the chunk split at :252-269,442-489 and the
  // interpolation at :659-677,846-866.  Halo rows y in {0,ny+1} and
  // z in {0,nz+1} of the x-halo planes are then overwritten by the y and z
  // swaps (:1047-1308), so only the interior rows are computed here.
  void le_halo_exchange() {
    const double f = lefrac;
    const int e = (lelo >= 0) ? lelo : lelo - 1;
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y) {
        const Site &a = at(nx, y, wz(z + e));
        const Site &b = at(nx, y, wz(z + e + 1));
        Site &h = at(0, y, z);
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) h.n[c][q] = (1.0 - f) * a.n[c][q] + f * b.n[c][q];
        if (nc == 3)
          for (int k = 0; k < 3; ++k) {
            h.da[k] = (1.0 - f) * a.da[k] + f * b.da[k];
            h.db[k] = (1.0 - f) * a.db[k] + f * b.db[k];
          }
        h.rock = 0.0;
      }
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y) le_adjust(at(0, y, z), at(0, y, z), -1.0);
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y) {
        const Site &a = at(1, y, wz(z - e - 1));
        const Site &b = at(1, y, wz(z - e));
        Site &h = at(nx + 1, y, z);
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) h.n[c][q] = f * a.n[c][q] + (1.0 - f) * b.n[c][q];
        if (nc == 3)
          for (int k = 0; k < 3; ++k) {
            h.da[k] = f * a.da[k] + (1.0 - f) * b.da[k];
            h.db[k] = f * a.db[k] + (1.0 - f) * b.db[k];
          }
        h.rock = 0.0;
      }
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y) le_adjust(at(nx + 1, y, z), at(0, y, z), +1.0);
    // y and z swaps copy n, da, db and rock_state only (:1079-1172, :1216-1308)
    auto cp = [&](Site &d, const Site &s) {
      std::memcpy(d.n, s.n, sizeof(d.n));
      std::memcpy(d.da, s.da, sizeof(d.da));
      std::memcpy(d.db, s.db, sizeof(d.db));
      d.rock = s.rock;
    };
    for (int z = 1; z <= nz; ++z)
      for (int x = 0; x <= nx + 1; ++x) {
        cp(at(x, ny + 1, z), at(x, 1, z));
        cp(at(x, 0, z), at(x, ny, z));
      }
    for (int y = 0; y <= ny + 1; ++y)
      for (int x = 0; x <= nx + 1; ++x) {
        cp(at(x, y, nz + 1), at(x, y, 1));
        cp(at(x, y, 0), at(x, y, nz));
      }
  }

  void exchange() {
    if (le) {
      le_halo_exchange();
      update_loops();
    } else {
      halo_periodic();
    }
  }

  // ---- advection, code/lb3d_advection.F90:54-151 + bounce-back
  // code/lb3d_bc_bounce.F90:53-90.  Nbuf holds the pre-stream lattice, which
  // is what the rolling three-plane buffer of lb3d_advect provides.
  void advection() {
    Nbuf = N;
    const bool tern = (nc == 3);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) {
          Site &s = N[idx(x, y, z)];
          const Site &own = Nbuf[idx(x, y, z)];
          if (tern) s.da[0] = s.da[1] = s.da[2] = 0.0;
          // lb3d_bc_bounce_back_hw
          for (int q = 0; q < NNONREST; ++q) {
            int xa = x + CX[q], ya = y + CY[q], za = z + CZ[q];
            if (N[idx(xa, ya, za)].rock != 0.0) {
              if (own.rock == 0.0) {
                for (int c = 0; c < nc; ++c) s.n[c][BOUNCE[q]] = own.n[c][q];
                if (tern) {
                  const Site &nb = Nbuf[idx(xa, ya, za)];
                  for (int k = 0; k < 3; ++k)
                    s.da[k] = s.da[k] + (own.n[2][q] * (double)G[q]) * nb.db[k];
                }
              }
            }
          }
          // lb3d_advection_step
          for (int q = 0; q < NNONREST; ++q) {
            const Site &up = Nbuf[idx(x - CX[q], y - CY[q], z - CZ[q])];
            if (s.rock == 0.0) {
              if (up.rock == 0.0) {
                for (int c = 0; c < nc; ++c) s.n[c][q] = up.n[c][q];
                if (tern)
                  for (int k = 0; k < 3; ++k)
                    s.da[k] = s.da[k] + (up.n[2][q] * (double)G[q]) * up.db[k];
              }
            }
          }
          if (tern)
            for (int k = 0; k < 3; ++k)
              s.da[k] = s.da[k] + (own.n[2][REST] * (double)G[REST]) * own.db[k];
          update_density(s);
          update_velocity(s);
        }
  }

  // ---- lb3d_dipole_collision, code/lb3d_collision.F90:296-403 -------------
  void dipole_collision(int x, int y, int z) {
    Site &s = at(x, y, z);
    double h_c[3] = {0.0, 0.0, 0.0};
    double h_s[3] = {s.da[0], s.da[1], s.da[2]};
    double sN_tmp = fmax_f(s.rho[2], CLIP_RHO_S);
    double sd_tmp[3];
    for (int k = 0; k < 3; ++k) sd_tmp[k] = h_s[k] / sN_tmp;
    const double sgn = (p.g_bs >= 0.0) ? 1.0 : -1.0;  // sign(dble(1.0),g_bs)
    for (int q = 0; q < NNONREST; ++q) {
      const Site &nb = at(x + CX[q], y + CY[q], z + CZ[q]);
      double psi_r = 0.0 + nb.rho[0];
      double psi_b = 0.0 + nb.rho[1];
      double pas[3] = {nb.da[0], nb.da[1], nb.da[2]};
      double hc_m = -(sgn * (psi_b - psi_r) * (double)GSC[q]);
      const double c[3] = {(double)CX[q], (double)CY[q], (double)CZ[q]};
      for (int k = 0; k < 3; ++k) h_c[k] = h_c[k] + hc_m * c[k];
      double hs_dot = 2.0 * ((c[0] * pas[0] + c[1] * pas[1]) + c[2] * pas[2]);
      for (int k = 0; k < 3; ++k) h_s[k] = h_s[k] + (pas[k] - c[k] * hs_dot) * (double)GSC[q];
    }
    double h[3];
    for (int k = 0; k < 3; ++k) h[k] = h_c[k] + h_s[k];
    double h_m = p.beta * std::sqrt((h[0] * h[0] + h[1] * h[1]) + h[2] * h[2]);
    double sd_eq[3];
    const double third = 1.0 / 3.0;
    for (int k = 0; k < 3; ++k) sd_eq[k] = (third * p.beta) * h[k];
    if (h_m > 10.0e-3) {
      double exh = 1.0 / m_tanh(h_m);
      double sd_mag = exh - 1.0 / h_m;
      for (int k = 0; k < 3; ++k) sd_eq[k] = ((p.beta * h[k]) / h_m) * sd_mag;
    }
    for (int k = 0; k < 3; ++k) sd_eq[k] = sd_eq[k] * p.d_0;
    for (int k = 0; k < 3; ++k) s.db[k] = omega_d * sd_eq[k] + (1.0 - omega_d) * sd_tmp[k];
  }

  // ---- lb3d_calc_sc_force_binary, code/lb3d_force_shanchen.F90:127-210 ----
  void sc_force_binary(int x, int y, int z, double *fr, double *fb) {
    double f_br[3] = {0, 0, 0}, f_rb[3] = {0, 0, 0}, f_wr[3] = {0, 0, 0}, f_wb[3] = {0, 0, 0};
    for (int q = 0; q < NNONREST; ++q) {
      const Site &nb = at(x + CX[q], y + CY[q], z + CZ[q]);
      const double c[3] = {(double)CX[q], (double)CY[q], (double)CZ[q]};
      if (nb.rock != 0.0) {
        double psi_r = get_psi(nb.rho[0] + nb.rc[0]);
        double psi_b = get_psi(nb.rho[1] + nb.rc[1]);
        double green_r = psi_b * (double)GSC[q];
        double green_b = psi_r * (double)GSC[q];
        for (int k = 0; k < 3; ++k) {
          f_wb[k] = f_wb[k] + green_r * c[k];
          f_wr[k] = f_wr[k] + green_b * c[k];
        }
      } else {
        double psi_r = get_psi(nb.rho[0]);
        double psi_b = get_psi(nb.rho[1]);
        double green_r = psi_b * (double)GSC[q];
        double green_b = psi_r * (double)GSC[q];
        for (int k = 0; k < 3; ++k) {
          f_rb[k] = f_rb[k] + green_r * c[k];
          f_br[k] = f_br[k] + green_b * c[k];
        }
      }
    }
    const Site &s = at(x, y, z);
    double pb = get_psi(s.rho[1]), prr = get_psi(s.rho[0]);
    for (int k = 0; k < 3; ++k) {
      double br = -(p.g_br * f_br[k]);
      double rb = -(p.g_br * f_rb[k]);
      double wr = -(p.g_wr * f_wr[k]);
      double wb = -(p.g_wb * f_wb[k]);
      fb[k] = (br + ((wb / tau[1]) * p.tau_wb)) * pb;
      fr[k] = (rb + ((wr / tau[0]) * p.tau_wr)) * prr;
    }
  }

  // ---- lb3d_calc_sc_force_ternary, code/lb3d_force_shanchen.F90:215-330 ---
  void sc_force_ternary(int x, int y, int z, double *fr, double *fb, double *fs) {
    double f_br[3] = {0, 0, 0}, f_rb[3] = {0, 0, 0}, f_cs[3] = {0, 0, 0}, f_sc[3] = {0, 0, 0},
           f_ss[3] = {0, 0, 0};
    const Site &s = at(x, y, z);
    const double *dbx = s.db;
    for (int q = 0; q < NNONREST; ++q) {
      const Site &nb = at(x + CX[q], y + CY[q], z + CZ[q]);
      const double c[3] = {(double)CX[q], (double)CY[q], (double)CZ[q]};
      const double g = (double)GSC[q];
      double psi_r = get_psi(nb.rho[0]);
      double psi_b = get_psi(nb.rho[1]);
      double green_r = psi_b * g;
      double green_b = psi_r * g;
      for (int k = 0; k < 3; ++k) {
        f_rb[k] = f_rb[k] + green_r * c[k];
        f_br[k] = f_br[k] + green_b * c[k];
      }
      double pss = get_psi(nb.rho[2]);
      double da[3] = {nb.db[0] * pss, nb.db[1] * pss, nb.db[2] * pss};
      double d_dotc = (da[0] * c[0] + da[1] * c[1]) + da[2] * c[2];
      for (int k = 0; k < 3; ++k) f_cs[k] = f_cs[k] + (da[k] - (2.0 * d_dotc) * c[k]) * g;
      double di_dotc = (dbx[0] * c[0] + dbx[1] * c[1]) + dbx[2] * c[2];
      double greenc_s = (psi_b - psi_r) * g;
      for (int k = 0; k < 3; ++k) f_sc[k] = f_sc[k] + greenc_s * (dbx[k] - (2.0 * di_dotc) * c[k]);
      double di_dot_d = (da[0] * dbx[0] + da[1] * dbx[1]) + da[2] * dbx[2];
      double green_ss = 8.0 * g;  // 2.d0*D*g_sc(s) with D = 4
      for (int k = 0; k < 3; ++k)
        f_ss[k] = f_ss[k] + green_ss * (((di_dot_d - (2.0 * di_dotc) * d_dotc) * c[k] +
                                          da[k] * di_dotc) +
                                         d_dotc * dbx[k]);
    }
    double pb = get_psi(s.rho[1]), prr = get_psi(s.rho[0]), ps = get_psi(s.rho[2]);
    for (int k = 0; k < 3; ++k) {
      double br = -(p.g_br * f_br[k]);
      double rb = -(p.g_br * f_rb[k]);
      double sc = (2.0 * p.g_bs) * f_sc[k];
      double cs = -((2.0 * p.g_bs) * f_cs[k]);
      double ss = -(p.g_ss * f_ss[k]);
      fb[k] = (br + cs) * pb;
      fr[k] = (rb - cs) * prr;
      fs[k] = (sc + ss) * ps;
    }
  }

  void sc_forces(int x, int y, int z, double *f /*[comp][3]*/) {
    for (int i = 0; i < 9; ++i) f[i] = 0.0;
    if (at(x, y, z).rock == 0.0) {
      if (nc == 2)
        sc_force_binary(x, y, z, f + 0, f + 3);
      else
        sc_force_ternary(x, y, z, f + 0, f + 3, f + 6);
    }
  }

  // lb3d_get_applyforce, code/lb3d_collision.F90:431-460, in global
  // coordinates (a y-slab adds its offset).
  bool applyforce(int x, int y, int z) const {
    if (p.inv_fluid == 9) return (z == 1) || (z == nz);
    if (p.inv_fluid == 20 || p.inv_fluid == 21) return z == 1;
    const int gy = y + y_off;
    return (z >= p.g_accn_min) && (z <= p.g_accn_max) && (x >= p.g_accn_min_x) &&
           (x <= p.g_accn_max_x) && (gy >= p.g_accn_min_y) && (gy <= p.g_accn_max_y);
  }

  // ---- lb3d_collision_step, code/lb3d_collision.F90:59-291 ---------------
  void collision() {
    if (nc == 3) {
#pragma omp parallel for collapse(2) schedule(static)
      for (int z = 1; z <= nz; ++z)
        for (int y = 1; y <= ny; ++y)
          for (int x = 1; x <= nx; ++x) dipole_collision(x, y, z);
      exchange();
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) sc_forces(x, y, z, &F[9 * iidx(x, y, z)]);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) {
          Site &s = at(x, y, z);
          double *f = &F[9 * iidx(x, y, z)];
          // lb3d_get_body_force, :465-484 (FORCE_BODY)
          if (applyforce(x, y, z)) {
            for (int c = 0; c < nc; ++c) {
              double mass = amass[c] * s.rho[c];
              f[3 * c + 2] = f[3 * c + 2] + mass * p.g_accn;
              f[3 * c + 1] = f[3 * c + 1] + mass * p.g_accn_y;
              f[3 * c + 0] = f[3 * c + 0] + mass * p.g_accn_x;
            }
          }
          // lb3d_get_sc_u_eq, :560-587
          double pt[3], rho_tilde;
          for (int k = 0; k < 3; ++k) pt[k] = (amass[0] * omega[0]) * s.u[0][k];
          for (int c = 1; c < nc; ++c)
            for (int k = 0; k < 3; ++k) pt[k] = pt[k] + (amass[c] * omega[c]) * s.u[c][k];
          rho_tilde = (amass[0] * s.rho[0]) * omega[0];
          for (int c = 1; c < nc; ++c) rho_tilde = rho_tilde + (amass[c] * s.rho[c]) * omega[c];
          double ut[3];
          double rt = fmax_f(rho_tilde, CLIP_RHO);
          for (int k = 0; k < 3; ++k) ut[k] = pt[k] / rt;
          for (int c = 0; c < nc; ++c) {
            // lb3d_get_sc_du, :523-556
            double pon = 1.0 / fmax_f(s.rho[c], CLIP_RHO);
            double du[3];
            for (int k = 0; k < 3; ++k) du[k] = ((tau[c] * pon) * f[3 * c + k]) / amass[c];
            double boltz[19];
            boltz_dist2(ut[0], ut[1], ut[2], du[0], du[1], du[2], boltz);
            for (int q = 0; q < 19; ++q) {
              double eq = s.rho[c] * boltz[q];
              s.n[c][q] = s.n[c][q] - omega[c] * (s.n[c][q] - eq);
            }
          }
        }
  }

  // ---- Zou-He flux boundaries, code/lb3d_invasion.F90:2143-2457 ---------
  // lbe_invade_zouandheflux on one rank (both z planes are boundary
  // planes), applied to the post-stream populations at stage 8 before the
  // halo exchange.  Per fluid site of the plane and per component (the
  // surfactant first, then red, then blue): with F = n g, the unknown
  // populations entering the lattice are closed from the known ones and
  // the prescribed inflow uz (a velocity, or a flux divided by the density
  // for inv_type < 0), n = F / g; the surfactant's advected dipole flux is
  // then recomputed from its new populations.  Densities and velocities
  // keep their advection values (the reference recomputes them only for
  // Lees-Edwards).  F(i) below is the reference's 1-based direction i.
  void zouhe_flux_site(double *Fp, double uz, bool bottom, int itype) {
    auto F = [&](int i) -> double & { return Fp[i - 1]; };
    const double ux = 0., uy = 0.;
    double rho;
    if (bottom) {
      if (itype < 0) {
        rho = F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
              2. * (F(6) + F(10) + F(14) + F(16) + F(18)) + uz;
        if (rho > 0.)
          uz = uz / rho;
        else
          uz = 0.;
      } else {
        rho = (F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
               2. * (F(6) + F(10) + F(14) + F(16) + F(18))) /
              (1. - uz);
      }
      F(5) = F(6) + uz * rho / 3.;
      if (itype == 0) {
        F(15) = F(18) - (F(3) - F(4)) / 4. + rho * uz / 6.;
        F(17) = F(16) + (F(3) - F(4)) / 4. + rho * uz / 6.;
        F(9) = F(14) - (F(1) - F(2)) / 4. + rho * uz / 6.;
        F(13) = F(10) + (F(1) - F(2)) / 4. + rho * uz / 6.;
      } else if (itype == 1 || itype == -1) {
        F(15) = F(18) - (F(7) + F(11) + F(3) - F(8) - F(12) - F(4)) / 2. + uz * rho / 6. + uy * rho / 2.;
        F(17) = F(16) - (F(8) + F(12) + F(4) - F(7) - F(11) - F(3)) / 2. + uz * rho / 6. - uy * rho / 2.;
        F(9) = F(14) - (F(7) + F(8) + F(1) - F(11) - F(12) - F(2)) / 2. + uz * rho / 6. + ux * rho / 2.;
        F(13) = F(10) - (F(11) + F(12) + F(2) - F(7) - F(8) - F(1)) / 2. + uz * rho / 6. - ux * rho / 2.;
      }
    } else {
      if (itype < 0) {
        rho = F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
              2. * (F(5) + F(9) + F(13) + F(15) + F(17)) - uz;
        if (rho > 0.)
          uz = uz / rho;
        else
          uz = 0.;
      } else {
        rho = (F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
               2. * (F(5) + F(9) + F(13) + F(15) + F(17))) /
              (uz + 1.);
      }
      F(6) = F(5) - uz * rho / 3.;
      if (itype == 0) {
        F(18) = F(15) + (F(3) - F(4)) / 4. - rho * uz / 6.;
        F(16) = F(17) - (F(3) - F(4)) / 4. - rho * uz / 6.;
        F(14) = F(9) + (F(1) - F(2)) / 4. - rho * uz / 6.;
        F(10) = F(13) - (F(1) - F(2)) / 4. - rho * uz / 6.;
      } else if (itype == 1 || itype == -1) {
        F(18) = F(15) + (F(7) + F(11) + F(3) - F(8) - F(12) - F(4)) / 2. - uz * rho / 6. - uy * rho / 2.;
        F(16) = F(17) + (F(8) + F(12) + F(4) - F(7) - F(11) - F(3)) / 2. - uz * rho / 6. + uy * rho / 2.;
        F(14) = F(9) + (F(7) + F(8) + F(1) - F(11) - F(12) - F(2)) / 2. - uz * rho / 6. - ux * rho / 2.;
        F(10) = F(13) + (F(11) + F(12) + F(2) - F(7) - F(8) - F(1)) / 2. - uz * rho / 6. + ux * rho / 2.;
      }
    }
  }
  void invade_zouhe_flux() {
    // inflow per component: red pr, blue pb, surfactant pg
    const double uzc[3] = {p.pr, p.pb, p.pg};
    const int order[3] = {2, 0, 1};  // surfactant, red, blue
    for (int plane = 0; plane < 2; ++plane) {
      const int z = plane == 0 ? 1 : nz;
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) {
          Site &s = at(x, y, z);
          if (s.rock != 0.0) continue;
          for (int k = 0; k < 3; ++k) {
            const int c = order[k];
            if (c >= nc) continue;
            double F[19];
            for (int q = 0; q < 19; ++q) F[q] = s.n[c][q] * (double)G[q];
            zouhe_flux_site(F, uzc[c], plane == 0, p.inv_type);
            for (int q = 0; q < 19; ++q) s.n[c][q] = F[q] / (double)G[q];
            if (c == 2) {
              for (int a = 0; a < 3; ++a) s.da[a] = 0.0;
              for (int q = 0; q < 19; ++q) {
                const Site &b = at(x - CX[q], y - CY[q], z - CZ[q]);
                for (int a = 0; a < 3; ++a) s.da[a] = s.da[a] + s.n[2][q] * (double)G[q] * b.db[a];
              }
            }
          }
        }
    }
  }

  // Zou-He density boundaries, lbe_invade_zouandhe
  // (code/lb3d_invasion.F90:1459-1796), of the red and blue populations at
  // z = 1 (densities rho_in, :1510-1589) or z = nz (rho_out, :1690-1748),
  // with the Shan-Chen terms of the non-SINGLEFLUID build set to zero.  The
  // velocity closure the routine runs first writes only the five
  // populations that these density formulas then overwrite, and reads none
  // of them, so it leaves no trace in the result.  F(i) is the reference's
  // 1-based direction i; am13 is the mass in the rho/6/am term of F(13),
  // which the reference writes with amass_r for blue as well (:1567).
  void zouhe_density_site(double *Fp, double rho, double am, double am13, double tau, bool bottom) {
    auto F = [&](int i) -> double & { return Fp[i - 1]; };
    const double fx = 0.0, fy = 0.0;
    if (bottom) {
      F(5) = (-2.0 * F(10) - F(11) - F(12) - 2.0 * F(14) - 2.0 * F(16) - 2.0 * F(18) - F(19) - F(1) -
              F(2) - F(3) - F(4) + F(6) - F(7) - F(8)) / 3.0 + rho / 3.0 / am;
      F(9) = (-F(10) + F(11) + F(12) + 2.0 * F(14) - F(16) - F(18) - F(19) / 2.0 - 2.0 * F(1) + F(2) -
              F(3) / 2.0 - F(4) / 2.0 - F(6) - 2.0 * F(7) - 2.0 * F(8)) / 3.0 + rho / 6.0 / am -
             fx * tau / 4.0 / am;
      F(13) = (2.0 * F(10) - 2.0 * F(11) - 2.0 * F(12) - F(14) - F(16) - F(18) - F(19) / 2.0 + F(1) -
               2.0 * F(2) - F(3) / 2.0 - F(4) / 2.0 - F(6) + F(7) + F(8)) / 3.0 + rho / 6.0 / am13 +
              fx * tau / 4.0 / am;
      F(15) = (-F(10) - 2.0 * F(11) + F(12) - F(14) - F(16) + 2.0 * F(18) - F(19) / 2.0 - F(1) / 2.0 -
               F(2) / 2.0 - 2.0 * F(3) + F(4) - F(6) - 2.0 * F(7) + F(8)) / 3.0 + rho / 6.0 / am -
              fy * tau / 4.0 / am;
      F(17) = (-F(10) + F(11) - 2.0 * F(12) - F(14) + 2.0 * F(16) - F(18) - F(19) / 2.0 - F(1) / 2.0 -
               F(2) / 2.0 + F(3) - 2.0 * F(4) - F(6) + F(7) - 2.0 * F(8)) / 3.0 + rho / 6.0 / am +
              fy * tau / 4.0 / am;
    } else {
      F(6) = (-F(11) - F(12) - 2.0 * F(13) - 2.0 * F(15) - 2.0 * F(17) - F(19) - F(1) - F(2) - F(3) -
              F(4) + F(5) - F(7) - F(8) - 2.0 * F(9)) / 3.0 + rho / 3.0 / am;
      F(10) = (F(11) + F(12) + 2.0 * F(13) - F(15) - F(17) - F(19) / 2.0 - 2.0 * F(1) + F(2) -
               F(3) / 2.0 - F(4) / 2.0 - F(5) - 2.0 * F(7) - 2.0 * F(8) - F(9)) / 3.0 + rho / 6.0 / am -
              fx * tau / 4.0 / am;
      F(14) = (-2.0 * F(11) - 2.0 * F(12) - F(13) - F(15) - F(17) - F(19) / 2.0 + F(1) - 2.0 * F(2) -
               F(3) / 2.0 - F(4) / 2.0 - F(5) + F(7) + F(8) + 2.0 * F(9)) / 3.0 + rho / 6.0 / am +
              fx * tau / 4.0 / am;
      F(16) = (-2.0 * F(11) + F(12) - F(13) - F(15) + 2.0 * F(17) - F(19) / 2.0 - F(1) / 2.0 -
               F(2) / 2.0 - 2.0 * F(3) + F(4) - F(5) - 2.0 * F(7) + F(8) - F(9)) / 3.0 + rho / 6.0 / am -
              fy * tau / 4.0 / am;
      F(18) = (F(11) - 2.0 * F(12) - F(13) + 2.0 * F(15) - F(17) - F(19) / 2.0 - F(1) / 2.0 -
               F(2) / 2.0 + F(3) - 2.0 * F(4) - F(5) + F(7) - 2.0 * F(8) - F(9)) / 3.0 + rho / 6.0 / am +
              fy * tau / 4.0 / am;
    }
  }
  void invade_zouhe_density() {
    for (int plane = 0; plane < 2; ++plane) {
      const bool bottom = plane == 0;
      const int z = bottom ? 1 : nz;
      const double rho_c[2] = {bottom ? p.fr : p.pr, bottom ? p.fb : p.pb};
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) {
          Site &s = at(x, y, z);
          if (s.rock != 0.0) continue;
          for (int c = 0; c < 2; ++c) {
            double F[19];
            for (int q = 0; q < 19; ++q) F[q] = s.n[c][q] * (double)G[q];
            zouhe_density_site(F, rho_c[c], amass[c], bottom ? amass[0] : amass[c], tau[c], bottom);
            for (int q = 0; q < 19; ++q) s.n[c][q] = F[q] / (double)G[q];
          }
        }
    }
  }

  // lbe_invade_binary (code/lb3d_invasion.F90:1257-1358), binary builds
  // (inv_fluid 7: mr = 1, mb = 0; 8: mr = 0, mb = 1): the two bottom planes
  // z = 1, 2 are recoloured to red = mr * (n_r + n_b), blue = mb * (n_r + n_b)
  // per population, then the two top planes z = nz - 1, nz the other way
  // round, skipping rock sites.
  void invade_recolour(double mr, double mb) {
    const int zs[4] = {1, 2, nz - 1, nz};
    for (int k = 0; k < 4; ++k) {
      const double a = k < 2 ? mr : mb, b = k < 2 ? mb : mr;
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) {
          Site &s = at(x, y, zs[k]);
          if (s.rock != 0.0) continue;
          for (int q = 0; q < 19; ++q) {
            const double pop = s.n[0][q] + s.n[1][q];
            s.n[0][q] = a * pop;
            s.n[1][q] = b * pop;
          }
        }
    }
  }

  void bc_apply(int stage) {
    if (stage == 6) {
      if (le) {
        shear_u = shear_tmp * std::cos(p.shear_omega * (double)nt);
        le_neighbours();
        le_halo_exchange();
        update_loops();
      } else {
        halo_periodic();
      }
    } else if (stage == 8) {
      // code/lb3d_bc.F90:125-133: invasion first, then the halo exchange
      if (p.boundary_cond != 0 && p.inv_fluid == 12) invade_zouhe_flux();
      if (p.boundary_cond != 0 && p.inv_fluid == 11) invade_zouhe_density();
      if (p.boundary_cond != 0 && p.inv_fluid == 7) invade_recolour(1.0, 0.0);
      if (p.boundary_cond != 0 && p.inv_fluid == 8) invade_recolour(0.0, 1.0);
      exchange();
    }
  }

  void step() {
    nt += 1;
    bc_apply(6);
    advection();
    bc_apply(8);
    collision();
  }
};

}  // namespace

static int g_threads = 0;

extern "C" {

void lb3do_set_math(int det) { g_detmath = det ? 1 : 0; }

void lb3do_set_threads(int n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}

void *lb3do_create(const lb3do_params *p) {
  if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1) return nullptr;
  if (p->ncomp != 2 && p->ncomp != 3) return nullptr;
  if (p->bdist != 2) return nullptr;
  bool le = (p->boundary_cond != 0) && (p->inv_fluid == 5 || p->inv_fluid == 6);
  // code/lb3d_compatibility.F90:105-111: ternary + Lees-Edwards is fatal.
  if (p->ncomp == 3 && le) return nullptr;
  // Invasion boundaries other than the Lees-Edwards no-ops, the Zou-He flux
  // and density boundaries and the binary recolouring are outside this restatement
  // (code/lb3d_bc.F90:129-133).  Recolouring exists in binary builds only
  // (code/lb3d_invasion.F90:80-85) and needs two planes.
  const bool recolour = p->boundary_cond != 0 && (p->inv_fluid == 7 || p->inv_fluid == 8);
  if (recolour && (p->ncomp != 2 || p->nz < 2)) return nullptr;
  const bool zouhe = p->boundary_cond != 0 && (p->inv_fluid == 11 || p->inv_fluid == 12);
  if (zouhe && p->nz < 2) return nullptr;
  if (p->boundary_cond != 0 && p->inv_fluid >= 0 && !le && !zouhe && !recolour) return nullptr;
  Oracle *o = new Oracle();
  o->p = *p;
  o->nx = p->nx;
  o->ny = p->ny;
  o->nz = p->nz;
  o->nc = p->ncomp;
  o->tau[0] = p->tau_r;
  o->tau[1] = p->tau_b;
  o->tau[2] = p->tau_s;
  o->amass[0] = p->amass_r;
  o->amass[1] = p->amass_b;
  o->amass[2] = p->amass_s;
  for (int c = 0; c < 3; ++c) o->omega[c] = 1.0 / o->tau[c];  // code/lb3d_config.F90:886-889
  o->omega_d = 1.0 / p->tau_d;
  o->le = le;
  o->N.assign((size_t)(p->nx + 2) * (p->ny + 2) * (p->nz + 2), Site());
  std::memset(o->N.data(), 0, o->N.size() * sizeof(Site));
  o->F.assign((size_t)9 * p->nx * p->ny * p->nz, 0.0);
  o->nt = 0;
  o->shear_u = p->shear_u;
  o->shear_tmp = 0.0;
  o->shear_sum = 0.0;
  o->lelo = 0;
  o->lefrac = 0.0;
  return o;
}

void lb3do_destroy(void *h) { delete static_cast<Oracle *>(h); }

int lb3do_load(void *h, const double *n, const double *db, const double *rock, double shear_sum,
               int nt0) {
  Oracle *o = static_cast<Oracle *>(h);
  const int nx = o->nx, ny = o->ny, nz = o->nz, nc = o->nc;
  const size_t ns = (size_t)nx * ny * nz;
  for (int z = 1; z <= nz; ++z)
    for (int y = 1; y <= ny; ++y)
      for (int x = 1; x <= nx; ++x) {
        size_t i = o->iidx(x, y, z);
        Site &s = o->at(x, y, z);
        for (int c = 0; c < nc; ++c)
          for (int q = 0; q < 19; ++q) s.n[c][q] = n[((size_t)c * 19 + q) * ns + i];
        for (int k = 0; k < 3; ++k) {
          s.db[k] = (db && nc == 3) ? db[k * ns + i] : 0.0;
          s.da[k] = s.db[k];
        }
        s.rock = rock ? (rock[i] != 0.0 ? 1.0 : 0.0) : 0.0;
      }
  // lbe_init_rock_colour, code/lb3d_ic_rock.F90:146-189; rock_colour ->
  // rock_colour_r/_b as in code/lb3d_config.F90:661-664 (done by the caller).
  for (int z = 1; z <= nz; ++z)
    for (int y = 1; y <= ny; ++y)
      for (int x = 1; x <= nx; ++x) {
        Site &s = o->at(x, y, z);
        if (s.rock != 0.0) {
          for (int c = 0; c < nc; ++c)
            for (int q = 0; q < 19; ++q) s.n[c][q] = 0.0;
          if (nc == 3)
            for (int k = 0; k < 3; ++k) s.da[k] = s.db[k] = 0.0;
          if (o->p.rock_colour_r > 0) s.rc[0] = o->p.rock_colour_r;
          if (o->p.rock_colour_b > 0) s.rc[1] = o->p.rock_colour_b;
        }
      }
  o->nt = nt0;
  o->shear_sum = shear_sum;
  // lb3d_bc_init(4), code/lb3d_bc.F90:48-90
  if (o->le) {
    o->shear_u = ((double)nx / ((double)nx - 1.0)) * o->p.shear_u;
    o->shear_tmp = o->shear_u;
    if (o->p.restore) o->shear_sum = o->shear_sum - o->shear_u;
    o->le_neighbours();
    o->le_halo_exchange();
    o->update_loops();
  } else {
    o->halo_periodic();
  }
  return 0;
}

int lb3do_stage(void *h, int stage) {
  Oracle *o = static_cast<Oracle *>(h);
  switch (stage) {
    case 6:
      o->nt += 1;
      o->bc_apply(6);
      return 0;
    case 7:
      o->advection();
      return 0;
    case 8:
      o->bc_apply(8);
      return 0;
    case 9:
      o->collision();
      return 0;
    default:
      return -1;
  }
}

int lb3do_set_slab(void *h, int y_off, lb3do_halo_fn fn, void *ctx) {
  Oracle *o = static_cast<Oracle *>(h);
  if (o->le || y_off < 0) return -1;  // Lees-Edwards lattices are one slab
  o->y_off = y_off;
  o->yhook = fn;
  o->yctx = ctx;
  return 0;
}

long long lb3do_yplane_doubles(const void *h) {
  const Oracle *o = static_cast<const Oracle *>(h);
  return (long long)(o->nx + 2) * o->nz * (long long)(sizeof(Site) / sizeof(double));
}

int lb3do_yplane(void *h, int y, double *buf, int put) {
  Oracle *o = static_cast<Oracle *>(h);
  if (y < 0 || y > o->ny + 1) return -1;
  static_assert(sizeof(Site) % sizeof(double) == 0, "Site is a block of doubles");
  const size_t sd = sizeof(Site) / sizeof(double);
  for (int z = 1; z <= o->nz; ++z)
    for (int x = 0; x <= o->nx + 1; ++x) {
      double *b = buf + ((size_t)(z - 1) * (o->nx + 2) + x) * sd;
      Site &s = o->at(x, y, z);
      if (put)
        std::memcpy(&s, b, sizeof(Site));
      else
        std::memcpy(b, &s, sizeof(Site));
    }
  return 0;
}

int lb3do_run(void *h, int nsteps) {
  Oracle *o = static_cast<Oracle *>(h);
  for (int i = 0; i < nsteps; ++i) o->step();
  return 0;
}

int lb3do_get(const void *h, double *n, double *db, double *rho, double *mom, double *da) {
  const Oracle *o = static_cast<const Oracle *>(h);
  const int nx = o->nx, ny = o->ny, nz = o->nz, nc = o->nc;
  const size_t ns = (size_t)nx * ny * nz;
  for (int z = 1; z <= nz; ++z)
    for (int y = 1; y <= ny; ++y)
      for (int x = 1; x <= nx; ++x) {
        size_t i = o->iidx(x, y, z);
        const Site &s = o->N[o->idx(x, y, z)];
        for (int c = 0; c < nc; ++c) {
          if (n)
            for (int q = 0; q < 19; ++q) n[((size_t)c * 19 + q) * ns + i] = s.n[c][q];
          if (rho) rho[c * ns + i] = s.rho[c];
          if (mom)
            for (int k = 0; k < 3; ++k) mom[((size_t)c * 3 + k) * ns + i] = s.u[c][k];
        }
        for (int k = 0; k < 3; ++k) {
          if (db) db[k * ns + i] = s.db[k];
          if (da) da[k * ns + i] = s.da[k];
        }
      }
  return 0;
}

int lb3do_dump(void *hh, const char *field, double *out) {
  Oracle *o = static_cast<Oracle *>(hh);
  const int nx = o->nx, ny = o->ny, nz = o->nz, nc = o->nc;
  auto sumg = [&](const Site &s, int c, const int *cc) {
    double acc = 0.0;
    for (int q = 0; q < 19; ++q)
      acc = acc + (s.n[c][q] * (double)G[q]) * (cc ? (double)cc[q] : 1.0);
    return acc;
  };
  std::string f(field);
  // With post = .true. and an XDR dump format the reference gathers the
  // interior into a fresh arena Nm and fills its halo with a plain periodic
  // copy before dumping (postprocess, code/lb3d_io.F90:387-442, and
  // recv_final_lattice, code/lb3d_mpi.F90:783-859).  The dump-time
  // Shan-Chen forces therefore see periodic halos, also under Lees-Edwards.
  std::vector<Site> saved;
  if (o->le) {
    saved = o->N;
    o->halo_periodic();
  }
  struct Restore {
    Oracle *o;
    std::vector<Site> *s;
    ~Restore() {
      if (!s->empty()) o->N.swap(*s);
    }
  } restore_guard{o, &saved};
  for (int z = 1; z <= nz; ++z)
    for (int y = 1; y <= ny; ++y)
      for (int x = 1; x <= nx; ++x) {
        size_t i = o->iidx(x, y, z);
        const Site &s = o->at(x, y, z);
        if (f == "od") {  // code/lb3d_io_dump_data.F90:1100-1130
          out[i] = (s.rock == 0.0) ? o->amass[0] * sumg(s, 0, nullptr) : 0.0;
        } else if (f == "wd") {  // :1136-1166
          out[i] = (s.rock == 0.0) ? o->amass[1] * sumg(s, 1, nullptr) : 0.0;
        } else if (f == "sur") {  // :922-948
          out[i] = (nc == 3) ? o->amass[2] * sumg(s, 2, nullptr) : 0.0;
        } else if (f == "dir") {  // :955-980
          for (int k = 0; k < 3; ++k) out[3 * i + k] = s.db[k];
        } else if (f == "rock") {
          out[i] = s.rock;
        } else if (f == "vel") {  // :986-1096
          if (s.rock == 0.0) {
            double v = 0.0, den = 0.0;
            for (int c = 0; c < nc; ++c) {
              double term = (sumg(s, c, CZ) * o->amass[c]) * o->omega[c];
              v = (c == 0) ? term : v + term;
              double dterm = (sumg(s, c, nullptr) * o->amass[c]) * o->omega[c];
              den = (c == 0) ? dterm : den + dterm;
            }
            v = v / fmax_f(10.0e-9, den);
            if ((z >= o->p.g_accn_min) && (z <= o->p.g_accn_max) && (x >= o->p.g_accn_min_x) &&
                (x <= o->p.g_accn_max_x) && (y + o->y_off >= o->p.g_accn_min_y) &&
                (y + o->y_off <= o->p.g_accn_max_y))
              v = v - o->p.g_accn / 2.0;
            out[i] = v;
          } else {
            out[i] = 0.0;
          }
        } else if (f == "arr") {  // :1308-1460
          double fsc[9];
          o->sc_forces(x, y, z, fsc);
          const int *cv[3] = {CX, CY, CZ};
          double den = 0.0;
          for (int c = 0; c < nc; ++c) {
            double t = sumg(s, c, nullptr) * o->amass[c];
            den = (c == 0) ? t : den + t;
          }
          // max(10.e-9, real(...)): both FP32, the quotient in FP64.
          float denf = std::max(1.0e-8f, (float)den);
          for (int k = 0; k < 3; ++k) {
            double v = 0.0;
            for (int c = 0; c < nc; ++c) {
              double mom = sumg(s, c, cv[k]) * o->amass[c];
              double corr = ((fsc[3 * c + k] / 2.0) * sumg(s, c, nullptr)) * o->amass[c];
              v = (c == 0) ? (mom - corr) : ((v + mom) - corr);
            }
            out[3 * i + k] = v / (double)denf;
          }
          if ((z >= o->p.g_accn_min) && (z <= o->p.g_accn_max) && (x >= o->p.g_accn_min_x) &&
              (x <= o->p.g_accn_max_x) && (y + o->y_off >= o->p.g_accn_min_y) &&
                (y + o->y_off <= o->p.g_accn_max_y)) {
            if (s.rock == 0.0) {
              out[3 * i + 0] = out[3 * i + 0] - o->p.g_accn_x / 2.0;
              out[3 * i + 1] = out[3 * i + 1] - o->p.g_accn_y / 2.0;
              out[3 * i + 2] = out[3 * i + 2] - o->p.g_accn / 2.0;
            }
          }
        } else {
          return -1;
        }
      }
  return 0;
}

int lb3do_sums(const void *h, double mass[3], double mom[3]) {
  const Oracle *o = static_cast<const Oracle *>(h);
  for (int k = 0; k < 3; ++k) mass[k] = mom[k] = 0.0;
  for (int z = 1; z <= o->nz; ++z)
    for (int y = 1; y <= o->ny; ++y)
      for (int x = 1; x <= o->nx; ++x) {
        const Site &s = o->N[o->idx(x, y, z)];
        if (s.rock != 0.0) continue;
        for (int c = 0; c < o->nc; ++c) {
          double r = 0.0, m[3] = {0, 0, 0};
          for (int q = 0; q < 19; ++q) {
            double ng = s.n[c][q] * (double)G[q];
            r += ng;
            m[0] += ng * CX[q];
            m[1] += ng * CY[q];
            m[2] += ng * CZ[q];
          }
          mass[c] += r;
          for (int k = 0; k < 3; ++k) mom[k] += m[k];
        }
      }
  return 0;
}

// lbe_sanity_check's velocity statistics, code/lb3d_sanity.F90:130-229: the
// reference's x-outer, z-inner loop over fluid sites; per species with
// |rho| > 1e-12 the velocity sum(n g c) amass / rho, the running maximum of
// each |v_k| taken with `>=` (ties move to the later site), the sum of v_k,
// and the sites where some species has norm(v) > 0.1.
int lb3do_sanity_velocity(const void *h, double maxvel[9], int maxpos[27], double velsum[9],
                          long long *n_fluid, long long *n_too_fast) {
  const Oracle *o = static_cast<const Oracle *>(h);
  const double small = 1.0e-12, max_vel = 0.1;
  for (int k = 0; k < 9; ++k) {
    maxvel[k] = 0.0;
    velsum[k] = 0.0;
    for (int a = 0; a < 3; ++a) maxpos[3 * k + a] = 0;
  }
  long long fs = 0, tf = 0;
  for (int x = 1; x <= o->nx; ++x)
    for (int y = 1; y <= o->ny; ++y)
      for (int z = 1; z <= o->nz; ++z) {
        const Site &s = o->N[o->idx(x, y, z)];
        if (s.rock != 0.0) continue;
        ++fs;
        bool fast = false;
        for (int c = 0; c < o->nc; ++c) {
          double r = 0.0, m[3] = {0, 0, 0};
          for (int q = 0; q < 19; ++q) {
            const double ng = s.n[c][q] * (double)G[q];
            r = r + ng;
            m[0] = m[0] + ng * CX[q];
            m[1] = m[1] + ng * CY[q];
            m[2] = m[2] + ng * CZ[q];
          }
          if (std::fabs(r) > small) {
            double v[3];
            for (int k = 0; k < 3; ++k) v[k] = m[k] * o->amass[c] / r;
            for (int k = 0; k < 3; ++k) {
              velsum[3 * c + k] = velsum[3 * c + k] + v[k];
              if (std::fabs(v[k]) >= maxvel[3 * c + k]) {
                maxvel[3 * c + k] = std::fabs(v[k]);
                maxpos[9 * c + 3 * k] = x;
                maxpos[9 * c + 3 * k + 1] = y;
                maxpos[9 * c + 3 * k + 2] = z;
              }
            }
            if (std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) > max_vel) fast = true;
          }
        }
        if (fast) ++tf;
      }
  if (n_fluid) *n_fluid = fs;
  if (n_too_fast) *n_too_fast = tf;
  return 0;
}

double lb3do_shear_sum(const void *h) { return static_cast<const Oracle *>(h)->shear_sum; }
int lb3do_nt(const void *h) { return static_cast<const Oracle *>(h)->nt; }

}  // extern "C"
