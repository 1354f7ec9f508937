// le_common.cuh -- FP64 pieces shared by the FP64 and FP32 paths: the
// bdist = 2 equilibrium and the Lees-Edwards halo adjustment
// (code/lb3d_bc_leesedwards.F90:147-1315, one rank), compiled without FMA
// contraction by every file that includes it.
#pragma once

#include "common.cuh"

namespace lb3d {

// Fortran max(a,b) for the clipping constants.
__device__ __forceinline__ double fmaxf_(double a, double b) { return (a < b) ? b : a; }

// The FP32 literals 10.e-5 and 10.e-9 widened to FP64
// (code/lb3d_collision.F90:345,546,586).
#define CLIP_RHO_S ((double)1.0e-4f)
#define CLIP_RHO ((double)1.0e-8f)

// boltz_dist, bdist = 2, code/lb3d_bdist.F90:301-370.
__device__ __forceinline__ void boltz2(double ux, double uy, double uz, double dux, double duy,
                                       double duz, double *b) {
  const double T = 1.0 / 3.0;
  const double holdit = 1.0 / T;
  const double w1 = 1.0 / 36.0;
  const double w0 = 1.0 / 3.0;
  double tux = ux + dux, tuy = uy + duy, tuz = uz + duz;
  double tuxt = tux * holdit, tuyt = tuy * holdit, tuzt = tuz * holdit;
  double uke = 0.5 * (tux * tuxt + tuy * tuyt + tuz * tuzt);
  double cst = 1.0 - uke;
  double c1 = w1 * cst;
  double wb2 = w1 / 2.0, wb6 = w1 / 6.0;
#define LB3D_PAIR(CD, I, J)                                 \
  {                                                         \
    double cdotu = (CD);                                    \
    double even = c1 + wb2 * (cdotu * cdotu);               \
    double odd = c1 * cdotu + wb6 * (cdotu * cdotu * cdotu); \
    b[I] = even + odd;                                      \
    b[J] = even - odd;                                      \
  }
  LB3D_PAIR(tuxt, 0, 1)
  LB3D_PAIR(tuyt, 2, 3)
  LB3D_PAIR(tuzt, 4, 5)
  LB3D_PAIR(tuxt + tuyt, 6, 11)
  LB3D_PAIR(tuxt - tuyt, 7, 10)
  LB3D_PAIR(tuxt + tuzt, 8, 13)
  LB3D_PAIR(tuxt - tuzt, 9, 12)
  LB3D_PAIR(tuyt + tuzt, 14, 17)
  LB3D_PAIR(tuyt - tuzt, 15, 16)
#undef LB3D_PAIR
  b[REST] = w0 * cst;
}

// ---------------------------------------------------------------------------
// Lees-Edwards x-halo (code/lb3d_bc_leesedwards.F90:147-1315, one rank).
// One thread per (y,z) builds both halo sites, the bottom one first: the
// clipping branch of the top halo reads the adjusted bottom site
// (:951-986).
// ---------------------------------------------------------------------------
// The first half of the adjustment: the equilibrium shift df of the halo
// site h; returns whether h + df would go negative somewhere, the case in
// which the clipping rule reads the reference site.
template <int NC>
__device__ bool le_adjust_df(const DevParams &P, const double h[NC][19], double shear_u, double sign,
                             double df[NC][19]) {
  double p[NC][3], ns[NC];
  for (int c = 0; c < NC; ++c) {
    ns[c] = 0.0;
    p[c][0] = p[c][1] = p[c][2] = 0.0;
  }
#pragma unroll
  for (int q = 0; q < 19; ++q)
    for (int c = 0; c < NC; ++c) {
      ns[c] = ns[c] + h[c][q] * (double)gw(q);
      double ng = h[c][q] * (double)gw(q);
      p[c][0] = p[c][0] + ng * (double)cx(q);
      p[c][1] = p[c][1] + ng * (double)cy(q);
      p[c][2] = p[c][2] + ng * (double)cz(q);
    }
  double pt[3];
  for (int k = 0; k < 3; ++k) pt[k] = (P.amass[0] * P.omega[0]) * p[0][k];
  double rho_c = P.amass[0] * ns[0];
  double rho_tilde = rho_c * P.omega[0];
  for (int c = 1; c < NC; ++c) {
    for (int k = 0; k < 3; ++k) pt[k] = pt[k] + (P.amass[c] * P.omega[c]) * p[c][k];
    rho_c = P.amass[c] * ns[c];
    rho_tilde = rho_tilde + rho_c * P.omega[c];
  }
  double rho_tmp = fmaxf_(rho_tilde, CLIP_RHO);
  double ut[3];
  for (int k = 0; k < 3; ++k) ut[k] = pt[k] / rho_tmp;
  double b_udu[19], b_u[19];
  double uz2 = (sign < 0.0) ? ((ut[2] - shear_u) - shear_u) : ((ut[2] + shear_u) + shear_u);
  boltz2(ut[0], ut[1], uz2, 0.0, 0.0, 0.0, b_udu);
  boltz2(ut[0], ut[1], ut[2], 0.0, 0.0, 0.0, b_u);
  bool neg = false;
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      df[c][q] = ns[c] * (b_udu[q] - b_u[q]);
      if (h[c][q] + df[c][q] < 0.0) neg = true;
    }
  return neg;
}

// The second half: h + df, or, when that goes negative, the reference site
// plus df scaled to keep it non-negative (ref is read only then).
template <int NC>
__device__ void le_adjust_apply(double h[NC][19], const double ref[NC][19], const double df[NC][19],
                                bool neg) {
  if (neg) {
    double mn = ref[0][0];
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q) mn = fmin(mn, ref[c][q]);
    double df_scale;
    if (mn > 0.0) {
      df_scale = -df[0][0] / ref[0][0];
      for (int c = 0; c < NC; ++c)
        for (int q = 0; q < 19; ++q) df_scale = fmaxf_(df_scale, -df[c][q] / ref[c][q]);
    } else {
      df_scale = 0.0;
    }
    if (fabs(df_scale) > 1.0) {
      for (int c = 0; c < NC; ++c)
        for (int q = 0; q < 19; ++q) h[c][q] = ref[c][q] + df[c][q] / df_scale;
    } else {
      for (int c = 0; c < NC; ++c)
        for (int q = 0; q < 19; ++q) h[c][q] = ref[c][q];
    }
  } else {
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q) h[c][q] = h[c][q] + df[c][q];
  }
}

template <int NC>
__device__ void le_adjust(const DevParams &P, double h[NC][19], const double ref[NC][19],
                          double shear_u, double sign) {
  double df[NC][19];
  const bool neg = le_adjust_df<NC>(P, h, shear_u, sign, df);
  le_adjust_apply<NC>(h, ref, df, neg);
}

}  // namespace lb3d
