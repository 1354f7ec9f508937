// inflow.cuh -- the Zou-He closures of the stage-8 invasion boundaries,
// templated on the value type: FP64 for the drop-in path (bit-identical to
// the oracle's restatement, every literal exact in both types) and FP32 for
// the deviation path.  F(i) is the reference's 1-based direction i; Fp holds
// the populations times their degeneracy g.
#pragma once

// Zou-He flux boundary of one component at z = 1 (bottom) or z = nz
// (code/lb3d_invasion.F90:2143-2457): the entering populations are closed
// from the known ones and the inflow uz (a flux divided by the density when
// itype < 0), in the expression order of the reference.
template <typename T>
__device__ __forceinline__ void zouhe_flux_site(T *Fp, T uz, bool bottom, int itype) {
  auto F = [&](int i) -> T & { return Fp[i - 1]; };
  const T ux = T(0), uy = T(0);
  T rho;
  if (bottom) {
    if (itype < 0) {
      rho = F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
            T(2) * (F(6) + F(10) + F(14) + F(16) + F(18)) + uz;
      uz = (rho > T(0)) ? uz / rho : T(0);
    } else {
      rho = (F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
             T(2) * (F(6) + F(10) + F(14) + F(16) + F(18))) /
            (T(1) - uz);
    }
    F(5) = F(6) + uz * rho / T(3);
    if (itype == 0) {
      F(15) = F(18) - (F(3) - F(4)) / T(4) + rho * uz / T(6);
      F(17) = F(16) + (F(3) - F(4)) / T(4) + rho * uz / T(6);
      F(9) = F(14) - (F(1) - F(2)) / T(4) + rho * uz / T(6);
      F(13) = F(10) + (F(1) - F(2)) / T(4) + rho * uz / T(6);
    } else if (itype == 1 || itype == -1) {
      F(15) = F(18) - (F(7) + F(11) + F(3) - F(8) - F(12) - F(4)) / T(2) + uz * rho / T(6) + uy * rho / T(2);
      F(17) = F(16) - (F(8) + F(12) + F(4) - F(7) - F(11) - F(3)) / T(2) + uz * rho / T(6) - uy * rho / T(2);
      F(9) = F(14) - (F(7) + F(8) + F(1) - F(11) - F(12) - F(2)) / T(2) + uz * rho / T(6) + ux * rho / T(2);
      F(13) = F(10) - (F(11) + F(12) + F(2) - F(7) - F(8) - F(1)) / T(2) + uz * rho / T(6) - ux * rho / T(2);
    }
  } else {
    if (itype < 0) {
      rho = F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
            T(2) * (F(5) + F(9) + F(13) + F(15) + F(17)) - uz;
      uz = (rho > T(0)) ? uz / rho : T(0);
    } else {
      rho = (F(19) + F(1) + F(2) + F(3) + F(4) + F(7) + F(11) + F(12) + F(8) +
             T(2) * (F(5) + F(9) + F(13) + F(15) + F(17))) /
            (uz + T(1));
    }
    F(6) = F(5) - uz * rho / T(3);
    if (itype == 0) {
      F(18) = F(15) + (F(3) - F(4)) / T(4) - rho * uz / T(6);
      F(16) = F(17) - (F(3) - F(4)) / T(4) - rho * uz / T(6);
      F(14) = F(9) + (F(1) - F(2)) / T(4) - rho * uz / T(6);
      F(10) = F(13) - (F(1) - F(2)) / T(4) - rho * uz / T(6);
    } else if (itype == 1 || itype == -1) {
      F(18) = F(15) + (F(7) + F(11) + F(3) - F(8) - F(12) - F(4)) / T(2) - uz * rho / T(6) - uy * rho / T(2);
      F(16) = F(17) + (F(8) + F(12) + F(4) - F(7) - F(11) - F(3)) / T(2) - uz * rho / T(6) + uy * rho / T(2);
      F(14) = F(9) + (F(7) + F(8) + F(1) - F(11) - F(12) - F(2)) / T(2) - uz * rho / T(6) - ux * rho / T(2);
      F(10) = F(13) + (F(11) + F(12) + F(2) - F(7) - F(8) - F(1)) / T(2) - uz * rho / T(6) + ux * rho / T(2);
    }
  }
}

// Zou-He density boundary of one component (code/lb3d_invasion.F90:1459-1796,
// non-SINGLEFLUID build, Shan-Chen terms zero): the five entering
// populations from the known ones and the imposed density rho; am13 is the
// mass in the rho/6/am term of F(13), amass_r for blue as well (:1567).
template <typename T>
__device__ __forceinline__ void zouhe_density_site(T *Fp, T rho, T am, T am13, T tau,
                                                   bool bottom) {
#define F(i) Fp[(i)-1]
  const T fx = T(0), fy = T(0);
  if (bottom) {
    F(5) = (-T(2) * F(10) - F(11) - F(12) - T(2) * F(14) - T(2) * F(16) - T(2) * F(18) - F(19) - F(1) -
            F(2) - F(3) - F(4) + F(6) - F(7) - F(8)) / T(3) + rho / T(3) / am;
    F(9) = (-F(10) + F(11) + F(12) + T(2) * F(14) - F(16) - F(18) - F(19) / T(2) - T(2) * F(1) + F(2) -
            F(3) / T(2) - F(4) / T(2) - F(6) - T(2) * F(7) - T(2) * F(8)) / T(3) + rho / T(6) / am -
           fx * tau / T(4) / am;
    F(13) = (T(2) * F(10) - T(2) * F(11) - T(2) * F(12) - F(14) - F(16) - F(18) - F(19) / T(2) + F(1) -
             T(2) * F(2) - F(3) / T(2) - F(4) / T(2) - F(6) + F(7) + F(8)) / T(3) + rho / T(6) / am13 +
            fx * tau / T(4) / am;
    F(15) = (-F(10) - T(2) * F(11) + F(12) - F(14) - F(16) + T(2) * F(18) - F(19) / T(2) - F(1) / T(2) -
             F(2) / T(2) - T(2) * F(3) + F(4) - F(6) - T(2) * F(7) + F(8)) / T(3) + rho / T(6) / am -
            fy * tau / T(4) / am;
    F(17) = (-F(10) + F(11) - T(2) * F(12) - F(14) + T(2) * F(16) - F(18) - F(19) / T(2) - F(1) / T(2) -
             F(2) / T(2) + F(3) - T(2) * F(4) - F(6) + F(7) - T(2) * F(8)) / T(3) + rho / T(6) / am +
            fy * tau / T(4) / am;
  } else {
    F(6) = (-F(11) - F(12) - T(2) * F(13) - T(2) * F(15) - T(2) * F(17) - F(19) - F(1) - F(2) - F(3) -
            F(4) + F(5) - F(7) - F(8) - T(2) * F(9)) / T(3) + rho / T(3) / am;
    F(10) = (F(11) + F(12) + T(2) * F(13) - F(15) - F(17) - F(19) / T(2) - T(2) * F(1) + F(2) -
             F(3) / T(2) - F(4) / T(2) - F(5) - T(2) * F(7) - T(2) * F(8) - F(9)) / T(3) + rho / T(6) / am -
            fx * tau / T(4) / am;
    F(14) = (-T(2) * F(11) - T(2) * F(12) - F(13) - F(15) - F(17) - F(19) / T(2) + F(1) - T(2) * F(2) -
             F(3) / T(2) - F(4) / T(2) - F(5) + F(7) + F(8) + T(2) * F(9)) / T(3) + rho / T(6) / am +
            fx * tau / T(4) / am;
    F(16) = (-T(2) * F(11) + F(12) - F(13) - F(15) + T(2) * F(17) - F(19) / T(2) - F(1) / T(2) -
             F(2) / T(2) - T(2) * F(3) + F(4) - F(5) - T(2) * F(7) + F(8) - F(9)) / T(3) + rho / T(6) / am -
            fy * tau / T(4) / am;
    F(18) = (F(11) - T(2) * F(12) - F(13) + T(2) * F(15) - F(17) - F(19) / T(2) - F(1) / T(2) -
             F(2) / T(2) + F(3) - T(2) * F(4) - F(5) + F(7) - T(2) * F(8) - F(9)) / T(3) + rho / T(6) / am +
            fy * tau / T(4) / am;
  }
#undef F
}
