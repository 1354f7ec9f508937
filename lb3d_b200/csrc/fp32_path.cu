// fp32_path.cu -- FP32 deviation storage, one fused stream-collide pass.
//
// Populations are stored as FP32 deviations delta_{c,i} = n_{c,i} - w_i rho0
// from the rest state (w_i = 1/36 moving, 1/3 rest), so the stored values
// and the moment sums carry the small variations at full FP32 relative
// precision.  One kernel launch advances a step: each CTA owns a TX x TY
// column tile and a range of z planes and marches in z with three stages
// per plane, keeping every intermediate field on chip:
//
//   A(k)   post-stream moments on the tile plus a halo of H sites
//          (H = 2 ternary, 1 binary): pull 19*nc deviations, densities,
//          psi deviations dpsi = psi(rho) - psi(rho0) = -e^{-rho0}
//          expm1(-drho), and (ternary) the advected dipole flux da using the
//          previous dipoles staged in shared memory.
//   B(k-1) (ternary) dipole relaxation on the tile plus a one-site halo
//          from the A ring (code/lb3d_collision.F90:296-403).
//   C(k-H) Shan-Chen force from the on-chip psi/dipole rings, body force,
//          the pull of the own site's populations (an L2 hit: the same
//          values were pulled by stage A two planes earlier), the
//          equilibrium of code/lb3d_bdist.F90:301-370 in deviation form
//          and the BGK update, written to the other buffer.
//
// HBM traffic per site and step is therefore one read and one write of the
// 19*nc deviations (plus the dipoles and a rock byte), against ~800 B for a
// three-kernel split.  Nothing in the path is a dense contraction, so there
// are no tensor cores; the roofline is HBM bandwidth.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstring>
#include <vector>

#include "fp32_path.h"
#include "reduce.h"
#include "fp64_path.h"
#include "le_common.cuh"

namespace lb3d {
namespace f32 {

constexpr float W1 = 1.0f / 36.0f;
constexpr float W0 = 1.0f / 3.0f;
LB3D_HDI constexpr float wq(int q) { return q == 18 ? W0 : W1; }

__device__ __forceinline__ int pmod(int v, int n) {
  int r = v % n;
  return r < 0 ? r + n : r;
}
// Periodic wrap without a division when v lies within one period of the
// lattice (-n <= v < 2n), the case of every tile and halo coordinate of a
// lattice at least as large as the halo; pmod otherwise.
__device__ __forceinline__ int wrapz(int v, int n) {
  if (v >= -n && v < 2 * n) return v < 0 ? v + n : (v >= n ? v - n : v);
  return pmod(v, n);
}

// Langevin function L(x) = coth x - 1/x, accurate in FP32 for small x.
__device__ __forceinline__ float langevin(float x) {
  if (x < 0.3f) {
    float x2 = x * x;
    return x * fmaf(x2, fmaf(x2, fmaf(x2, -1.0f / 4725.0f, 2.0f / 945.0f), -1.0f / 45.0f), 1.0f / 3.0f);
  }
  float t = tanhf(x);
  return 1.0f / t - 1.0f / x;
}

// Equilibrium deviation for one component: deq_i = rho*(E_i(v) - w_i) + drho*w_i
// with E of bdist = 2 (code/lb3d_bdist.F90:301-370), then the BGK update
// d_i <- d_i + omega (deq_i - d_i), evaluated as (1 - omega) d_i + omega deq_i
// with omega folded into the equilibrium's coefficients.  Every multiply-add
// is written out (fmaf), so bgk_update2 below can repeat the same roundings
// lane by lane.
__device__ __forceinline__ void bgk_update(float d[19], float rho, float drho, float vx, float vy,
                                           float vz, float omega) {
  const float tx = 3.0f * vx, ty = 3.0f * vy, tz = 3.0f * vz;
  const float uke = 0.5f * fmaf(tz, vz, fmaf(ty, vy, tx * vx));
  const float a = -uke;          // even part minus w
  const float b = 1.0f + a;      // odd linear coefficient
  const float orw = (omega * rho) * W1;
  const float obase = (omega * drho) * W1;
  const float om1 = 1.0f - omega;
#define LB3D_PAIR32(CD, I, J)                                             \
  {                                                                       \
    const float e = (CD);                                                 \
    const float e2 = e * e;                                               \
    const float ev = fmaf(orw, fmaf(0.5f, e2, a), obase);                 \
    const float od = (orw * e) * fmaf(e2, 1.0f / 6.0f, b);                \
    d[I] = fmaf(om1, d[I], ev + od);                                      \
    d[J] = fmaf(om1, d[J], ev - od);                                      \
  }
  LB3D_PAIR32(tx, 0, 1)
  LB3D_PAIR32(ty, 2, 3)
  LB3D_PAIR32(tz, 4, 5)
  LB3D_PAIR32(tx + ty, 6, 11)
  LB3D_PAIR32(tx - ty, 7, 10)
  LB3D_PAIR32(tx + tz, 8, 13)
  LB3D_PAIR32(tx - tz, 9, 12)
  LB3D_PAIR32(ty + tz, 14, 17)
  LB3D_PAIR32(ty - tz, 15, 16)
#undef LB3D_PAIR32
  const float oeq0 = fmaf((omega * rho) * W0, a, (omega * drho) * W0);
  d[18] = fmaf(om1, d[18], oeq0);
}

// Paired FP32 arithmetic (sm_100 FADD2/FMUL2/FFMA2: two lanes per
// instruction, each rounded as its scalar counterpart).
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// bgk_update for two components at once (lane x, lane y), bit for bit the
// scalar routine on each lane.
__device__ __forceinline__ void bgk_update2(float2 d[19], float2 rho, float2 drho, float2 vx,
                                            float2 vy, float2 vz, float2 omega) {
  const float2 tx = mul2(f2(3.0f), vx), ty = mul2(f2(3.0f), vy), tz = mul2(f2(3.0f), vz);
  const float2 uke = mul2(f2(0.5f), fma2(tz, vz, fma2(ty, vy, mul2(tx, vx))));
  const float2 a = neg2(uke);
  const float2 b = add2(f2(1.0f), a);
  const float2 orw = mul2(mul2(omega, rho), f2(W1));
  const float2 obase = mul2(mul2(omega, drho), f2(W1));
  const float2 om1 = add2(f2(1.0f), neg2(omega));
#define LB3D_PAIR2(CD, I, J)                                                  \
  {                                                                           \
    const float2 e = (CD);                                                    \
    const float2 e2 = mul2(e, e);                                             \
    const float2 ev = fma2(orw, fma2(f2(0.5f), e2, a), obase);                \
    const float2 od = mul2(mul2(orw, e), fma2(e2, f2(1.0f / 6.0f), b));       \
    d[I] = fma2(om1, d[I], add2(ev, od));                                     \
    d[J] = fma2(om1, d[J], add2(ev, neg2(od)));                               \
  }
  LB3D_PAIR2(tx, 0, 1)
  LB3D_PAIR2(ty, 2, 3)
  LB3D_PAIR2(tz, 4, 5)
  LB3D_PAIR2(add2(tx, ty), 6, 11)
  LB3D_PAIR2(add2(tx, neg2(ty)), 7, 10)
  LB3D_PAIR2(add2(tx, tz), 8, 13)
  LB3D_PAIR2(add2(tx, neg2(tz)), 9, 12)
  LB3D_PAIR2(add2(ty, tz), 14, 17)
  LB3D_PAIR2(add2(ty, neg2(tz)), 15, 16)
#undef LB3D_PAIR2
  const float2 oeq0 = fma2(mul2(mul2(omega, rho), f2(W0)), a, mul2(mul2(omega, drho), f2(W0)));
  d[18] = fma2(om1, d[18], oeq0);
}

// Equilibrium deviations of one component written straight to the output
// (full relaxation: the BGK update with omega = 1), with bgk_update's
// arithmetic; out[q * S] receives population q.
__device__ __forceinline__ void eq_store(float *out, unsigned S, float rho, float drho, float vx, float vy,
                                         float vz, float omega) {
  const float tx = 3.0f * vx, ty = 3.0f * vy, tz = 3.0f * vz;
  const float uke = 0.5f * fmaf(tz, vz, fmaf(ty, vy, tx * vx));
  const float a = -uke;
  const float b = 1.0f + a;
  const float orw = (omega * rho) * W1;
  const float obase = (omega * drho) * W1;
#define LB3D_EQ32(CD, I, J)                                               \
  {                                                                       \
    const float e = (CD);                                                 \
    const float e2 = e * e;                                               \
    const float ev = fmaf(orw, fmaf(0.5f, e2, a), obase);                 \
    const float od = (orw * e) * fmaf(e2, 1.0f / 6.0f, b);                \
    __stcs(out + (I) * S, ev + od);                                       \
    __stcs(out + (J) * S, ev - od);                                       \
  }
  LB3D_EQ32(tx, 0, 1)
  LB3D_EQ32(ty, 2, 3)
  LB3D_EQ32(tz, 4, 5)
  LB3D_EQ32(tx + ty, 6, 11)
  LB3D_EQ32(tx - ty, 7, 10)
  LB3D_EQ32(tx + tz, 8, 13)
  LB3D_EQ32(tx - tz, 9, 12)
  LB3D_EQ32(ty + tz, 14, 17)
  LB3D_EQ32(ty - tz, 15, 16)
#undef LB3D_EQ32
  __stcs(out + 18 * S, fmaf((omega * rho) * W0, a, (omega * drho) * W0));
}
// eq_store for two components (lanes x, y) with bgk_update2's paired
// arithmetic; lane x goes to outA, lane y to outB.
// With bA (optional) the two components' values also go to bA[q * SB] and
// bB[q * SB].
__device__ __forceinline__ void eq_store2(float *outA, float *outB, unsigned S, float2 rho, float2 drho,
                                          float2 vx, float2 vy, float2 vz, float2 omega,
                                          float *bA = nullptr, float *bB = nullptr, unsigned SB = 0) {
  const float2 tx = mul2(f2(3.0f), vx), ty = mul2(f2(3.0f), vy), tz = mul2(f2(3.0f), vz);
  const float2 uke = mul2(f2(0.5f), fma2(tz, vz, fma2(ty, vy, mul2(tx, vx))));
  const float2 a = neg2(uke);
  const float2 b = add2(f2(1.0f), a);
  const float2 orw = mul2(mul2(omega, rho), f2(W1));
  const float2 obase = mul2(mul2(omega, drho), f2(W1));
#define LB3D_EQ2(CD, I, J)                                                    \
  {                                                                           \
    const float2 e = (CD);                                                    \
    const float2 e2 = mul2(e, e);                                             \
    const float2 ev = fma2(orw, fma2(f2(0.5f), e2, a), obase);                \
    const float2 od = mul2(mul2(orw, e), fma2(e2, f2(1.0f / 6.0f), b));       \
    const float2 p = add2(ev, od), m = add2(ev, neg2(od));                    \
    __stcs(outA + (I) * S, p.x);                                              \
    __stcs(outB + (I) * S, p.y);                                              \
    __stcs(outA + (J) * S, m.x);                                              \
    __stcs(outB + (J) * S, m.y);                                              \
    if (bA) {                                                                 \
      bA[(I) * SB] = p.x;                                                     \
      bB[(I) * SB] = p.y;                                                     \
      bA[(J) * SB] = m.x;                                                     \
      bB[(J) * SB] = m.y;                                                     \
    }                                                                         \
  }
  LB3D_EQ2(tx, 0, 1)
  LB3D_EQ2(ty, 2, 3)
  LB3D_EQ2(tz, 4, 5)
  LB3D_EQ2(add2(tx, ty), 6, 11)
  LB3D_EQ2(add2(tx, neg2(ty)), 7, 10)
  LB3D_EQ2(add2(tx, tz), 8, 13)
  LB3D_EQ2(add2(tx, neg2(tz)), 9, 12)
  LB3D_EQ2(add2(ty, tz), 14, 17)
  LB3D_EQ2(add2(ty, neg2(tz)), 15, 16)
#undef LB3D_EQ2
  const float2 oeq0 = fma2(mul2(mul2(omega, rho), f2(W0)), a, mul2(mul2(omega, drho), f2(W0)));
  __stcs(outA + 18 * S, oeq0.x);
  __stcs(outB + 18 * S, oeq0.y);
  if (bA) {
    bA[18 * SB] = oeq0.x;
    bB[18 * SB] = oeq0.y;
  }
}

// Own-site moments of one component's post-stream deviations d[q * ST]:
// drho = sum_q g_q d_q and j = sum_q g_q c_q d_q, in q order, one fused
// multiply-add per term.
template <int ST>
__device__ __forceinline__ void own_moments(const float *d, float &dr, float &j0, float &j1,
                                            float &j2) {
  float r = 0.f, a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const float v = d[q * ST], g = (float)gw(q);
    r = fmaf(g, v, r);
    if (cx(q)) a0 = fmaf(g * (float)cx(q), v, a0);
    if (cy(q)) a1 = fmaf(g * (float)cy(q), v, a1);
    if (cz(q)) a2 = fmaf(g * (float)cz(q), v, a2);
  }
  dr = r;
  j0 = a0;
  j1 = a1;
  j2 = a2;
}
// own_moments2 of values already in registers (lane x, lane y).
__device__ __forceinline__ void own_moments2_reg(const float2 v[19], float2 &dr, float2 &j0,
                                                 float2 &j1, float2 &j2) {
  float2 r = f2(0.f), a0 = f2(0.f), a1 = f2(0.f), a2 = f2(0.f);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const float g = (float)gw(q);
    r = fma2(f2(g), v[q], r);
    if (cx(q)) a0 = fma2(f2(g * (float)cx(q)), v[q], a0);
    if (cy(q)) a1 = fma2(f2(g * (float)cy(q)), v[q], a1);
    if (cz(q)) a2 = fma2(f2(g * (float)cz(q)), v[q], a2);
  }
  dr = r;
  j0 = a0;
  j1 = a1;
  j2 = a2;
}
// own_moments of two components (lanes x, y) with paired instructions.
template <int ST>
__device__ __forceinline__ void own_moments2(const float *dA, const float *dB, float2 &dr,
                                             float2 &j0, float2 &j1, float2 &j2) {
  float2 r = f2(0.f), a0 = f2(0.f), a1 = f2(0.f), a2 = f2(0.f);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const float2 v = make_float2(dA[q * ST], dB[q * ST]);
    const float g = (float)gw(q);
    r = fma2(f2(g), v, r);
    if (cx(q)) a0 = fma2(f2(g * (float)cx(q)), v, a0);
    if (cy(q)) a1 = fma2(f2(g * (float)cy(q)), v, a1);
    if (cz(q)) a2 = fma2(f2(g * (float)cz(q)), v, a2);
  }
  dr = r;
  j0 = a0;
  j1 = a1;
  j2 = a2;
}

// Site offsets (32-bit, relative to the lattice base) of the -1, 0, +1
// neighbours along each axis, with the periodic wrap applied once.
struct Nbr {
  int cx[3], ry[3], rz[3];
};

__device__ __forceinline__ void make_nbr(Nbr &n, int gx, int gy, int gz, int nx, int ny, int nz) {
  const int pl = nx * ny;
  n.cx[0] = gx == 0 ? nx - 1 : gx - 1;
  n.cx[1] = gx;
  n.cx[2] = gx == nx - 1 ? 0 : gx + 1;
  n.ry[0] = (gy == 0 ? ny - 1 : gy - 1) * nx;
  n.ry[1] = gy * nx;
  n.ry[2] = (gy == ny - 1 ? 0 : gy + 1) * nx;
  n.rz[0] = (gz == 0 ? nz - 1 : gz - 1) * pl;
  n.rz[1] = gz * pl;
  n.rz[2] = (gz == nz - 1 ? 0 : gz + 1) * pl;
}
// site offset of x + s*c_q (s = +1 neighbour, s = -1 upstream)
template <int Q, int SGN>
__device__ __forceinline__ int noff(const Nbr &n) {
  return n.cx[1 + SGN * cx(Q)] + n.ry[1 + SGN * cy(Q)] + n.rz[1 + SGN * cz(Q)];
}

// Pulls the post-stream deviations of component C of one site (with
// half-way bounce-back when ROCK): d[q] = delta*(x - c_q, q), or
// delta*(x, bounce(q)) when x - c_q is rock (code/lb3d_bc_bounce.F90:53-90
// with code/lb3d_advection.F90:109-151).  F points at component 0 of the
// lattice; the component stride is 19*S.
// LAST selects the last-use load hint (the final read of these values by
// this CTA), which lets L2 drop the lines early.  NARROW forms the component
// offset c*19*S in 32 bits (lattices with 19*nc*S < 2^32), which keeps the
// register-capped moments pass free of 64-bit products.
template <bool ROCK, bool LAST = false, bool NARROW = false>
__device__ __forceinline__ void pull_comp(const float *__restrict__ F, unsigned S, int c, const Nbr &n,
                                          int self, const uint8_t *__restrict__ rk, float d[19]) {
  const float *fc = NARROW ? F + (unsigned)(c * 19) * S : F + (size_t)(c * 19) * S;
  d[18] = LAST ? __ldlu(fc + 18 * S + self) : __ldg(fc + 18 * S + self);
#define LB3D_PULL(Q)                                                     \
  {                                                                      \
    const int up = noff<Q, -1>(n);                                       \
    bool uf = true;                                                      \
    if (ROCK) uf = __ldg(rk + up) == 0;                                  \
    const float *a_ = fc + (uf ? Q * S + up : bounce(Q) * S + self);     \
    d[Q] = LAST ? __ldlu(a_) : __ldg(a_);                                \
  }
  LB3D_PULL(0) LB3D_PULL(1) LB3D_PULL(2) LB3D_PULL(3) LB3D_PULL(4) LB3D_PULL(5)
  LB3D_PULL(6) LB3D_PULL(7) LB3D_PULL(8) LB3D_PULL(9) LB3D_PULL(10) LB3D_PULL(11)
  LB3D_PULL(12) LB3D_PULL(13) LB3D_PULL(14) LB3D_PULL(15) LB3D_PULL(16) LB3D_PULL(17)
#undef LB3D_PULL
}

// Lees-Edwards pulls (binary, no rock; code/lb3d_bc_leesedwards.F90:147-1315
// feeding code/lb3d_advection.F90:109-151): across x = 0 (c_x = +1) and
// x = nx - 1 (c_x = -1) the upstream site lies in the sheared halo planes
// Lg.le_h[0] / Lg.le_h[1], [nc][19][nz][ny], at the wrapped (y - c_y, z - c_z).
struct LeYZ {
  int y[3], z[3];  // wrap(gy + k - 1) and ny * wrap(gz + k - 1)
};
__device__ __forceinline__ void make_leyz(LeYZ &w, int gy, int gz, int ny, int nz) {
  w.y[0] = gy == 0 ? ny - 1 : gy - 1;
  w.y[1] = gy;
  w.y[2] = gy == ny - 1 ? 0 : gy + 1;
  w.z[0] = ny * (gz == 0 ? nz - 1 : gz - 1);
  w.z[1] = ny * gz;
  w.z[2] = ny * (gz == nz - 1 ? 0 : gz + 1);
}
// With ROCK (walls) the sheared halo sites are never rock, as the
// reference's exchange leaves them (code/lb3d_bc_leesedwards.F90:678,866),
// and a pull from a rock site inside the lattice bounces back.
template <int Q, bool ROCK = false>
__device__ __forceinline__ const float *le_src(const float *fc, unsigned S, int c, const Nbr &n, int gx,
                                               int nx, const LeYZ &w, const LatDesc &Lg, int NP,
                                               int self = 0, const uint8_t *__restrict__ rk = nullptr) {
  if (cx(Q) == 1 && gx == 0) return Lg.le_h[0] + (c * 19 + Q) * NP + w.y[1 - cy(Q)] + w.z[1 - cz(Q)];
  if (cx(Q) == -1 && gx == nx - 1)
    return Lg.le_h[1] + (c * 19 + Q) * NP + w.y[1 - cy(Q)] + w.z[1 - cz(Q)];
  const int up = noff<Q, -1>(n);
  if (ROCK && __ldg(rk + up) != 0) return fc + bounce(Q) * S + self;
  return fc + Q * S + up;
}
template <bool NARROW = false, bool ROCK = false>
__device__ __forceinline__ void pull_comp_le(const float *__restrict__ F, unsigned S, int c, const Nbr &n,
                                             int self, int gx, int nx, const LeYZ &w,
                                             const LatDesc &Lg, int NP, float d[19],
                                             const uint8_t *__restrict__ rk = nullptr) {
  const float *fc = NARROW ? F + (unsigned)(c * 19) * S : F + (size_t)(c * 19) * S;
  d[18] = __ldg(fc + 18 * S + self);
#define LB3D_PULL_LE(Q) d[Q] = __ldg(le_src<Q, ROCK>(fc, S, c, n, gx, nx, w, Lg, NP, self, rk));
  LB3D_PULL_LE(0) LB3D_PULL_LE(1) LB3D_PULL_LE(2) LB3D_PULL_LE(3) LB3D_PULL_LE(4) LB3D_PULL_LE(5)
  LB3D_PULL_LE(6) LB3D_PULL_LE(7) LB3D_PULL_LE(8) LB3D_PULL_LE(9) LB3D_PULL_LE(10) LB3D_PULL_LE(11)
  LB3D_PULL_LE(12) LB3D_PULL_LE(13) LB3D_PULL_LE(14) LB3D_PULL_LE(15) LB3D_PULL_LE(16) LB3D_PULL_LE(17)
#undef LB3D_PULL_LE
}

// Writes one component's 19 deviations of a site on the x boundary of a
// Lees-Edwards lattice to the compact boundary planes: set 0 (pre-stream,
// le_b[0] at x = nx - 1, le_b[1] at x = 0) or set 2 (post-stream, le_b[2],
// le_b[3]); sites elsewhere write nothing.
__device__ __forceinline__ void le_store_boundary(const LatDesc &Lg, int set, int c, int gx, int gy,
                                                  int gz, const float d[19]) {
  const int nx = Lg.nx, NP = Lg.ny * Lg.nz;
  const int o = (c * 19) * NP + gy + Lg.ny * gz;
  if (gx == nx - 1) {
    float *b = Lg.le_b[set] + o;
#pragma unroll
    for (int q = 0; q < 19; ++q) b[q * NP] = d[q];
  }
  if (gx == 0) {
    float *b = Lg.le_b[set + 1] + o;
#pragma unroll
    for (int q = 0; q < 19; ++q) b[q * NP] = d[q];
  }
}

// ---------------------------------------------------------------------------
// The fused kernel.  Grid: persistent CTAs over a tile list.  Populations
// of lattice L live at f[(c*19+q)*S + L.base + site]; each component's
// base is a 64-bit pointer and the offsets within a component are unsigned
// 32-bit, which bounds the packed capacity at 19*S < 2^32 sites.
//
// On-chip rings (float4 entries, one per site):
//   A  ternary: {rho_b - rho_r, da_x, da_y, da_z}, {drho_s, dpsi_r, dpsi_b,
//      dpsi_s} on the tile + 2 halo, 4 planes;  binary: {dpsi_r, dpsi_b, -, -}
//      on the tile + 1 halo, 3 planes
//   B  ternary: new dipoles {d_x, d_y, d_z, -} on the tile + 1 halo, 3 planes
//   D  ternary: previous dipoles on the tile + 3 halo, 3 planes
// ---------------------------------------------------------------------------
#include "fp32_stencil.cuh"
#include "inflow.cuh"

// Stage-8 inflow boundaries of one site on the FP32 path
// (code/lb3d_bc.F90:125-133 runs them between advection and collision):
// applied to the site's post-stream deviations after its own moments were
// taken, as the reference's collision keeps the advection moments.  Each
// closure works on the populations n = d + w rho0 in FP32 and writes the
// deviations back.  Recolouring (code/lb3d_invasion.F90:1257-1358) visits
// z = 0, 1 and then z = nz - 2, nz - 1 in that order, so planes that are
// both are recoloured twice as the reference's two loops do; the Zou-He
// closures (inflow.cuh) act on z = 0 and z = nz - 1 per component,
// surfactant first.
template <int NC>
__device__ __forceinline__ void inflow_site(float2 d01[19], float ds[19], const LatDesc &Lg, int gz,
                                            int nz) {
  const float r0 = Lg.rho0;
  if (Lg.invk == 1) {
    const float mr = Lg.inv_fluid == 7 ? 1.0f : 0.0f, mb = 1.0f - mr;
    const int zs[4] = {0, 1, nz - 2, nz - 1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (gz != zs[k]) continue;
      const float a = k < 2 ? mr : mb, b = k < 2 ? mb : mr;
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        const float w = wq(q) * r0;
        const float pop = (d01[q].x + w) + (d01[q].y + w);
        d01[q].x = a * pop - w;
        d01[q].y = b * pop - w;
      }
    }
    return;
  }
  const bool bottom = gz == 0;
  if (!bottom && gz != nz - 1) return;
  float F[19];
  if (NC == 3 && Lg.invk == 3) {
#pragma unroll
    for (int q = 0; q < 19; ++q) F[q] = (ds[q] + wq(q) * r0) * (float)gw(q);
    zouhe_flux_site<float>(F, Lg.zh_uz[2], bottom, Lg.inv_type);
#pragma unroll
    for (int q = 0; q < 19; ++q) ds[q] = F[q] / (float)gw(q) - wq(q) * r0;
  }
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int q = 0; q < 19; ++q) F[q] = ((c ? d01[q].y : d01[q].x) + wq(q) * r0) * (float)gw(q);
    if (Lg.invk == 3)
      zouhe_flux_site<float>(F, Lg.zh_uz[c], bottom, Lg.inv_type);
    else
      zouhe_density_site<float>(F, bottom ? Lg.zh_in[c] : Lg.zh_uz[c], Lg.amass[c],
                                bottom ? Lg.amass[0] : Lg.amass[c], Lg.tau[c], bottom);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      const float d = F[q] / (float)gw(q) - wq(q) * r0;
      if (c) d01[q].y = d; else d01[q].x = d;
    }
  }
}

// Kernel modes.  FUSED: one pass per step (moments recomputed on the halo).
// MOMENTS + COLLIDE: the split strategy, two passes per step: MOMENTS
// writes each site's post-stream moment entry (the A-ring entry) to a
// global field M exactly once, COLLIDE loads M with its halo into the same
// rings and runs the dipole, force and BGK stages.
constexpr int MODE_FUSED = 0, MODE_MOMENTS = 1, MODE_COLLIDE = 2;

template <int NC, int TX, int TY, int MODE>
struct FusedGeom {
  static constexpr int NT = TX * TY;
  static constexpr int H = (MODE == MODE_MOMENTS) ? 0 : ((NC == 3) ? 2 : 1);
  static constexpr int AW = TX + 2 * H, AH = TY + 2 * H, AN = AW * AH;
  static constexpr int AV = (NC == 3) ? 2 : 1;  // float4 per A entry
  static constexpr int AR = (NC == 3) ? 4 : 3;  // A ring depth
  static constexpr int BW = TX + 2, BH = TY + 2, BN = BW * BH;
  static constexpr int DH_ = (MODE == MODE_MOMENTS) ? 1 : 3;  // D-ring halo
  static constexpr int DW = TX + 2 * DH_, DH = TY + 2 * DH_, DN = DW * DH;
  static constexpr int A_F4 = (MODE == MODE_MOMENTS) ? 0 : AR * AV * AN;
  static constexpr int B_F4 = (NC == 3 && MODE != MODE_MOMENTS) ? 3 * BN : 0;
  static constexpr int D_F4 = (NC == 3 && MODE != MODE_COLLIDE) ? 3 * DN : 0;
  static constexpr int SMEM = 16 * (A_F4 + B_F4 + D_F4);
};

template <int NC, int TX, int TY, bool ROCK, bool BODY, int MODE, bool LE = false,
          bool NARROW = false>
__global__ void __launch_bounds__(TX *TY, (MODE == MODE_MOMENTS ? 1024 / (TX * TY) : (TX * TY >= 512 ? 1 : (TX * TY >= 256 ? 2 : 3))))
    k_fused(const LatDesc *__restrict__ lats, const Tile *__restrict__ tiles, int ntiles,
            float *f0, float *f1, float *db0, float *db1, const uint8_t *__restrict__ rock, unsigned S,
            float4 *__restrict__ Mf, float4 *__restrict__ Jf) {
  using G = FusedGeom<NC, TX, TY, MODE>;
  constexpr int NT = G::NT, H = G::H, AW = G::AW, AN = G::AN, AV = G::AV, AR = G::AR;
  constexpr int BW = G::BW, BN = G::BN, DW = G::DW, DN = G::DN, DHH = G::DH_;
  extern __shared__ float4 smem4[];
  float4 *ringA = smem4;              // [AR][AV][AN]
  float4 *ringB = ringA + G::A_F4;    // [3][BN]
  float4 *ringD = ringB + G::B_F4;    // [3][DN]
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;

  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    const LatDesc &Lg = lats[T.lat];
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    const int base = (int)Lg.base;
    const int par = Lg.parity;
    const float *__restrict__ F = (par ? f1 : f0) + base;
    float *__restrict__ Fo = (par ? f0 : f1) + base;
    const float *__restrict__ DBi = (NC == 3) ? (par ? db1 : db0) + base : nullptr;
    float *__restrict__ DBo = (NC == 3) ? (par ? db0 : db1) + base : nullptr;
    const uint8_t *__restrict__ RK = rock + base;
    const float rho0 = Lg.rho0, em0 = Lg.em0, psi0 = Lg.psi0;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    const int zfirst = z0 - H;
    const int niter = zc + 2 * H;
    float4 *__restrict__ Mb = Mf ? Mf + base : nullptr;  // moment field of this lattice
    float4 *__restrict__ Jb = Jf ? Jf + base : nullptr;  // own-site moments
    // halo coordinates wrap with wrapz (a division only when the lattice is
    // narrower than the halo)
    auto wx = [&](int v) { return wrapz(v, nx); };
    auto wy = [&](int v) { return wrapz(v, ny); };

    auto load_db_plane = [&](int j) {
      const int gz = wrapz(zfirst - 1 + j, nz);
      float4 *dst = ringD + (j % 3) * DN;
      for (int s = tid; s < DN; s += NT) {
        const int gx = wx(x0 - DHH + s % DW), gy = wy(y0 - DHH + s / DW);
        const int i = gx + nx * (gy + ny * gz);
        dst[s] = make_float4(__ldg(DBi + i), __ldg(DBi + S + i), __ldg(DBi + 2 * S + i), 0.0f);
      }
    };
    if (NC == 3 && MODE != MODE_COLLIDE) {
      load_db_plane(0);
      load_db_plane(1);
    }

    for (int it = 0; it < niter; ++it) {
      const int zA = zfirst + it;
      if (NC == 3 && MODE != MODE_COLLIDE) load_db_plane(it + 2);
      __syncthreads();
      // ---------------- stage A: post-stream moments on the haloed tile ----
      {
        float4 *slot = ringA + (it % AR) * AV * AN;
        const int gz = wrapz(zA, nz);
        // D ring: plane zfirst - 1 + j sits in slot j % 3
        const float4 *Dm = ringD + (it % 3) * DN;        // plane zA - 1
        const float4 *D0 = ringD + ((it + 1) % 3) * DN;  // plane zA
        const float4 *Dp = ringD + ((it + 2) % 3) * DN;  // plane zA + 1
        for (int s = tid; s < AN; s += NT) {
          const int ax = s % AW, ay = s / AW;
          const int gx = wx(x0 - H + ax), gy = wy(y0 - H + ay);
          Nbr nb;
          make_nbr(nb, gx, gy, gz, nx, ny, nz);
          const int self = noff<18, 1>(nb);
          LeYZ lw;
          if constexpr (LE) make_leyz(lw, gy, gz, ny, nz);
          float dr[NC], jm[NC][3];
          float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            float d[19];
            if constexpr (LE) {
              if (ROCK && __ldg(RK + self) != 0) {
                // a rock site keeps its (zero) populations
                // (code/lb3d_advection.F90:109-151 pulls into fluid sites only)
                const float *fc = F + (size_t)(c * 19) * S + self;
#pragma unroll
                for (int q = 0; q < 19; ++q) d[q] = __ldg(fc + q * S);
              } else {
                pull_comp_le<NARROW, ROCK>(F, S, c, nb, self, gx, nx, lw, Lg, ny * nz, d, RK);
              }
              // the post-stream populations of the x boundary planes, for
              // the stage-8 halo kernel
              if (MODE == MODE_MOMENTS && x0 + ax < nx && y0 + ay < ny)
                le_store_boundary(Lg, 2, c, gx, gy, gz, d);
            } else {
              pull_comp<ROCK, false, NARROW>(F, S, c, nb, self, RK, d);
            }
            if (MODE == MODE_MOMENTS) {
              own_moments<1>(d, dr[c], jm[c][0], jm[c][1], jm[c][2]);
            } else {
              float acc = 0.0f;
#pragma unroll
              for (int q = 0; q < 19; ++q) acc = fmaf((float)gw(q), d[q], acc);
              dr[c] = acc;
            }
            if (NC == 3 && c == 2) {
              // Zou-He flux boundaries change the surfactant's populations on
              // the z planes before its advected dipole flux is summed
              // (code/lb3d_invasion.F90:2143-2457 recomputes it there)
              if (MODE == MODE_MOMENTS && Lg.invk == 3 && (gz == 0 || gz == nz - 1)) {
                float Fs[19];
#pragma unroll
                for (int q = 0; q < 19; ++q) Fs[q] = (d[q] + wq(q) * rho0) * (float)gw(q);
                zouhe_flux_site<float>(Fs, Lg.zh_uz[2], gz == 0, Lg.inv_type);
#pragma unroll
                for (int q = 0; q < 19; ++q) d[q] = Fs[q] / (float)gw(q) - wq(q) * rho0;
              }
              // da = sum_q (n_s(x - c_q, q) g_q) db(x - c_q) + n_s(x, rest) db(x)
              // (code/lb3d_advection.F90:137-148)
              const int ds0 = (ax + 1) + DW * (ay + 1);  // A-local -> D-local
#pragma unroll
              for (int q = 0; q < 19; ++q) {
                const float4 *Dq = cz(q) == 1 ? Dm : (cz(q) == -1 ? Dp : D0);
                const float4 b = Dq[ds0 - cx(q) - DW * cy(q)];
                const float ng = (float)gw(q) * fmaf(wq(q), rho0, d[q]);
                a0 = fmaf(ng, b.x, a0);
                a1 = fmaf(ng, b.y, a1);
                a2 = fmaf(ng, b.z, a2);
              }
            }
          }
          float4 e0, e1;
          if (NC == 3) {
            e0 = make_float4(dr[1] - dr[0], a0, a1, a2);
            e1 = make_float4(dr[NC - 1], -em0 * expm1f(-dr[0]), -em0 * expm1f(-dr[1]),
                             -em0 * expm1f(-dr[NC - 1]));
          } else {
            e0 = make_float4(-em0 * expm1f(-dr[0]), -em0 * expm1f(-dr[1]), 0.f, 0.f);
          }
          if (MODE == MODE_MOMENTS) {
            // one entry per site, the tile only (H = 0)
            if (x0 + ax < nx && y0 + ay < ny) {
              if (NC == 3) {
                Mb[self] = e0;
                Mb[S + self] = e1;
                if (Jb) {
                  Jb[self] = make_float4(dr[0], dr[1], dr[2], jm[0][0]);
                  Jb[S + self] = make_float4(jm[0][1], jm[0][2], jm[1][0], jm[1][1]);
                  Jb[2 * S + self] = make_float4(jm[1][2], jm[NC - 1][0], jm[NC - 1][1], jm[NC - 1][2]);
                }
              } else {
                reinterpret_cast<float2 *>(Mb)[self] = make_float2(e0.x, e0.y);
                if (Jb) {
                  Jb[self] = make_float4(dr[0], dr[1], jm[0][0], jm[0][1]);
                  Jb[S + self] = make_float4(jm[0][2], jm[1][0], jm[1][1], jm[1][2]);
                }
              }
            }
          } else {
            slot[s] = e0;
            if (NC == 3) slot[AN + s] = e1;
          }
        }
      }  // stage A
      __syncthreads();
      if (MODE == MODE_MOMENTS) continue;
      // ---------------- stage B (ternary): dipole relaxation ----------------
      if constexpr (NC == 3) if (it >= 2) {
        float4 *slotB = ringB + (it % 3) * BN;
        const int zB = zA - 1;
        const float4 *Am = ringA + ((it - 2) % AR) * AV * AN;  // plane zB - 1
        const float4 *A0 = ringA + ((it - 1) % AR) * AV * AN;  // plane zB
        const float4 *Ap = ringA + ((it) % AR) * AV * AN;      // plane zB + 1
        for (int s = tid; s < BN; s += NT) {
          const int bx = s % BW, by = s / BW;
          const int as = (bx + 1) + AW * (by + 1);
          const float3 nd = dipole_site<AW>(Am, A0, Ap, as, Lg, rho0, A0[AN + as].x);
          const float n0 = nd.x, n1 = nd.y, n2 = nd.z;
          slotB[s] = make_float4(n0, n1, n2, 0.0f);
          if (bx >= 1 && bx <= TX && by >= 1 && by <= TY && zB >= z0 && zB < z0 + zc) {
            const int gx = x0 + bx - 1, gy = y0 + by - 1;
            if (gx < nx && gy < ny) {
              const int i = gx + nx * (gy + ny * wrapz(zB, nz));
              __stcs(DBo + i, n0);
              __stcs(DBo + S + i, n1);
              __stcs(DBo + 2 * S + i, n2);
            }
          }
        }
        __syncthreads();
      }
      // ---------------- stage C: force + BGK on the tile ---------------------
      const int itC = it - H;  // A iteration of plane zC
      const int zC = zA - H;
      if (zC >= z0 && zC < z0 + zc) {
        const int gx = x0 + tx, gy = y0 + ty;
        if (gx < nx && gy < ny) {
          const int gz = wrapz(zC, nz);
          Nbr nb;
          make_nbr(nb, gx, gy, gz, nx, ny, nz);
          const int self = noff<18, 1>(nb);
          bool own_rock = false;
          if (ROCK) own_rock = __ldg(RK + self) != 0;
          if (!own_rock) {
            const int as = (tx + H) + AW * (ty + H);
            const float4 *Am = ringA + ((itC + AR - 1) % AR) * AV * AN;
            const float4 *A0 = ringA + (itC % AR) * AV * AN;
            const float4 *Ap = ringA + ((itC + 1) % AR) * AV * AN;
            float Fx[NC][3];
            if constexpr (NC == 3) {
              // ---- ternary Shan-Chen force, code/lb3d_force_shanchen.F90:215-330
              const int itB = itC + 1;  // B computed plane zC at iteration itC + 1
              const int bs = (tx + 1) + BW * (ty + 1);
              force_ternary<AW, BW>(Am + AN, A0 + AN, Ap + AN, DipF4{ringB + ((itB + 2) % 3) * BN},
                                    DipF4{ringB + (itB % 3) * BN}, DipF4{ringB + ((itB + 1) % 3) * BN},
                                    as, bs, Lg, psi0, reinterpret_cast<float(*)[3]>(Fx));
            } else {
              // ---- binary Shan-Chen force with walls, :127-210
              force_binary<AW, ROCK>(Am, A0, Ap, as, nb, RK, Lg, psi0,
                                     reinterpret_cast<float(*)[3]>(Fx));
            }
            // ---- pass 1: moments of the own post-stream populations (the
            // pulls hit L2: stage A fetched them H planes earlier)
            float dr[NC], j[NC][3];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              float d[19];
              pull_comp<ROCK>(F, S, c, nb, self, RK, d);
              own_moments<1>(d, dr[c], j[c][0], j[c][1], j[c][2]);
            }
            float rho[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) rho[c] = rho0 + dr[c];
            if (BODY) {
              const int x1 = gx + 1, y1 = gy + 1, z1 = gz + 1;
              bool on;
              if (Lg.inv_fluid == 9)
                on = (z1 == 1) || (z1 == nz);
              else if (Lg.inv_fluid == 20 || Lg.inv_fluid == 21)
                on = z1 == 1;
              else
                on = z1 >= Lg.amin_z && z1 <= Lg.amax_z && x1 >= Lg.amin_x && x1 <= Lg.amax_x &&
                     y1 >= Lg.amin_y && y1 <= Lg.amax_y;
              if (on) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                  const float m = Lg.amass[c] * rho[c];
                  Fx[c][0] = fmaf(m, Lg.g_accn_x, Fx[c][0]);
                  Fx[c][1] = fmaf(m, Lg.g_accn_y, Fx[c][1]);
                  Fx[c][2] = fmaf(m, Lg.g_accn, Fx[c][2]);
                }
              }
            }
            // common velocity u~ (code/lb3d_collision.F90:560-587)
            float p0 = 0.f, p1 = 0.f, p2 = 0.f, rt = 0.f;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              const float am = Lg.amass[c] * Lg.omega[c];
              p0 = fmaf(am, j[c][0], p0);
              p1 = fmaf(am, j[c][1], p1);
              p2 = fmaf(am, j[c][2], p2);
              rt = fmaf(am, rho[c], rt);
            }
            const float irt = 1.0f / fmaxf(rt, 1.0e-8f);
            const float u0 = p0 * irt, u1 = p1 * irt, u2 = p2 * irt;
            // ---- pass 2: reload, relax, store
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              // du = tau F / (amass max(rho, 1e-8))  (:523-556)
              const float k = Lg.tau[c] / (Lg.amass[c] * fmaxf(rho[c], 1.0e-8f));
              float d[19];
              pull_comp<ROCK, true>(F, S, c, nb, self, RK, d);
              bgk_update(d, rho[c], dr[c], fmaf(k, Fx[c][0], u0), fmaf(k, Fx[c][1], u1),
                         fmaf(k, Fx[c][2], u2), Lg.omega[c]);
              float *fo = Fo + (size_t)(c * 19) * S + self;
              // streaming stores: the new populations are not read again in
              // this launch, so they should not displace the inputs from L2
#pragma unroll
              for (int q = 0; q < 19; ++q) __stcs(fo + q * S, d[q]);
            }
          }
        }
      }
      __syncthreads();
    }
  }
}

#include "fp32_split.cuh"
#include "fp32_mfield.cuh"

__global__ void k_flip(LatDesc *lats, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && (lats[i].flags & LAT_ACTIVE)) lats[i].parity ^= 1;
}

// FP32 state -> FP64 populations n = delta + w rho0 (dumps, reductions).
// The products and sums are rounded separately (no contraction), as the
// host-side conversions of the ensemble do, so both routes agree bit for bit.
__global__ void k_to_fp64(const float *__restrict__ f, double *__restrict__ n, long long S,
                          long long base, long long N, int nc, double rho0) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int c = 0; c < nc; ++c)
    for (int q = 0; q < 19; ++q)
      n[((long long)c * 19 + q) * N + i] =
          __dadd_rn((double)f[((long long)c * 19 + q) * S + base + i],
                    __dmul_rn(q == 18 ? 1.0 / 3.0 : 1.0 / 36.0, rho0));
}

// FP64 populations -> FP32 deviations (upload); rock sites (rock[i] != 0,
// when rock is given) hold n = 0.
__global__ void k_from_fp64(const double *__restrict__ n, float *__restrict__ f, long long S,
                            long long base, long long N, int nc, double rho0,
                            const uint8_t *__restrict__ rock = nullptr) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const bool solid = rock && rock[i] != 0;
  for (int c = 0; c < nc; ++c)
    for (int q = 0; q < 19; ++q) {
      const double w = __dmul_rn(q == 18 ? 1.0 / 3.0 : 1.0 / 36.0, rho0);
      const double v = solid ? 0.0 : n[((long long)c * 19 + q) * N + i];
      f[((long long)c * 19 + q) * S + base + i] = (float)__dsub_rn(v, w);
    }
}

// One population plane FP64 <-> FP32 deviations (w = w_q rho0), rounded as
// k_to_fp64 / k_from_fp64; the upload writes both buffers.
__global__ void k_plane_from_fp64(const double *__restrict__ src, float *__restrict__ d0,
                                  float *__restrict__ d1, long long N, double w,
                                  const uint8_t *__restrict__ rock) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double v = (rock && rock[i] != 0) ? 0.0 : src[i];
  const float x = (float)__dsub_rn(v, w);
  d0[i] = x;
  d1[i] = x;
}
__global__ void k_plane_to_fp64(const float *__restrict__ src, double *__restrict__ dst, long long N,
                                double w) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  dst[i] = __dadd_rn((double)src[i], w);
}

}  // namespace f32

using namespace f32;

cudaError_t fp32_to_fp64(const float *f, double *out, long long S, long long base, long long N,
                         int nc, double rho0, cudaStream_t st) {
  if (N <= 0) return cudaSuccess;
  k_to_fp64<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(f, out, S, base, N, nc, rho0);
  return cudaGetLastError();
}

__global__ void k_planes_f2d(const float *__restrict__ src, double *__restrict__ dst, long long S,
                             long long base, long long N, int planes) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int k = 0; k < planes; ++k) dst[(long long)k * N + i] = (double)src[(long long)k * S + base + i];
}

cudaError_t fp32_planes_to_fp64(const float *src, double *dst, long long S, long long base,
                                long long N, int planes, cudaStream_t st) {
  if (N <= 0) return cudaSuccess;
  k_planes_f2d<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(src, dst, S, base, N, planes);
  return cudaGetLastError();
}

cudaError_t fp32_from_fp64(const double *n, float *f, long long S, long long base, long long N,
                           int nc, double rho0, const uint8_t *rock, cudaStream_t st) {
  if (N <= 0) return cudaSuccess;
  k_from_fp64<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(n, f, S, base, N, nc, rho0, rock);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launch table
// ---------------------------------------------------------------------------
constexpr int MODE_DIPOLE = 3, MODE_COLLIDE2 = 4;
// the moments pass with 32-bit component offsets (k_fused<..., NARROW>)
constexpr int MODE_MOMENTS32 = 5;

size_t fp32_mode_smem(int nc, const FusedShape &sh, int mode) {
  if (mode == MODE_MOMENTS32) mode = MODE_MOMENTS;
  const size_t AN1 = (size_t)(sh.tx + 2) * (sh.ty + 2);
  if (mode == MODE_DIPOLE) return 16 * 5 * AN1 + (size_t)4 * 5 * sh.tx * sh.ty;
  if (mode == MODE_COLLIDE2)  // Collide2Geom: ring slots x entry bytes + population stage
    return 5 * AN1 * (nc == 3 ? 16 + 12 : 8) + (size_t)19 * nc * sh.tx * sh.ty * 4;
  if (mode == MODE_COLLIDE) return 16 * 3 * AN1 * (nc == 3 ? 2 : 1);
  const int H = mode == MODE_MOMENTS ? 0 : (nc == 3 ? 2 : 1);
  const int dh = mode == MODE_MOMENTS ? 1 : 3;
  const size_t AN = (size_t)(sh.tx + 2 * H) * (sh.ty + 2 * H);
  const size_t BN = (size_t)(sh.tx + 2) * (sh.ty + 2);
  const size_t DN = (size_t)(sh.tx + 2 * dh) * (sh.ty + 2 * dh);
  size_t f4 = 0;
  if (mode != MODE_MOMENTS) f4 += (nc == 3 ? 4 * 2 : 3) * AN;
  if (nc == 3 && mode != MODE_MOMENTS) f4 += 3 * BN;
  if (nc == 3) f4 += 3 * DN;
  return 16 * f4;
}
size_t fp32_fused_smem(int nc, const FusedShape &sh) { return fp32_mode_smem(nc, sh, MODE_FUSED); }

template <int NC, int TX, int TY, bool ROCK, bool BODY, int MODE, bool LE, bool INF = false>
static const void *fused_ptr() {
  if constexpr (MODE == MODE_COLLIDE)
    return (const void *)k_split_collide<NC, TX, TY, ROCK, BODY>;
  else if constexpr (MODE == MODE_COLLIDE2)
    return (const void *)k_split_collide2<NC, TX, TY, ROCK, BODY, LE, INF>;
  else if constexpr (MODE == MODE_DIPOLE)
    return (const void *)k_split_dipole<TX, TY>;
  else if constexpr (MODE == MODE_MOMENTS32)
    return (const void *)k_fused<NC, TX, TY, ROCK, BODY, MODE_MOMENTS, LE, true>;
  else
    return (const void *)k_fused<NC, TX, TY, ROCK, BODY, MODE, LE>;
}

// LE: the Lees-Edwards variants, built for binary lattices without rock and
// only for the moments and staged collide passes (strategy 2).
// INF: the staged collide variant with the stage-8 inflow boundaries.
template <int MODE, bool LE = false, bool INF = false>
static const void *mode_fn(int nc, bool rock, bool body, const FusedShape &sh) {
#define LB3D_SHAPES(NC, R, B)                                                            \
  if (sh.tx == 32 && sh.ty == 8) return fused_ptr<NC, 32, 8, R, B, MODE, LE, INF>();     \
  if (sh.tx == 32 && sh.ty == 4) return fused_ptr<NC, 32, 4, R, B, MODE, LE, INF>();     \
  if (sh.tx == 16 && sh.ty == 16) return fused_ptr<NC, 16, 16, R, B, MODE, LE, INF>();   \
  if (sh.tx == 16 && sh.ty == 8) return fused_ptr<NC, 16, 8, R, B, MODE, LE, INF>();     \
  if (sh.tx == 64 && sh.ty == 4) return fused_ptr<NC, 64, 4, R, B, MODE, LE, INF>();
  // the moments and dipole passes do not apply the body force
  if (MODE == MODE_MOMENTS || MODE == MODE_MOMENTS32 || MODE == MODE_DIPOLE) body = false;
  if constexpr (LE) {
    static_assert(MODE == MODE_MOMENTS || MODE == MODE_MOMENTS32 || MODE == MODE_COLLIDE2,
                  "no Lees-Edwards variant");
    if (nc != 2) return nullptr;
    if (rock) {
      if (body) { LB3D_SHAPES(2, true, true) } else { LB3D_SHAPES(2, true, false) }
    } else {
      if (body) { LB3D_SHAPES(2, false, true) } else { LB3D_SHAPES(2, false, false) }
    }
    return nullptr;
  }
  if (MODE == MODE_DIPOLE) rock = false;
  if (nc == 3) {
    if (body) { LB3D_SHAPES(3, false, true) } else { LB3D_SHAPES(3, false, false) }
  } else {
    if (MODE == MODE_DIPOLE) return nullptr;
    if (rock) {
      if (body) { LB3D_SHAPES(2, true, true) } else { LB3D_SHAPES(2, true, false) }
    } else {
      if (body) { LB3D_SHAPES(2, false, true) } else { LB3D_SHAPES(2, false, false) }
    }
  }
#undef LB3D_SHAPES
  return nullptr;
}

static const void *kernel_fn(int nc, bool rock, bool body, const FusedShape &sh, int mode,
                             bool le = false, bool inf = false) {
  if (inf && mode == MODE_COLLIDE2) return mode_fn<MODE_COLLIDE2, false, true>(nc, rock, body, sh);
  if (le) {
    if (mode == MODE_MOMENTS) return mode_fn<MODE_MOMENTS, true>(nc, rock, body, sh);
    if (mode == MODE_MOMENTS32) return mode_fn<MODE_MOMENTS32, true>(nc, rock, body, sh);
    if (mode == MODE_COLLIDE2) return mode_fn<MODE_COLLIDE2, true>(nc, rock, body, sh);
    return nullptr;
  }
  if (mode == MODE_MOMENTS) return mode_fn<MODE_MOMENTS>(nc, rock, body, sh);
  if (mode == MODE_MOMENTS32) return mode_fn<MODE_MOMENTS32>(nc, rock, body, sh);
  if (mode == MODE_COLLIDE) return mode_fn<MODE_COLLIDE>(nc, rock, body, sh);
  if (mode == MODE_DIPOLE) return mode_fn<MODE_DIPOLE>(nc, rock, body, sh);
  if (mode == MODE_COLLIDE2) return mode_fn<MODE_COLLIDE2>(nc, rock, body, sh);
  return mode_fn<MODE_FUSED>(nc, rock, body, sh);
}
static const void *fused_fn(int nc, bool rock, bool body, const FusedShape &sh) {
  return kernel_fn(nc, rock, body, sh, MODE_FUSED);
}

static int mode_ctas_per_sm(int nc, bool rock, bool body, const FusedShape &sh, int mode) {
  const void *fn = kernel_fn(nc, rock, body, sh, mode);
  if (!fn) return 0;
  size_t smem = fp32_mode_smem(nc, sh, mode);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, sh.tx * sh.ty, smem) != cudaSuccess) return 0;
  return n;
}

int fp32_fused_ctas_per_sm(int nc, bool rock, bool body, const FusedShape &sh) {
  int a = mode_ctas_per_sm(nc, rock, body, sh,
                           sh.split == 2 ? MODE_COLLIDE2 : (sh.split ? MODE_COLLIDE : MODE_FUSED));
  if (!sh.split) return a;
  int b = mode_ctas_per_sm(nc, rock, body, sh, MODE_MOMENTS);
  int c = nc == 3 ? mode_ctas_per_sm(nc, rock, body, sh, MODE_DIPOLE) : b;
  return std::min(a, std::min(b, c));
}

// Grid of one pass: as many CTAs as are resident at once (up to the tile
// count), from the pass's own occupancy, so a pass with a large shared
// memory stage does not throttle the others.  The dynamic shared memory
// attribute and the occupancy are set up once per kernel and device.
static cudaError_t prepare_kernel(const void *fn, int nthreads, size_t smem, int *ctas_total) {
  static std::mutex mu;
  static std::map<std::tuple<const void *, size_t, int, int>, int> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const auto key = std::make_tuple(fn, smem, nthreads, dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) {
    *ctas_total = it->second;
    return cudaSuccess;
  }
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per = 0, nsm = 148;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, nthreads, smem);
  if (e != cudaSuccess) return e;
  if (per < 1) return cudaErrorInvalidConfiguration;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cache[key] = *ctas_total = per * nsm;
  return cudaSuccess;
}

static cudaError_t launch_mode(int mode, int nc, bool rock, bool body, const FusedShape &sh,
                               const LatDesc *d_lat, const Tile *d_tiles, int ntiles, int max_grid,
                               float *f0, float *f1, float *db0, float *db1, const uint8_t *rockp,
                               unsigned S, float4 *M, float4 *J, cudaStream_t st, bool le = false,
                               bool inf = false) {
  if (mode == MODE_MOMENTS && 19ull * nc * S < (1ull << 32)) mode = MODE_MOMENTS32;
  const void *fn = kernel_fn(nc, rock, body, sh, mode, le, inf);
  if (!fn) return cudaErrorInvalidConfiguration;
  size_t smem = fp32_mode_smem(nc, sh, mode);
  int resident = 0;
  cudaError_t e = prepare_kernel(fn, sh.tx * sh.ty, smem, &resident);
  if (e != cudaSuccess) return e;
  int grid = std::max(1, std::min(ntiles, resident));
  if (max_grid > 0) grid = std::min(grid, max_grid);
  if (mode == MODE_DIPOLE) {
    const float4 *Mc = M;
    void *args[] = {(void *)&d_lat, (void *)&d_tiles, (void *)&ntiles, (void *)&db0, (void *)&db1,
                    (void *)&Mc, (void *)&S};
    return cudaLaunchKernel(fn, dim3(grid), dim3(sh.tx * sh.ty), args, smem, st);
  }
  if (mode == MODE_COLLIDE2) {
    const float4 *Mc = M;
    void *args[] = {(void *)&d_lat, (void *)&d_tiles, (void *)&ntiles, (void *)&f0, (void *)&f1,
                    (void *)&db0, (void *)&db1, (void *)&rockp, (void *)&S, (void *)&Mc};
    return cudaLaunchKernel(fn, dim3(grid), dim3(sh.tx * sh.ty), args, smem, st);
  }
  if (mode == MODE_COLLIDE) {
    const float4 *Mc = M, *Jc = J;
    void *args[] = {(void *)&d_lat, (void *)&d_tiles, (void *)&ntiles, (void *)&f0, (void *)&f1,
                    (void *)&db0, (void *)&db1, (void *)&rockp, (void *)&S, (void *)&Mc, (void *)&Jc};
    return cudaLaunchKernel(fn, dim3(grid), dim3(sh.tx * sh.ty), args, smem, st);
  }
  void *args[] = {(void *)&d_lat, (void *)&d_tiles, (void *)&ntiles, (void *)&f0, (void *)&f1,
                  (void *)&db0, (void *)&db1, (void *)&rockp, (void *)&S, (void *)&M, (void *)&J};
  return cudaLaunchKernel(fn, dim3(grid), dim3(sh.tx * sh.ty), args, smem, st);
}

cudaError_t fp32_launch_fused(int nc, bool rock, bool body, const FusedShape &sh,
                              const LatDesc *d_lat, const Tile *d_tiles, int ntiles, int max_grid,
                              float *f0, float *f1, float *db0, float *db1, const uint8_t *rockp,
                              long long S64, cudaStream_t st, float4 *M, float4 *J,
                              const LEStep *le, const DevParams *P) {
  if (S64 * 19 >= (1LL << 32)) return cudaErrorInvalidValue;
  const unsigned S = (unsigned)S64;
  if (le) {
    // stage 6 halo, moments pass, stage 8 halo, staged collide pass
    if (!P || nc != 2 || sh.split != 2 || !M) return cudaErrorInvalidValue;
    // two threads per (y, z) of the x-halo planes (one per side): 64-thread
    // blocks spread the few thousand threads over every SM
    const unsigned g = (unsigned)((2 * P->ny * P->nz + 63) / 64);
    k_le_pre32<2><<<g, 64, 0, st>>>(*P, *le, d_lat, f0, f1, S);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = launch_mode(MODE_MOMENTS, nc, rock, body, sh, d_lat, d_tiles, ntiles, max_grid, f0, f1, db0,
                      db1, rockp, S, M, nullptr, st, true);
    if (e != cudaSuccess) return e;
    k_le_post32<2><<<g, 64, 0, st>>>(*P, *le, d_lat, f0, f1, S);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_mode(MODE_COLLIDE2, nc, rock, body, sh, d_lat, d_tiles, ntiles, max_grid, f0, f1,
                       db0, db1, rockp, S, M, nullptr, st, true);
  }
  // lattices with inflow boundaries run the staged collide's inflow variant
  const bool inf = P && P->invk != 0;
  if (inf && sh.split != 2) return cudaErrorInvalidValue;
  if (!sh.split)
    return launch_mode(MODE_FUSED, nc, rock, body, sh, d_lat, d_tiles, ntiles, max_grid, f0, f1, db0,
                       db1, rockp, S, nullptr, nullptr, st);
  if (!M || (sh.split == 1 && !J)) return cudaErrorInvalidValue;
  // strategy 2 recomputes the own moments in the collide pass: no J field
  if (sh.split == 2) J = nullptr;
  cudaError_t e = launch_mode(MODE_MOMENTS, nc, rock, body, sh, d_lat, d_tiles, ntiles, max_grid, f0,
                              f1, db0, db1, rockp, S, M, J, st);
  if (e == cudaSuccess && nc == 3)
    e = launch_mode(MODE_DIPOLE, nc, rock, body, sh, d_lat, d_tiles, ntiles, max_grid, f0, f1, db0,
                    db1, rockp, S, M, J, st);
  if (e != cudaSuccess) return e;
  return launch_mode(sh.split == 2 ? MODE_COLLIDE2 : MODE_COLLIDE, nc, rock, body, sh, d_lat,
                     d_tiles, ntiles, max_grid, f0, f1, db0, db1, rockp, S, M, J, st, false, inf);
}

cudaError_t fp32_flip_parity(LatDesc *d_lat, int nlat, cudaStream_t st) {
  k_flip<<<(nlat + 127) / 128, 128, 0, st>>>(d_lat, nlat);
  return cudaGetLastError();
}

void fp32_tiles_for(const LatDesc &L, int lat_id, const FusedShape &sh, std::vector<Tile> &out) {
  const int zc = std::min(sh.zc, L.nz);
  for (int z0 = 0; z0 < L.nz; z0 += zc)
    for (int y0 = 0; y0 < L.ny; y0 += sh.ty)
      for (int x0 = 0; x0 < L.nx; x0 += sh.tx) {
        Tile t;
        t.lat = lat_id;
        t.x0 = (short)x0;
        t.y0 = (short)y0;
        t.z0 = (short)z0;
        t.zc = (short)std::min(zc, L.nz - z0);
        out.push_back(t);
      }
}

LatDesc fp32_make_desc(const DevParams &P, double rho0, long long base, bool rock) {
  LatDesc L{};
  L.nx = P.nx;
  L.ny = P.ny;
  L.nz = P.nz;
  L.nc = P.nc;
  L.base = base;
  L.parity = 0;
  for (int c = 0; c < 3; ++c) {
    L.omega[c] = (float)P.omega[c];
    L.tau[c] = (float)P.tau[c];
    L.amass[c] = (float)P.amass[c];
  }
  L.g_br = (float)P.g_br;
  L.g_bs = (float)P.g_bs;
  L.g_ss = (float)P.g_ss;
  L.wall_r = (float)(-P.g_wr * P.tau_wr / P.tau[0]);
  L.wall_b = (float)(-P.g_wb * P.tau_wb / P.tau[1]);
  L.psiw_r = (float)(1.0 - std::exp(-P.rc_r));
  L.psiw_b = (float)(1.0 - std::exp(-P.rc_b));
  L.beta = (float)P.beta;
  L.d0 = (float)P.d_0;
  L.omega_d = (float)P.omega_d;
  L.g_accn = (float)P.g_accn;
  L.g_accn_x = (float)P.g_accn_x;
  L.g_accn_y = (float)P.g_accn_y;
  L.amin_x = P.g_accn_min_x;
  L.amax_x = P.g_accn_max_x;
  L.amin_y = P.g_accn_min_y;
  L.amax_y = P.g_accn_max_y;
  L.amin_z = P.g_accn_min;
  L.amax_z = P.g_accn_max;
  L.inv_fluid = P.inv_fluid;
  L.invk = P.invk;
  L.inv_type = P.inv_type;
  L.zh_in[0] = (float)P.zh_in[0];
  L.zh_in[1] = (float)P.zh_in[1];
  for (int c = 0; c < 3; ++c) L.zh_uz[c] = (float)P.zh_uz[c];
  L.rho0 = (float)rho0;
  L.em0 = (float)std::exp(-rho0);
  L.psi0 = (float)(1.0 - std::exp(-rho0));
  bool body = (P.g_accn != 0.0 || P.g_accn_x != 0.0 || P.g_accn_y != 0.0);
  L.flags = LAT_ACTIVE | (rock ? LAT_ROCK : 0) | (body ? LAT_BODY : 0);
  return L;
}

// ---------------------------------------------------------------------------
// single-lattice handle
// ---------------------------------------------------------------------------
long long fp32_footprint(const lb3dc_params &p) {
  const long long N = (long long)p.nx * p.ny * p.nz;
  const bool le = p.boundary_cond != 0 && (p.inv_fluid == 5 || p.inv_fluid == 6);
  const long long np = (long long)p.ny * p.nz;
  // the moment field of strategy 3 when every component relaxes fully
  const bool full = p.tau_r == 1.0 && p.tau_b == 1.0 && (p.ncomp == 2 || p.tau_s == 1.0);
  const long long mf = full ? (long long)(p.nx + 2 * MF_PAD) * (p.ny + 2 * MF_PAD) * p.nz *
                                             (p.ncomp == 3 ? 48 : 16) + N * 12
                                   : 0;
  return 2LL * p.ncomp * 19 * N * 4 + (p.ncomp == 3 ? 6LL * N * 4 : 0) +
         N * fp32_moment_bytes(p.ncomp) + mf +
         (le ? 2 * np * (p.ncomp * 19 * 4 + 8) + 4 * np * p.ncomp * 19 * 4 : 0) + N * 16 + 4096;
}

// ---------------------------------------------------------------------------
// moment-field strategy (split 3): eligibility, field, tensor maps, launches
// ---------------------------------------------------------------------------
bool fp32_mf_eligible(const DevParams &P) {
  if ((P.le && P.nc != 2) || P.invk) return false;
  for (int c = 0; c < P.nc; ++c)
    if (P.omega[c] != 1.0) return false;
  if (P.nx < 2 || P.ny < 2) return false;
  return (long long)(P.nx + 2 * MF_PAD) * (P.ny + 2 * MF_PAD) * P.nz < (1LL << 31);
}

long long fp32_mf_bytes(const DevParams &P) {
  return (long long)(P.nx + 2 * MF_PAD) * (P.ny + 2 * MF_PAD) * P.nz * (P.nc == 3 ? 48 : 16) +
         P.nsites * (P.nc == 3 ? 12 : 8) + 64;
}

static int ensure_mf(const DevParams &P, Fp32State &s, cudaStream_t st) {
  if (s.MF1) return LB3DC_OK;
  const size_t plane = (size_t)(P.nx + 2 * MF_PAD) * (P.ny + 2 * MF_PAD) * P.nz * sizeof(float4);
  bool ok = cudaMalloc(&s.MF1, plane) == cudaSuccess;
  if (ok && P.nc == 3) ok = cudaMalloc(&s.MF2, plane) == cudaSuccess;
  if (ok && P.nc == 3) ok = cudaMalloc(&s.DD, plane) == cudaSuccess;
  if (ok) ok = cudaMalloc(&s.MFp, (size_t)P.nsites * sizeof(float2)) == cudaSuccess;
  if (ok && P.nc == 3) ok = cudaMalloc(&s.DS, (size_t)P.nsites * sizeof(float)) == cudaSuccess;
  if (ok && !s.err) ok = cudaMalloc(&s.err, sizeof(int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    if (s.MF1) cudaFree(s.MF1);
    if (s.MF2) cudaFree(s.MF2);
    if (s.DD) cudaFree(s.DD);
    if (s.MFp) cudaFree(s.MFp);
    if (s.DS) cudaFree(s.DS);
    s.MF1 = s.MF2 = s.DD = nullptr;
    s.MFp = nullptr;
    s.DS = nullptr;
    return LB3DC_ENOMEM;
  }
  // padding entries that no site writes are read only by inactive lanes
  cudaMemsetAsync(s.MF1, 0, plane, st);
  if (s.MF2) cudaMemsetAsync(s.MF2, 0, plane, st);
  if (s.DD) cudaMemsetAsync(s.DD, 0, plane, st);
  cudaMemsetAsync(s.err, 0, sizeof(int), st);
  s.bytes += (long long)plane * (P.nc == 3 ? 3 : 1) + P.nsites * (P.nc == 3 ? 12 : 8);
  return LB3DC_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// A padded float4 field as a 4-D FP32 tensor {component 0..3, padded x,
// padded y, z}; one box is the tile plus one halo site in x and y, one plane
// deep.
static int encode_mf_map(CUtensorMap *m, float4 *base, const DevParams &P, int tx, int ty) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return LB3DC_ECUDA;
  const cuuint64_t XP = (cuuint64_t)P.nx + 2 * MF_PAD, YP = (cuuint64_t)P.ny + 2 * MF_PAD;
  const cuuint64_t dims[4] = {4, XP, YP, (cuuint64_t)P.nz};
  const cuuint64_t strides[3] = {16, 16 * XP, 16 * XP * YP};
  const cuuint32_t box[4] = {4, (cuuint32_t)(tx + 2), (cuuint32_t)(ty + 2), 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LB3DC_OK : LB3DC_ECUDA;
}

template <int NC, int TX, int TY, bool ROCK, bool BODY, bool LE>
static void mf_ptrs(bool narrow, const void **mom, const void **dip, const void **col) {
  *mom = narrow ? (const void *)k_mf_moments<NC, TX, TY, ROCK, true, LE>
                : (const void *)k_mf_moments<NC, TX, TY, ROCK, false, LE>;
  *dip = NC == 3 ? (const void *)k_mf_dipole<TX, TY> : nullptr;
  *col = (const void *)k_mf_collide<NC, TX, TY, ROCK, BODY, LE>;
}
// The kernels of strategy 3 for a lattice kind and tile shape (false if the
// shape is not compiled); dip is null for binary lattices.  The
// Lees-Edwards variants exist for binary lattices without walls.
static bool mf_fns(int nc, bool rock, bool body, int tx, int ty, bool narrow, const void **mom,
                   const void **dip, const void **col, bool le = false) {
#define LB3D_MF(NC, R, B, L)                                                                   \
  if (tx == 32 && ty == 8) return mf_ptrs<NC, 32, 8, R, B, L>(narrow, mom, dip, col), true;   \
  if (tx == 32 && ty == 4) return mf_ptrs<NC, 32, 4, R, B, L>(narrow, mom, dip, col), true;   \
  if (tx == 16 && ty == 16) return mf_ptrs<NC, 16, 16, R, B, L>(narrow, mom, dip, col), true; \
  if (tx == 16 && ty == 8) return mf_ptrs<NC, 16, 8, R, B, L>(narrow, mom, dip, col), true;   \
  if (tx == 64 && ty == 4) return mf_ptrs<NC, 64, 4, R, B, L>(narrow, mom, dip, col), true;
  if (le) {
    if (nc != 2) return false;
    if (rock) {
      if (body) { LB3D_MF(2, true, true, true) } else { LB3D_MF(2, true, false, true) }
    } else {
      if (body) { LB3D_MF(2, false, true, true) } else { LB3D_MF(2, false, false, true) }
    }
    return false;
  }
  if (nc == 3) {
    if (rock) return false;
    if (body) { LB3D_MF(3, false, true, false) } else { LB3D_MF(3, false, false, false) }
  } else if (rock) {
    if (body) { LB3D_MF(2, true, true, false) } else { LB3D_MF(2, true, false, false) }
  } else {
    if (body) { LB3D_MF(2, false, true, false) } else { LB3D_MF(2, false, false, false) }
  }
#undef LB3D_MF
  return false;
}
// Dynamic shared memory of pass `which` (0 moments, 1 dipole, 2 collide);
// mirrors MfGeom.
static size_t mf_smem(int nc, int tx, int ty, int which) {
  const size_t an = (size_t)(tx + 2) * (ty + 2), field = (16 * an + 127) / 128 * 128;
  if (which == 0) return nc == 3 ? 4 * an * 16 : 0;
  if (which == 1) return 8 * ((field + 1023) / 1024 * 1024) + 1024;
  const size_t slot = ((nc == 3 ? 2 : 1) * field + 1023) / 1024 * 1024;
  return 8 * slot + 4 * an * 8 + 1024;
}

// One step of strategy 3: the moments pass, (ternary) the dipole pass and the
// collide pass, each on its own tile list and resident grid; with le (a
// binary Lees-Edwards lattice) the stage-6 halo kernel runs before the
// moments pass and the stage-8 one before the collide pass.
// One pass of strategy 3, launched with programmatic stream serialization
// (pdl): its CTAs may start while the previous kernel on the stream
// finishes, and wait for it before reading its results (pdl_wait_previous).
// Lattices with rock launch plainly (the overlap measured 0.8 % slower on
// the porous lattice, 0.9-1 % faster on the periodic and sheared ones).
static cudaError_t launch_pdl(const void *fn, dim3 grid, dim3 block, void **args, size_t smem,
                              cudaStream_t st, bool pdl) {
  if (!pdl) return cudaLaunchKernel(fn, grid, block, args, smem, st);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

static cudaError_t launch_mf(const DevParams &P, Fp32State &s, const uint8_t *rockp, cudaStream_t st,
                             const LEStep *le) {
  const bool rock = (s.lat.flags & LAT_ROCK) != 0, body = (s.lat.flags & LAT_BODY) != 0;
  const unsigned S = (unsigned)s.S;
  const bool narrow = 19ull * P.nc * s.S < (1ull << 32);
  const void *fn[3] = {nullptr, nullptr, nullptr};
  if (!mf_fns(P.nc, rock, body, s.tx, s.ty, narrow, &fn[0], &fn[1], &fn[2], le != nullptr))
    return cudaErrorInvalidConfiguration;
  if (le && !s.le_h[0]) return cudaErrorInvalidValue;
  const unsigned leg = (unsigned)((2 * P.ny * P.nz + 63) / 64);  // two threads per (y, z)
  if (s.mf_tx != s.tx || s.mf_ty != s.ty || !s.mf_tiles) return cudaErrorInvalidConfiguration;
  const int nt = s.tx * s.ty;
  const LatDesc *dl = s.d_lat;
  cudaError_t e = cudaSuccess;
  for (int pass = 0; pass < 3 && e == cudaSuccess; ++pass) {
    if (!fn[pass]) continue;
    if (le && pass == 0) {
      k_le_pre32<2><<<leg, 64, 0, st>>>(P, *le, dl, s.f[0], s.f[1], S);
      if ((e = cudaGetLastError()) != cudaSuccess) break;
    }
    if (le && pass == 2) {
      k_le_post32<2><<<leg, 64, 0, st>>>(P, *le, dl, s.f[0], s.f[1], S);
      if ((e = cudaGetLastError()) != cudaSuccess) break;
    }
    const size_t sm = mf_smem(P.nc, s.tx, s.ty, pass);
    int res = 0;
    if ((e = prepare_kernel(fn[pass], nt, sm, &res)) != cudaSuccess) break;
    const Tile *dt = s.mf_tiles + s.mf_off[pass];
    int ntl = s.mf_ntiles[pass];
    const dim3 grid(std::max(1, std::min(ntl, res)));
    if (pass == 0) {
      const float *f0 = s.f[0], *f1 = s.f[1], *d0 = s.db[0], *d1 = s.db[1];
      void *args[] = {(void *)&dl, (void *)&dt, (void *)&ntl, (void *)&f0, (void *)&f1, (void *)&d0,
                      (void *)&d1, (void *)&rockp, (void *)&S, (void *)&s.MF1, (void *)&s.MF2,
                      (void *)&s.MFp, (void *)&s.DS};
      e = launch_pdl(fn[pass], grid, dim3(nt), args, sm, st, !rock);
    } else if (pass == 1) {
      const float *ds = s.DS;
      void *args[] = {(void *)&s.tm2, (void *)&dl, (void *)&dt, (void *)&ntl, (void *)&s.db[0],
                      (void *)&s.db[1], (void *)&ds, (void *)&s.DD, (void *)&s.err};
      e = launch_pdl(fn[pass], grid, dim3(nt), args, sm, st, !rock);
    } else {
      const float2 *mfp = s.MFp;
      void *args[] = {(void *)&s.tm1, (void *)&s.tmd, (void *)&dl, (void *)&dt, (void *)&ntl,
                      (void *)&s.f[0], (void *)&s.f[1], (void *)&s.db[0], (void *)&s.db[1], (void *)&rockp,
                      (void *)&S, (void *)&mfp, (void *)&s.err};
      e = launch_pdl(fn[pass], grid, dim3(nt), args, sm, st, !rock);
    }
  }
  return e;
}

// The z chunking of one pass of strategy 3: nxy column tiles, `resident`
// CTAs at once, `halo` planes each chunk reads beyond its own.  Chooses the
// number of chunks per column so that the tiles fill whole rounds of the
// resident grid (1 to 8 rounds), weighed against the halo planes that
// shorter chunks reload; the chunks of a column differ in length by at most
// one plane.
static int mf_chunks(int nz, int nxy, int resident, int halo) {
  int best = 1;
  double best_score = -1.0;
  for (int rounds = 1; rounds <= 8; ++rounds) {
    int k = std::min(nz, std::max(1, (int)((long long)rounds * resident / nxy)));
    const long long nt = (long long)nxy * k;
    const long long used = (nt + resident - 1) / resident * resident;
    const double zc = (double)nz / k;
    const double score = (double)nt / used * zc / (zc + halo);
    if (score > best_score + 1e-9) best_score = score, best = k;
  }
  return best;
}

static int mf_build_tiles(const DevParams &P, Fp32State &s, const FusedShape &sh, cudaStream_t st) {
  const void *fn[3];
  if (!mf_fns(P.nc, (s.lat.flags & LAT_ROCK) != 0, (s.lat.flags & LAT_BODY) != 0, sh.tx, sh.ty,
              19ull * P.nc * s.S < (1ull << 32), &fn[0], &fn[1], &fn[2], s.le_h[0] != nullptr))
    return LB3DC_EINVAL;
  const LatDesc &L = s.lat;
  const int nxt = (L.nx + sh.tx - 1) / sh.tx, nyt = (L.ny + sh.ty - 1) / sh.ty, nxy = nxt * nyt;
  std::vector<Tile> all;
  // planes a chunk reads beyond its own: the dipole and collide passes load
  // one field plane on each side; the moments pass counts one for the
  // dipole planes its ring loads ahead of its first plane
  const int halo[3] = {1, 2, 2};
  for (int pass = 0; pass < 3; ++pass) {
    s.mf_off[pass] = (int)all.size();
    s.mf_ntiles[pass] = 0;
    if (!fn[pass]) continue;
    int res = 0;
    if (prepare_kernel(fn[pass], sh.tx * sh.ty, mf_smem(P.nc, sh.tx, sh.ty, pass), &res) != cudaSuccess)
      return LB3DC_ECUDA;
    const int k = mf_chunks(L.nz, nxy, res, halo[pass]);
    for (int c = 0; c < k; ++c) {
      const int z0 = (int)((long long)L.nz * c / k), z1 = (int)((long long)L.nz * (c + 1) / k);
      for (int y0 = 0; y0 < L.ny; y0 += sh.ty)
        for (int x0 = 0; x0 < L.nx; x0 += sh.tx) {
          Tile t;
          t.lat = 0;
          t.x0 = (short)x0;
          t.y0 = (short)y0;
          t.z0 = (short)z0;
          t.zc = (short)(z1 - z0);
          all.push_back(t);
        }
    }
    s.mf_ntiles[pass] = (int)all.size() - s.mf_off[pass];
    s.mf_grid[pass] = std::min(s.mf_ntiles[pass], res);
  }
  if (s.mf_tiles) cudaFree(s.mf_tiles);
  s.mf_tiles = nullptr;
  if (cudaMalloc(&s.mf_tiles, all.size() * sizeof(Tile)) != cudaSuccess) return LB3DC_ENOMEM;
  if (cudaMemcpyAsync(s.mf_tiles, all.data(), all.size() * sizeof(Tile), cudaMemcpyHostToDevice, st) !=
      cudaSuccess)
    return LB3DC_ECUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? LB3DC_OK : LB3DC_ECUDA;
}

int fp32_take_error(Fp32State &s, cudaStream_t st) {
  if (!s.err) return LB3DC_OK;
  int v = 0;
  if (cudaMemcpyAsync(&v, s.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return LB3DC_ECUDA;
  if (v) cudaMemsetAsync(s.err, 0, sizeof(int), st);
  return v;
}

// Lees-Edwards lattices: the compact pre-stream boundary planes from the
// current state (after an upload or a restore; the collide passes keep them
// current from then on).
static cudaError_t le_gather(const DevParams &P, Fp32State &s, cudaStream_t st) {
  const long long n = (long long)P.nc * 19 * P.ny * P.nz;
  k_le_gather32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s.d_lat, s.f[0], s.f[1], (unsigned)s.S);
  return cudaGetLastError();
}

// The Lees-Edwards halo planes of a single lattice, referenced by its descriptor.
static void attach_le(Fp32State &s) {
  for (int b = 0; b < 2; ++b) {
    s.lat.le_h[b] = s.le_h[b];
    s.lat.le_p[b] = s.le_p[b];
  }
  for (int b = 0; b < 4; ++b) s.lat.le_b[b] = s.le_b[b];
}

// Shape before any autotuning: the split strategy with the staged collide
// pass, which measured fastest on 128^3 ternary and 256^3 binary lattices.
static FusedShape default_shape(const DevParams &P) {
  FusedShape sh{32, 4, P.nc == 3 ? 8 : 16, 2};
  if (P.nx < 32) sh.tx = 16, sh.ty = 8;
  return sh;
}

// The own-moment field J is read only by the plain split strategy (split 1);
// it is allocated the first time a lattice is switched to that strategy, so
// the other strategies hold no memory for it.
static int ensure_own(const DevParams &P, Fp32State &s) {
  if (s.J) return LB3DC_OK;
  const size_t b = (size_t)P.nsites * fp32_own_bytes(P.nc);
  if (cudaMalloc(&s.J, b) != cudaSuccess) {
    s.J = nullptr;
    cudaGetLastError();
    return LB3DC_ENOMEM;
  }
  s.bytes += (long long)b;
  return LB3DC_OK;
}

static int rebuild_tiles(const DevParams &P, Fp32State &s, const FusedShape &sh, cudaStream_t st) {
  if (sh.split == 1) {
    int rc = ensure_own(P, s);
    if (rc) return rc;
  }
  if (sh.split == 3) {
    if (!fp32_mf_eligible(P)) return LB3DC_ENOTSUP;
    const void *a, *b, *c;
    if (!mf_fns(P.nc, (s.lat.flags & LAT_ROCK) != 0, (s.lat.flags & LAT_BODY) != 0, sh.tx, sh.ty, true,
                &a, &b, &c, s.le_h[0] != nullptr))
      return LB3DC_EINVAL;
    int rc = ensure_mf(P, s, st);
    if (rc) return rc;
    if (s.mf_tx != sh.tx || s.mf_ty != sh.ty) {
      s.mf_tx = s.mf_ty = 0;
      if ((rc = encode_mf_map(&s.tm1, s.MF1, P, sh.tx, sh.ty)) != LB3DC_OK) return rc;
      if (P.nc == 3) {
        if ((rc = encode_mf_map(&s.tm2, s.MF2, P, sh.tx, sh.ty)) != LB3DC_OK) return rc;
        if ((rc = encode_mf_map(&s.tmd, s.DD, P, sh.tx, sh.ty)) != LB3DC_OK) return rc;
      } else {
        s.tm2 = s.tmd = s.tm1;  // unused by the binary kernels
      }
      s.mf_tx = sh.tx;
      s.mf_ty = sh.ty;
    }
    if ((rc = mf_build_tiles(P, s, sh, st)) != LB3DC_OK) return rc;
  }
  std::vector<Tile> tiles;
  fp32_tiles_for(s.lat, 0, sh, tiles);
  if (s.d_tiles) cudaFree(s.d_tiles);
  s.d_tiles = nullptr;
  if (cudaMalloc(&s.d_tiles, tiles.size() * sizeof(Tile)) != cudaSuccess) return LB3DC_ENOMEM;
  if (cudaMemcpyAsync(s.d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice,
                      st) != cudaSuccess)
    return LB3DC_ECUDA;
  s.ntiles = (int)tiles.size();
  s.tx = sh.tx;
  s.ty = sh.ty;
  s.zc = sh.zc;
  s.split = sh.split;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  bool rock = (s.lat.flags & LAT_ROCK) != 0, body = (s.lat.flags & LAT_BODY) != 0;
  if (sh.split == 3) {
    s.grid = s.ntiles;  // each pass sizes its own grid at launch
    return LB3DC_OK;
  }
  int per = fp32_fused_ctas_per_sm(P.nc, rock, body, sh);
  if (per < 1) return LB3DC_EINVAL;
  s.grid = std::min(s.ntiles, per * nsm);
  return LB3DC_OK;
}

int fp32_set_shape(const DevParams &P, Fp32State &s, const FusedShape &sh, cudaStream_t st) {
  if (!fused_fn(P.nc, false, false, sh)) return LB3DC_EINVAL;
  // Lees-Edwards lattices and lattices with inflow boundaries run the
  // staged split strategy only
  if ((s.le_h[0] && sh.split < 2) || (s.lat.invk && sh.split != 2)) return LB3DC_ENOTSUP;
  if (sh.split == 3 && !fp32_mf_eligible(P)) return LB3DC_ENOTSUP;
  if (sh.split && !s.M) return LB3DC_EINVAL;
  if (sh.split < 0 || sh.split > 3) return LB3DC_EINVAL;
  if (sh.zc < 1) return LB3DC_EINVAL;
  return rebuild_tiles(P, s, sh, st);
}

std::vector<FusedShape> fp32_candidate_shapes(const DevParams &P) {
  std::vector<FusedShape> out;
  const int xy[5][2] = {{32, 8}, {32, 4}, {16, 16}, {16, 8}, {64, 4}};
  const int zcs[3] = {8, 16, 32};
  for (auto &t : xy) {
    if (t[0] > 2 * P.nx && t[0] > 16) continue;
    for (int zc : zcs) {
      if (zc > P.nz && zc != 8) continue;
      for (int split = (P.le || P.invk) ? 2 : 0; split < 3; ++split)
        out.push_back(FusedShape{t[0], t[1], zc, split});
    }
  }
  // strategy 3 chunks z per pass from each pass's resident grid: one
  // candidate per tile shape (its zc is not used)
  if (fp32_mf_eligible(P)) {
    for (auto &t : xy) {
      if (t[0] > 2 * P.nx && t[0] > 16) continue;
      out.push_back(FusedShape{t[0], t[1], 16, 3});
    }
  }
  return out;
}

// The project's autotuner: time each candidate shape with CUDA events on a
// saved copy of the state, keep the fastest and restore the state.
int fp32_autotune(const DevParams &P, Fp32State &s, const uint8_t *rock, double *ms_out,
                  int *ntried, cudaStream_t st, const LEStep *le) {
  const size_t pop = (size_t)P.nc * 19 * s.S * sizeof(float);
  const size_t dbs = P.nc == 3 ? 3 * (size_t)s.S * sizeof(float) : 0;
  float *save = nullptr;
  if (cudaMalloc(&save, pop + dbs) != cudaSuccess) return LB3DC_ENOMEM;
  const int cur0 = s.lat.parity;
  cudaMemcpyAsync(save, s.f[cur0], pop, cudaMemcpyDeviceToDevice, st);
  if (dbs) cudaMemcpyAsync((char *)save + pop, s.db[cur0], dbs, cudaMemcpyDeviceToDevice, st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  FusedShape best{s.tx, s.ty, s.zc, s.split};
  float best_ms = 1e30f;
  KernelTimer *saved_timer = s.timer;
  s.timer = nullptr;
  int n = 0;
  for (const FusedShape &sh : fp32_candidate_shapes(P)) {
    if (rebuild_tiles(P, s, sh, st) != LB3DC_OK) continue;
    if (fp32_run(P, s, rock, 2, st, le) != LB3DC_OK) continue;
    cudaEventRecord(e0, st);
    const int reps = 5;
    if (fp32_run(P, s, rock, reps, st, le) != LB3DC_OK) continue;
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= reps;
    if (ms_out && n < 64) ms_out[n] = ms;
    ++n;
    if (ms < best_ms) {
      best_ms = ms;
      best = sh;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // restore the state into the buffer the lattice now reads from
  const int cur = s.lat.parity;
  cudaMemcpyAsync(s.f[cur], save, pop, cudaMemcpyDeviceToDevice, st);
  if (dbs) cudaMemcpyAsync(s.db[cur], (char *)save + pop, dbs, cudaMemcpyDeviceToDevice, st);
  if (s.le_b[0]) le_gather(P, s, st);
  cudaStreamSynchronize(st);
  cudaFree(save);
  if (ntried) *ntried = n;
  s.timer = saved_timer;
  int rc = rebuild_tiles(P, s, best, st);
  if (rc) return rc;
  return cudaStreamSynchronize(st) == cudaSuccess ? LB3DC_OK : LB3DC_ECUDA;
}

int fp32_alloc(const DevParams &P, const lb3dc_params &p, Fp32State &s, cudaStream_t st) {
  const long long N = P.nsites;
  s.S = N;
  const size_t pop = (size_t)P.nc * 19 * N * sizeof(float);
  for (int b = 0; b < 2; ++b) {
    if (cudaMalloc(&s.f[b], pop) != cudaSuccess) return LB3DC_ENOMEM;
    s.bytes += pop;
    cudaMemsetAsync(s.f[b], 0, pop, st);
    if (P.nc == 3) {
      if (cudaMalloc(&s.db[b], 3 * N * sizeof(float)) != cudaSuccess) return LB3DC_ENOMEM;
      s.bytes += 3 * N * sizeof(float);
      cudaMemsetAsync(s.db[b], 0, 3 * N * sizeof(float), st);
    }
  }
  if (cudaMalloc(&s.M, (size_t)N * fp32_moment_bytes(P.nc)) != cudaSuccess) return LB3DC_ENOMEM;
  s.bytes += N * fp32_moment_bytes(P.nc);
  if (cudaMalloc(&s.d_lat, sizeof(LatDesc)) != cudaSuccess) return LB3DC_ENOMEM;
  if (cudaMalloc(&s.stage, 2 * (size_t)N * sizeof(double)) != cudaSuccess) return LB3DC_ENOMEM;
  s.bytes += 2 * N * (long long)sizeof(double);
  if (cudaStreamCreateWithFlags(&s.xs, cudaStreamNonBlocking) != cudaSuccess) return LB3DC_ECUDA;
  for (int i = 0; i < 4; ++i)
    if (cudaEventCreateWithFlags(&s.xev[i], cudaEventDisableTiming) != cudaSuccess) return LB3DC_ECUDA;
  if (P.le) {
    const size_t np = (size_t)P.ny * P.nz;
    for (int b = 0; b < 2; ++b) {
      if (cudaMalloc(&s.le_h[b], (size_t)P.nc * 19 * np * sizeof(float)) != cudaSuccess ||
          cudaMalloc(&s.le_p[b], np * sizeof(float2)) != cudaSuccess)
        return LB3DC_ENOMEM;
      s.bytes += (long long)(P.nc * 19 * np * sizeof(float) + np * sizeof(float2));
    }
    for (int b = 0; b < 4; ++b) {
      if (cudaMalloc(&s.le_b[b], (size_t)P.nc * 19 * np * sizeof(float)) != cudaSuccess)
        return LB3DC_ENOMEM;
      s.bytes += (long long)(P.nc * 19 * np * sizeof(float));
    }
  }
  s.lat = fp32_make_desc(P, p.rho0 > 0 ? p.rho0 : 0.7, 0, false);
  attach_le(s);
  return rebuild_tiles(P, s, default_shape(P), st);
}

void fp32_free(Fp32State &s) {
  for (int b = 0; b < 2; ++b) {
    if (s.f[b]) cudaFree(s.f[b]);
    if (s.db[b]) cudaFree(s.db[b]);
    s.f[b] = s.db[b] = nullptr;
  }
  if (s.d_lat) cudaFree(s.d_lat);
  if (s.d_tiles) cudaFree(s.d_tiles);
  if (s.M) cudaFree(s.M);
  if (s.J) cudaFree(s.J);
  if (s.MF1) cudaFree(s.MF1);
  if (s.MF2) cudaFree(s.MF2);
  if (s.DD) cudaFree(s.DD);
  if (s.MFp) cudaFree(s.MFp);
  if (s.DS) cudaFree(s.DS);
  if (s.err) cudaFree(s.err);
  if (s.mf_tiles) cudaFree(s.mf_tiles);
  s.MF1 = s.MF2 = s.DD = nullptr;
  s.MFp = nullptr;
  s.DS = nullptr;
  s.mf_tiles = nullptr;
  s.err = nullptr;
  s.mf_tx = s.mf_ty = 0;
  if (s.stage) cudaFree(s.stage);
  s.stage = nullptr;
  for (int i = 0; i < 4; ++i) {
    if (s.xev[i]) cudaEventDestroy(s.xev[i]);
    s.xev[i] = nullptr;
  }
  if (s.xs) cudaStreamDestroy(s.xs);
  s.xs = nullptr;
  for (int b = 0; b < 2; ++b) {
    if (s.le_h[b]) cudaFree(s.le_h[b]);
    if (s.le_p[b]) cudaFree(s.le_p[b]);
    s.le_h[b] = nullptr;
    s.le_p[b] = nullptr;
  }
  for (int b = 0; b < 4; ++b) {
    if (s.le_b[b]) cudaFree(s.le_b[b]);
    s.le_b[b] = nullptr;
  }
  s.d_lat = nullptr;
  s.d_tiles = nullptr;
  s.M = nullptr;
  s.J = nullptr;
}

int fp32_upload(const DevParams &P, const lb3dc_params &p, Fp32State &s, const double *n,
                const double *db, const uint8_t *rockp, cudaStream_t st) {
  const long long N = P.nsites;
  const double rho0 = s.lat.rho0;
  // the caller has uploaded the rock flags (rockp, device) and set any_rock
  const bool any = P.any_rock != 0;
  if (any && P.nc == 3) return LB3DC_EINVAL;
  s.lat = fp32_make_desc(P, rho0, 0, any);
  attach_le(s);
  s.lat.parity = 0;
  // one FP64 plane at a time through two staging planes: the copy of plane
  // cq + 1 (copy stream) overlaps the conversion of plane cq (populations to
  // deviations, dipoles rounded to FP32, into both buffers); xev[b] marks
  // staging plane b filled, xev[2 + b] drained
  const int nplanes = P.nc * 19 + (P.nc == 3 ? 3 : 0);
  cudaError_t e = cudaEventRecord(s.xev[2], st);
  if (e == cudaSuccess) e = cudaEventRecord(s.xev[3], st);
  for (int cq = 0; cq < nplanes && e == cudaSuccess; ++cq) {
    const int b = cq & 1;
    double *stg = s.stage + (size_t)b * N;
    const bool pop = cq < P.nc * 19;
    const double *src = pop ? n + (size_t)cq * N : db + (size_t)(cq - P.nc * 19) * N;
    float *d0 = pop ? s.f[0] + (size_t)cq * s.S : s.db[0] + (size_t)(cq - P.nc * 19) * s.S;
    float *d1 = pop ? s.f[1] + (size_t)cq * s.S : s.db[1] + (size_t)(cq - P.nc * 19) * s.S;
    const double w = pop ? (cq % 19 == 18 ? 1.0 / 3.0 : 1.0 / 36.0) * rho0 : 0.0;
    e = cudaStreamWaitEvent(s.xs, s.xev[2 + b], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(stg, src, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s.xs);
    if (e == cudaSuccess) e = cudaEventRecord(s.xev[b], s.xs);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, s.xev[b], 0);
    if (e != cudaSuccess) break;
    k_plane_from_fp64<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(stg, d0, d1, N, w,
                                                                    any ? rockp : nullptr);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(s.xev[2 + b], st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s.xs);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return LB3DC_ECUDA;
  if (cudaMemcpyAsync(s.d_lat, &s.lat, sizeof(LatDesc), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return LB3DC_ECUDA;
  if (s.le_b[0] && le_gather(P, s, st) != cudaSuccess) return LB3DC_ECUDA;
  // keep the launch shape chosen so far (set or autotuned); the kernel
  // variant may change with the rock flag
  int rc = rebuild_tiles(P, s, FusedShape{s.tx, s.ty, s.zc, s.split}, st);
  if (rc) return rc;
  (void)p;
  return cudaStreamSynchronize(st) == cudaSuccess ? LB3DC_OK : LB3DC_ECUDA;
}

int fp32_download(const DevParams &P, const lb3dc_params &p, Fp32State &s, double *n, double *db,
                  double *rho, double *mom, double *da, const uint8_t *rockp, cudaStream_t st) {
  const long long N = P.nsites;
  const int nc = P.nc;
  const int cur = s.lat.parity;
  const double rho0 = s.lat.rho0;
  std::vector<double> tmp;
  double *nn = n;
  if (!nn && (rho || mom)) {
    tmp.resize((size_t)nc * 19 * N);
    nn = tmp.data();
  }
  if (nn) {
    // deviations -> FP64 populations, one plane at a time through two
    // staging planes: the conversion of plane cq + 1 overlaps the copy of
    // plane cq (copy stream); xev[b] marks staging plane b filled, xev[2 + b]
    // drained
    cudaError_t e = cudaEventRecord(s.xev[2], s.xs);
    if (e == cudaSuccess) e = cudaEventRecord(s.xev[3], s.xs);
    for (int cq = 0; cq < nc * 19 && e == cudaSuccess; ++cq) {
      const int b = cq & 1;
      double *stg = s.stage + (size_t)b * N;
      const double w = (cq % 19 == 18 ? 1.0 / 3.0 : 1.0 / 36.0) * rho0;
      e = cudaStreamWaitEvent(st, s.xev[2 + b], 0);
      if (e != cudaSuccess) break;
      k_plane_to_fp64<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(s.f[cur] + (size_t)cq * s.S,
                                                                    stg, N, w);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaEventRecord(s.xev[b], st);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s.xs, s.xev[b], 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(nn + (size_t)cq * N, stg, (size_t)N * sizeof(double),
                            cudaMemcpyDeviceToHost, s.xs);
      if (e == cudaSuccess) e = cudaEventRecord(s.xev[2 + b], s.xs);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.xs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return LB3DC_ECUDA;
  }
  std::vector<uint8_t> rk(N, 0);
  if (rockp && (s.lat.flags & LAT_ROCK)) {
    if (cudaMemcpyAsync(rk.data(), rockp, N, cudaMemcpyDeviceToHost, st) != cudaSuccess) return LB3DC_ECUDA;
    cudaStreamSynchronize(st);
    // rock sites hold no populations (code/lb3d_ic_rock.F90:163-170)
    if (nn)
      for (long long i = 0; i < N; ++i)
        if (rk[i])
          for (int cq = 0; cq < nc * 19; ++cq) nn[(size_t)cq * N + i] = 0.0;
  }
  if (rho || mom) {
    for (int c = 0; c < nc; ++c)
      for (long long i = 0; i < N; ++i) {
        double r = 0, m0 = 0, m1 = 0, m2 = 0;
        for (int q = 0; q < 19; ++q) {
          const double ng = nn[((size_t)c * 19 + q) * N + i] * gw(q);
          r += ng;
          m0 += ng * cx(q);
          m1 += ng * cy(q);
          m2 += ng * cz(q);
        }
        if (rho) rho[(size_t)c * N + i] = r;
        if (mom) {
          mom[((size_t)c * 3 + 0) * N + i] = m0;
          mom[((size_t)c * 3 + 1) * N + i] = m1;
          mom[((size_t)c * 3 + 2) * N + i] = m2;
        }
      }
  }
  if (db) {
    if (nc == 3) {
      std::vector<float> d(3 * N);
      if (cudaMemcpyAsync(d.data(), s.db[cur], d.size() * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return LB3DC_ECUDA;
      cudaStreamSynchronize(st);
      for (long long i = 0; i < 3 * N; ++i) db[i] = d[i];
    } else {
      std::memset(db, 0, 3 * N * sizeof(double));
    }
  }
  if (da) std::memset(da, 0, 3 * N * sizeof(double));
  (void)p;
  return LB3DC_OK;
}

int fp32_step(const DevParams &P, Fp32State &s, const uint8_t *rock, cudaStream_t st,
              const LEStep *le) {
  return fp32_run(P, s, rock, 1, st, le);
}

int fp32_run(const DevParams &P, Fp32State &s, const uint8_t *rock, int nsteps, cudaStream_t st,
             const LEStep *le) {
  FusedShape sh{s.tx, s.ty, s.zc, s.split};
  const bool rk = (s.lat.flags & LAT_ROCK) != 0, body = (s.lat.flags & LAT_BODY) != 0;
  if (le && !s.le_h[0]) return LB3DC_ESTATE;
  // kernels per step: the pass(es), two Lees-Edwards halo kernels, the parity flip
  const int passes = sh.split ? (P.nc == 3 ? 3 : 2) : 1;
  const int per_step = passes + (le ? 2 : 0) + 1;
  for (int i = 0; i < nsteps; ++i) {
    if (s.timer) s.timer->start(st);
    cudaError_t e = sh.split == 3
                        ? launch_mf(P, s, rock, st, le)
                        : fp32_launch_fused(P.nc, rk, body, sh, s.d_lat, s.d_tiles, s.ntiles, 0,
                                            s.f[0], s.f[1], s.db[0], s.db[1], rock, s.S, st, s.M,
                                            s.J, le, &P);
    if (s.timer) {
      s.timer->stop(st);
      s.timer->launches += per_step;
    }
    if (e != cudaSuccess) return LB3DC_ECUDA;
    e = fp32_flip_parity(s.d_lat, 1, st);
    if (e != cudaSuccess) return LB3DC_ECUDA;
    s.lat.parity ^= 1;
  }
  return LB3DC_OK;
}

// Dumps of the FP32 state: the deviations are converted to FP64
// populations on the device and the FP64 dump kernels are applied, with the
// densities recomputed from the current populations (the FP32 path does not
// keep the post-stream moments between steps).
int fp32_dump(const DevParams &P, Fp32State &s, int field, const uint8_t *rock, double *out,
              cudaStream_t st) {
  const long long N = P.nsites;
  const int nc = P.nc;
  double *n = nullptr, *rho = nullptr, *psi = nullptr, *mom = nullptr, *db = nullptr;
  size_t bytes = ((size_t)nc * 19 * N + 2 * (size_t)nc * N + 3 * (size_t)nc * N + 3 * (size_t)N) * 8;
  if (cudaMalloc(&n, bytes) != cudaSuccess) return LB3DC_ENOMEM;
  rho = n + (size_t)nc * 19 * N;
  psi = rho + (size_t)nc * N;
  mom = psi + (size_t)nc * N;
  db = mom + 3 * (size_t)nc * N;
  const int cur = s.lat.parity;
  k_to_fp64<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(s.f[cur], n, s.S, 0, N, nc, s.lat.rho0);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = fp64_moments(P, n, rho, psi, mom, st);
  if (e == cudaSuccess && nc == 3) {
    std::vector<float> h(3 * N);
    std::vector<double> hd(3 * N);
    e = cudaMemcpyAsync(h.data(), s.db[cur], 3 * N * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    for (long long i = 0; i < 3 * N; ++i) hd[i] = h[i];
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, hd.data(), 3 * N * 8, cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = fp64_dump(P, field, n, rho, psi, db, rock, out, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(n);
  return e == cudaSuccess ? LB3DC_OK : LB3DC_ECUDA;
}

cudaError_t fp32_reduce_conservation(const DevParams &P, Fp32State &s, const uint8_t *rock,
                                     double *scratch, double mass[3], double mom[3],
                                     cudaStream_t st) {
  return reduce_conservation_fp32(P, s.f[s.lat.parity], s.S, 0, (double)s.lat.rho0, rock, scratch,
                                  mass, mom, st);
}

cudaError_t fp32_sanity_counts(const DevParams &P, Fp32State &s, unsigned long long *scratch,
                               unsigned long long cnt[2], cudaStream_t st) {
  return sanity_counts_fp32(P, s.f[s.lat.parity], s.S, 0, (double)s.lat.rho0, scratch, cnt, st);
}

cudaError_t fp32_sanity_velocity(const DevParams &P, Fp32State &s, const uint8_t *rock,
                                 void *scratch, SanityVelocity &out, cudaStream_t st) {
  return sanity_velocity_fp32(P, s.f[s.lat.parity], s.S, 0, (double)s.lat.rho0, rock, scratch, out,
                              st);
}

}  // namespace lb3d
