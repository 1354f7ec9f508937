// fp32_stencil.cuh -- per-site stencil arithmetic shared by the FP32 kernels
// (fused and split strategies), included by fp32_path.cu after its helpers:
// the dipole relaxation and the ternary and binary Shan-Chen forces, read
// from on-chip rings of per-site entries.

// Dipole relaxation of one site (code/lb3d_collision.F90:296-403) from the
// ring planes of moment entries {rho_b - rho_r, da_x, da_y, da_z} (row
// stride AW) and the site's own surfactant density deviation.  The dipole
// field h = sum_q g_q [-sgn c_q phi_q + da_q - 2 c_q (c_q . da_q)] + da_own
// is summed over the nine pairs of opposite neighbours (q, bounce(q)), whose
// c_q terms differ only in sign: per pair the difference of phi and the sum
// of da enter once.
// AP is a pointer to the entries or an accessor with operator[] (the
// moment-field strategy forms the entries from two ring boxes).
template <int AW, typename AP>
__device__ __forceinline__ float3 dipole_site(AP Am, AP A0, AP Ap, int as, const LatDesc &Lg, float rho0,
                                              float own_drs) {
  const float4 own0 = A0[as];
  float P0 = 0.f, P1 = 0.f, P2 = 0.f;  // sum g c (phi_q - phi_qbar)
  float S0 = 0.f, S1 = 0.f, S2 = 0.f;  // sum g (da_q + da_qbar)
  float B0 = 0.f, B1 = 0.f, B2 = 0.f;  // sum g c (c . (da_q + da_qbar))
  const float isN = 1.0f / fmaxf(rho0 + own_drs, 1.0e-4f);
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    if (bounce(q) < q) continue;  // each pair once, from its first member
    const int qb = bounce(q);
    const AP &Aq = cz(q) == 1 ? Ap : (cz(q) == -1 ? Am : A0);
    const AP &Ab = cz(qb) == 1 ? Ap : (cz(qb) == -1 ? Am : A0);
    const float4 e = Aq[as + cx(q) + AW * cy(q)];
    const float4 f = Ab[as + cx(qb) + AW * cy(qb)];
    const float g = (float)gw(q);
    const float dphi = e.x - f.x;
    const float s0 = e.y + f.y, s1 = e.z + f.z, s2 = e.w + f.w;
    S0 = fmaf(g, s0, S0);
    S1 = fmaf(g, s1, S1);
    S2 = fmaf(g, s2, S2);
    float t = 0.f;  // c . s
    if (cx(q)) t = fmaf((float)cx(q), s0, t);
    if (cy(q)) t = fmaf((float)cy(q), s1, t);
    if (cz(q)) t = fmaf((float)cz(q), s2, t);
    if (cx(q)) P0 = fmaf(g * (float)cx(q), dphi, P0), B0 = fmaf(g * (float)cx(q), t, B0);
    if (cy(q)) P1 = fmaf(g * (float)cy(q), dphi, P1), B1 = fmaf(g * (float)cy(q), t, B1);
    if (cz(q)) P2 = fmaf(g * (float)cz(q), dphi, P2), B2 = fmaf(g * (float)cz(q), t, B2);
  }
  const float msgn = (Lg.g_bs >= 0.0f) ? -1.0f : 1.0f;
  const float h0 = fmaf(msgn, P0, fmaf(-2.0f, B0, own0.y + S0));
  const float h1 = fmaf(msgn, P1, fmaf(-2.0f, B1, own0.z + S1));
  const float h2 = fmaf(msgn, P2, fmaf(-2.0f, B2, own0.w + S2));
  const float hn = sqrtf(fmaf(h2, h2, fmaf(h1, h1, h0 * h0)));
  const float hm = Lg.beta * hn;
  const float fac = (hm > 1.0e-2f) ? Lg.d0 * langevin(hm) / hn : Lg.d0 * Lg.beta * (1.0f / 3.0f);
  const float od = Lg.omega_d, om1 = (1.0f - od) * isN;
  const float of = od * fac;
  return make_float3(fmaf(of, h0, om1 * own0.y), fmaf(of, h1, om1 * own0.z),
                     fmaf(of, h2, om1 * own0.w));
}

// Ternary Shan-Chen force (code/lb3d_force_shanchen.F90:215-330) of one
// site from psi entries P = {-, dpsi_r, dpsi_b, dpsi_s} (row stride WP, the
// site at index ap) and dipole entries B (row stride WB, the site at bp),
// accumulated as neighbour moments so that the own dipole d enters once:
//   f_cs = SA - 2V, f_sc = SG d - 2 T d, f_ss = M^T d + M d + tr(M) d - 2 Q d
// with a = d(y) psi_s(y), SA = sum g a, V = sum g (a.c) c, G = g (psi_b -
// psi_r), SG = sum G, T = sum G c c^T, M = sum 8g a c^T, Q = sum 8g (a.c) c c^T.
// Dipole ring planes, read as float3 at an entry index: float4 entries
// {d_x, d_y, d_z, -}, or three axis planes of `np` entries each.
struct DipF4 {
  const float4 *p;
  __device__ __forceinline__ float3 operator()(int i) const {
    const float4 v = p[i];
    return make_float3(v.x, v.y, v.z);
  }
};
struct DipAxes {
  const float *p;
  int np;
  __device__ __forceinline__ float3 operator()(int i) const {
    return make_float3(p[i], p[np + i], p[2 * np + i]);
  }
};

template <int WP, int WB, typename DR>
__device__ __forceinline__ void force_ternary(const float4 *Pm, const float4 *P0, const float4 *Pp,
                                              DR Bm, DR B0, DR Bp, int ap, int bp,
                                              const LatDesc &Lg, float psi0, float Fx[3][3]) {
  // paired accumulators: FB[k] = (f_rb, f_br)_k, SA01 = (SA_x, SA_y),
  // M01[k] = (M_xk, M_yk), TQ[K] = (T_K, Q_K)
  float2 FB[3] = {f2(0.f), f2(0.f), f2(0.f)}, M01[3] = {f2(0.f), f2(0.f), f2(0.f)};
  float2 TQ[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};
  float2 SA01 = f2(0.f);
  float SA2 = 0.f, V[3] = {0, 0, 0}, M2[3] = {0, 0, 0}, SG = 0.f;
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    const float4 *Pq = cz(q) == 1 ? Pp : (cz(q) == -1 ? Pm : P0);
    const DR &Bq = cz(q) == 1 ? Bp : (cz(q) == -1 ? Bm : B0);
    const float g = (float)gw(q);
    const int c[3] = {cx(q), cy(q), cz(q)};
    const float4 e = Pq[ap + cx(q) + WP * cy(q)];
    const float3 b = Bq(bp + cx(q) + WB * cy(q));
    const float ps = psi0 + e.w;
    const float2 a01 = mul2(make_float2(b.x, b.y), f2(ps));
    const float a2 = b.z * ps;
    const float a[3] = {a01.x, a01.y, a2};
    float ac = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (c[k]) ac = fmaf((float)c[k], a[k], ac);
    const float Gq = g * (e.z - e.y);
    const float g8 = 8.0f * g;
    SG += Gq;
    SA01 = fma2(f2(g), a01, SA01);
    SA2 = fmaf(g, a2, SA2);
    const float2 ezy = make_float2(e.z, e.y);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (c[k]) {
        FB[k] = fma2(f2(g * (float)c[k]), ezy, FB[k]);
        V[k] = fmaf(g * (float)c[k], ac, V[k]);
        M01[k] = fma2(f2(g8 * (float)c[k]), a01, M01[k]);
        M2[k] = fmaf(g8 * (float)c[k], a2, M2[k]);
      }
    }
    const float2 gq = make_float2(Gq, g8 * ac);
#define LB3D_SYM(I, J, K)                                  \
  if (c[I] && c[J]) TQ[K] = fma2(gq, f2((float)(c[I] * c[J])), TQ[K]);
    LB3D_SYM(0, 0, 0) LB3D_SYM(1, 1, 1) LB3D_SYM(2, 2, 2)
    LB3D_SYM(0, 1, 3) LB3D_SYM(0, 2, 4) LB3D_SYM(1, 2, 5)
#undef LB3D_SYM
  }
  const float frb[3] = {FB[0].x, FB[1].x, FB[2].x}, fbr[3] = {FB[0].y, FB[1].y, FB[2].y};
  const float SA[3] = {SA01.x, SA01.y, SA2};
  const float T[6] = {TQ[0].x, TQ[1].x, TQ[2].x, TQ[3].x, TQ[4].x, TQ[5].x};
  const float Q[6] = {TQ[0].y, TQ[1].y, TQ[2].y, TQ[3].y, TQ[4].y, TQ[5].y};
  const float M[3][3] = {{M01[0].x, M01[1].x, M01[2].x}, {M01[0].y, M01[1].y, M01[2].y},
                         {M2[0], M2[1], M2[2]}};
  const float3 dd = B0(bp);
  const float d[3] = {dd.x, dd.y, dd.z};
  const float4 own = P0[ap];
  const float psr = psi0 + own.y, psb = psi0 + own.z, pss = psi0 + own.w;
  // products of the symmetric tensors with d, one fused multiply-add per term
  auto dot3 = [&](float a0, float a1, float a2) { return fmaf(a2, d[2], fmaf(a1, d[1], a0 * d[0])); };
  const float Td[3] = {dot3(T[0], T[3], T[4]), dot3(T[3], T[1], T[5]), dot3(T[4], T[5], T[2])};
  const float Qd[3] = {dot3(Q[0], Q[3], Q[4]), dot3(Q[3], Q[1], Q[5]), dot3(Q[4], Q[5], Q[2])};
  const float trM = M[0][0] + M[1][1] + M[2][2];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float MTd = dot3(M[0][k], M[1][k], M[2][k]);
    const float Md = dot3(M[k][0], M[k][1], M[k][2]);
    const float fcs = fmaf(-2.0f, V[k], SA[k]);
    const float fsc = fmaf(SG, d[k], -2.0f * Td[k]);
    const float fss = fmaf(-2.0f, Qd[k], fmaf(trM, d[k], MTd + Md));
    const float cs = (-2.0f * Lg.g_bs) * fcs;
    Fx[1][k] = fmaf(-Lg.g_br, fbr[k], cs) * psb;
    Fx[0][k] = fmaf(-Lg.g_br, frb[k], -cs) * psr;
    Fx[2][k] = fmaf(2.0f * Lg.g_bs, fsc, -Lg.g_ss * fss) * pss;
  }
}

// Binary force with walls (:127-210) from psi entries {dpsi_r, dpsi_b, -, -}.
// LE (a Lees-Edwards lattice; the site at gx, gy, gz): a neighbour across the
// sheared x boundary is a halo site, never rock; a rock neighbour reached
// through the periodic y or z wrap has no rock colour there, as the
// reference's y and z exchanges of a sheared lattice leave it
// (code/lb3d_bc_leesedwards.F90:1079-1308): psi(0) = 0 on the wall side.
template <int W, bool ROCK, typename E, bool LE = false>
__device__ __forceinline__ void force_binary(const E *Pm, const E *P0, const E *Pp,
                                             int as, const Nbr &nb, const uint8_t *__restrict__ RK,
                                             const LatDesc &Lg, float psi0, float Fx[2][3], int gx = 0,
                                             int gy = 0, int gz = 0) {
  float frb[3] = {0, 0, 0}, fbr[3] = {0, 0, 0}, fwr[3] = {0, 0, 0}, fwb[3] = {0, 0, 0};
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    const E *Pq = cz(q) == 1 ? Pp : (cz(q) == -1 ? Pm : P0);
    const int an = as + cx(q) + W * cy(q);
    const float g = (float)gw(q);
    const int c[3] = {cx(q), cy(q), cz(q)};
    bool nrock = false, colour = true;
    if (ROCK) {
      const bool xhalo = LE && (gx + cx(q) < 0 || gx + cx(q) >= Lg.nx);
      nrock = !xhalo && __ldg(RK + nb.cx[1 + cx(q)] + nb.ry[1 + cy(q)] + nb.rz[1 + cz(q)]) != 0;
      if (LE && nrock)
        colour = !(gy + cy(q) < 0 || gy + cy(q) >= Lg.ny || gz + cz(q) < 0 || gz + cz(q) >= Lg.nz);
    }
    const E e = Pq[an];
    const float pr = nrock ? -psi0 : e.x, pb = nrock ? -psi0 : e.y;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (c[k]) {
        frb[k] = fmaf(pb * g, (float)c[k], frb[k]);
        fbr[k] = fmaf(pr * g, (float)c[k], fbr[k]);
        if (ROCK && nrock && colour) {
          fwb[k] = fmaf(Lg.psiw_b * g, (float)c[k], fwb[k]);
          fwr[k] = fmaf(Lg.psiw_r * g, (float)c[k], fwr[k]);
        }
      }
  }
  const E own = P0[as];
  const float psr = psi0 + own.x, psb = psi0 + own.y;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Fx[1][k] = fmaf(-Lg.g_br, fbr[k], Lg.wall_b * fwb[k]) * psb;
    Fx[0][k] = fmaf(-Lg.g_br, frb[k], Lg.wall_r * fwr[k]) * psr;
  }
}

