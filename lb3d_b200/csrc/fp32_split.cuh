// fp32_split.cuh -- the split strategy of the FP32 deviation path, included
// by fp32_path.cu after its helpers.
//
// Per step, three passes over the tile list:
//   moments (k_fused in MODE_MOMENTS): post-stream moments of every site once,
//       written as the moment field M, two float4 per ternary site:
//       {rho_b - rho_r, da} (the dipole stencil input) and {drho_s, psi
//       deviations} (the force stencil input), and with strategy 1 also J
//       (the own-site densities and momenta the BGK update needs);
//   dipole  (k_split_dipole, ternary): new dipoles on each tile from M with a
//       one-site halo, code/lb3d_collision.F90:296-403;
//   collide (k_split_collide): Shan-Chen force from M and the new dipoles
//       with a one-site halo, body force, one pull of the own populations,
//       BGK, store.
// Each pass reads its stencil field through a three-plane ring in shared
// memory while marching in z, so every field is loaded from global memory
// once per tile plane (halos hit L2).

// Asynchronous copies global -> shared (cp.async, 4/8/16 bytes) in commit
// groups; a thread waits for its own groups, a barrier then publishes them.
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Dipole pass: the {rho_b - rho_r, da} entries of M stream through a
// five-slot ring, refilled with cp.async three planes ahead of the plane
// being relaxed (one barrier per plane); each thread also prefetches its own
// site's drho_s.
template <int TX, int TY>
__global__ void __launch_bounds__(TX *TY, 1280 / (TX * TY))
    k_split_dipole(const LatDesc *__restrict__ lats, const Tile *__restrict__ tiles, int ntiles,
                   float *db0, float *db1, const float4 *__restrict__ Mf, unsigned S) {
  constexpr int NT = TX * TY, AW = TX + 2, AN = AW * (TY + 2), RS = 5;
  extern __shared__ float4 sm4[];  // ring [RS][AN] float4, own drho_s [RS][NT] float
  float *owns = reinterpret_cast<float *>(sm4 + RS * AN);
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    const LatDesc &Lg = lats[T.lat];
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    const int base = (int)Lg.base;
    float *__restrict__ DBo = (Lg.parity ? db0 : db1) + base;
    const float4 *__restrict__ Mb = Mf + base;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool act = gx < nx && gy < ny;
    // the in-plane offsets of this thread's ring entries, once per tile
    constexpr int RE = (AN + NT - 1) / NT;
    int rxy[RE];
#pragma unroll
    for (int e = 0; e < RE; ++e) {
      const int s = tid + e * NT;
      rxy[e] = s < AN ? wrapz(x0 - 1 + s % AW, nx) + nx * wrapz(y0 - 1 + s / AW, ny) : 0;
    }
    const int own_xy = gx + nx * gy;
    // ring index r holds plane z0 - 1 + r in slot r % RS
    auto load_ring = [&](int r) {
      const float4 *plane = Mb + nx * ny * wrapz(z0 - 1 + r, nz);
      float4 *slot = sm4 + (r % RS) * AN;
#pragma unroll
      for (int e = 0; e < RE; ++e)
        if (tid + e * NT < AN) cp_async16(slot + tid + e * NT, plane + rxy[e]);
      if (act)
        cp_async4(owns + (r % RS) * NT + tid, reinterpret_cast<const float *>(plane + S + own_xy));
    };
    load_ring(0);
    load_ring(1);
    load_ring(2);
    cp_async_commit();
    for (int k = 0; k < zc; ++k) {
      if (k + 3 <= zc + 1) load_ring(k + 3);
      cp_async_commit();
      cp_async_wait<1>();  // ring planes up to k + 2 landed (this thread's copies)
      __syncthreads();     // ... and everybody's
      if (act) {
        const int as = (tx + 1) + AW * (ty + 1);
        const float3 d = dipole_site<AW>(sm4 + (k % RS) * AN, sm4 + ((k + 1) % RS) * AN,
                                         sm4 + ((k + 2) % RS) * AN, as, Lg, Lg.rho0,
                                         owns[((k + 1) % RS) * NT + tid]);
        const int i = own_xy + nx * ny * wrapz(z0 + k, nz);
        DBo[i] = d.x;
        DBo[S + i] = d.y;
        DBo[2 * S + i] = d.z;
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // the next tile refills ring slots 0..2
  }
}

template <int NC, int TX, int TY, bool ROCK, bool BODY>
__global__ void __launch_bounds__(TX *TY, 768 / (TX * TY))
    k_split_collide(const LatDesc *__restrict__ lats, const Tile *__restrict__ tiles, int ntiles,
                    float *f0, float *f1, float *db0, float *db1, const uint8_t *__restrict__ rock,
                    unsigned S, const float4 *__restrict__ Mf, const float4 *__restrict__ Jf) {
  constexpr int NT = TX * TY, AW = TX + 2, AN = AW * (TY + 2);
  constexpr int JV = (NC == 3) ? 3 : 2;
  extern __shared__ float4 sm4[];  // psi ring [3][AN], dipole ring [3][AN] (ternary)
  float4 *ringP = sm4;
  float4 *ringB = sm4 + 3 * AN;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    const LatDesc &Lg = lats[T.lat];
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    const int base = (int)Lg.base;
    const int par = Lg.parity;
    const float *__restrict__ F = (par ? f1 : f0) + base;
    float *__restrict__ Fo = (par ? f0 : f1) + base;
    const float *__restrict__ DBn = (NC == 3) ? (par ? db0 : db1) + base : nullptr;  // new dipoles
    const float4 *__restrict__ Mb = Mf + base;
    const float4 *__restrict__ Jb = Jf + base;
    const uint8_t *__restrict__ RK = rock + base;
    const float rho0 = Lg.rho0, psi0 = Lg.psi0;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    for (int it = 0; it < zc + 2; ++it) {
      const int zA = z0 - 1 + it, gz = wrapz(zA, nz);
      float4 *slotP = ringP + (it % 3) * AN;
      float4 *slotB = ringB + (it % 3) * AN;
      for (int s = tid; s < AN; s += NT) {
        const int vx = x0 - 1 + s % AW, vy = y0 - 1 + s / AW;
        const int gx = wrapz(vx, nx);
        const int gy = wrapz(vy, ny);
        const int i = gx + nx * (gy + ny * gz);
        if (NC == 3) {
          slotP[s] = __ldg(Mb + S + i);  // {da_z, dpsi_r, dpsi_b, dpsi_s}
          slotB[s] = make_float4(__ldg(DBn + i), __ldg(DBn + S + i), __ldg(DBn + 2 * S + i), 0.f);
        } else {
          const float2 v = __ldg(reinterpret_cast<const float2 *>(Mb) + i);
          slotP[s] = make_float4(v.x, v.y, 0.f, 0.f);
        }
      }
      __syncthreads();
      if (it >= 2) {
        const int gx = x0 + tx, gy = y0 + ty;
        if (gx < nx && gy < ny) {
          const int zC = zA - 1;
          const int gzc = wrapz(zC, nz);
          Nbr nb;
          make_nbr(nb, gx, gy, gzc, nx, ny, nz);
          const int self = noff<18, 1>(nb);
          bool own_rock = false;
          if (ROCK) own_rock = __ldg(RK + self) != 0;
          if (!own_rock) {
            const int as = (tx + 1) + AW * (ty + 1);
            const float4 *Pm = ringP + ((it - 2) % 3) * AN, *P0 = ringP + ((it - 1) % 3) * AN;
            float Fx[NC][3];
            if (NC == 3)
              force_ternary<AW, AW>(Pm, P0, slotP, DipF4{ringB + ((it - 2) % 3) * AN},
                                    DipF4{ringB + ((it - 1) % 3) * AN}, DipF4{slotB}, as, as, Lg, psi0,
                                    reinterpret_cast<float(*)[3]>(Fx));
            else
              force_binary<AW, ROCK>(Pm, P0, slotP, as, nb, RK, Lg, psi0,
                                     reinterpret_cast<float(*)[3]>(Fx));
            // own densities and momenta from the moments pass
            float J[4 * JV];
#pragma unroll
            for (int v = 0; v < JV; ++v) {
              const float4 w = __ldg(Jb + v * S + self);
              J[4 * v] = w.x;
              J[4 * v + 1] = w.y;
              J[4 * v + 2] = w.z;
              J[4 * v + 3] = w.w;
            }
            float dr[NC], rho[NC], j[NC][3];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              dr[c] = J[c];
              rho[c] = rho0 + dr[c];
              j[c][0] = J[NC + 3 * c];
              j[c][1] = J[NC + 3 * c + 1];
              j[c][2] = J[NC + 3 * c + 2];
            }
            if (BODY) {
              const int x1 = gx + 1, y1 = gy + 1, z1 = gzc + 1;
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
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              const float k = Lg.tau[c] / (Lg.amass[c] * fmaxf(rho[c], 1.0e-8f));
              float *fo = Fo + (size_t)(c * 19) * S + self;
              if (Lg.omega[c] == 1.0f) {
                // full relaxation: the BGK update is the equilibrium, the
                // populations drop out and need no pull (the own moments
                // came from the moments pass)
                eq_store(fo, S, rho[c], dr[c], fmaf(k, Fx[c][0], u0), fmaf(k, Fx[c][1], u1),
                         fmaf(k, Fx[c][2], u2), Lg.omega[c]);
                continue;
              }
              float d[19];
              pull_comp<ROCK, true>(F, S, c, nb, self, RK, d);
              bgk_update(d, rho[c], dr[c], fmaf(k, Fx[c][0], u0), fmaf(k, Fx[c][1], u1),
                         fmaf(k, Fx[c][2], u2), Lg.omega[c]);
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

// ---------------------------------------------------------------------------
// Collide pass with asynchronous staging (split strategy 2).
//
// The plain collide pass above is latency bound: each thread has at most one
// component's 19 pulls in flight, and nothing is in flight while it works
// through the force stencil.  Here every thread copies the 19*NC pulled
// deviations of its next site straight into its own shared-memory column
// with cp.async (no registers held) as soon as the current site's BGK
// update has read the previous ones, so the copies fly during the barrier,
// the ring refill and the whole force stencil of the next plane.  The
// psi/dipole rings are refilled the same way, three planes ahead, in a
// five-slot ring (one barrier per plane).  The own densities and momenta
// are summed from the staged values in the order the moments pass uses, so
// the J field is not needed and the result equals the plain collide pass
// bit for bit.
// ---------------------------------------------------------------------------
// Shared-memory layout of k_split_collide2 (bytes): psi ring [5][AN] float4
// (float2 for binary), dipole ring [5][3][AN] float (ternary; one plane per
// axis, so the 4-byte copies into it do not collide in banks), population
// stage [19*NC][NT] float.
// Five ring slots (one barrier per plane).  Ternary lattices run two CTAs
// of 128 threads per SM with up to 255 registers: measured faster than
// three CTAs at 168 registers, which were faster than four at 128 with a
// four-slot ring (the pass gains more from registers, i.e. independent work
// per warp, than from warps).  Binary lattices keep three CTAs, which the
// Lees-Edwards variant needs.
template <int NC, int TX, int TY>
struct Collide2Geom {
  static constexpr int NT = TX * TY, AW = TX + 2, AN = AW * (TY + 2);
  static constexpr int RS = 5, MINB = NT >= 256 ? (NC == 3 ? 1 : 2) : (NC == 3 ? 2 : 3);
  static constexpr int PB = (NC == 3) ? 16 : 8;  // psi entry bytes
  static constexpr int P_BYTES = RS * AN * PB;
  static constexpr int B_BYTES = (NC == 3) ? RS * AN * 12 : 0;
  static constexpr int F_BYTES = 19 * NC * NT * 4;
  static constexpr int SMEM = P_BYTES + B_BYTES + F_BYTES;
};

// Issues the pulls of component c of one site into the stage column
// (stage[q * NT]), with half-way bounce-back when ROCK (as pull_comp).
template <bool ROCK, int NT>
__device__ __forceinline__ void pull_async(const float *__restrict__ F, unsigned S, int c, const Nbr &n,
                                           int self, const uint8_t *__restrict__ rk, float *stage) {
  const float *fc = F + (size_t)(c * 19) * S;
  cp_async4(stage + 18 * NT, fc + 18 * S + self);
#define LB3D_APULL(Q)                                                    \
  {                                                                      \
    const int up = noff<Q, -1>(n);                                       \
    bool uf = true;                                                      \
    if (ROCK) uf = __ldg(rk + up) == 0;                                  \
    cp_async4(stage + (Q) * NT, fc + (uf ? Q * S + up : bounce(Q) * S + self)); \
  }
  LB3D_APULL(0) LB3D_APULL(1) LB3D_APULL(2) LB3D_APULL(3) LB3D_APULL(4) LB3D_APULL(5)
  LB3D_APULL(6) LB3D_APULL(7) LB3D_APULL(8) LB3D_APULL(9) LB3D_APULL(10) LB3D_APULL(11)
  LB3D_APULL(12) LB3D_APULL(13) LB3D_APULL(14) LB3D_APULL(15) LB3D_APULL(16) LB3D_APULL(17)
#undef LB3D_APULL
}

// pull_async with the Lees-Edwards halo planes across the x boundary (with
// ROCK: bounce-back from rock sites inside the lattice, as le_src)
template <int NT, bool ROCK = false>
__device__ __forceinline__ void pull_async_le(const float *__restrict__ F, unsigned S, int c, const Nbr &n,
                                              int self, int gx, int nx, const LeYZ &w,
                                              const LatDesc &Lg, int NP, float *stage,
                                              const uint8_t *__restrict__ rk = nullptr) {
  const float *fc = F + (size_t)(c * 19) * S;
  cp_async4(stage + 18 * NT, fc + 18 * S + self);
#define LB3D_APULL_LE(Q) cp_async4(stage + (Q) * NT, le_src<Q, ROCK>(fc, S, c, n, gx, nx, w, Lg, NP, self, rk));
  LB3D_APULL_LE(0) LB3D_APULL_LE(1) LB3D_APULL_LE(2) LB3D_APULL_LE(3) LB3D_APULL_LE(4)
  LB3D_APULL_LE(5) LB3D_APULL_LE(6) LB3D_APULL_LE(7) LB3D_APULL_LE(8) LB3D_APULL_LE(9)
  LB3D_APULL_LE(10) LB3D_APULL_LE(11) LB3D_APULL_LE(12) LB3D_APULL_LE(13) LB3D_APULL_LE(14)
  LB3D_APULL_LE(15) LB3D_APULL_LE(16) LB3D_APULL_LE(17)
#undef LB3D_APULL_LE
}

// INF: the lattice has stage-8 inflow boundaries on its z planes.
template <int NC, int TX, int TY, bool ROCK, bool BODY, bool LE = false, bool INF = false>
__global__ void __launch_bounds__(TX *TY, Collide2Geom<NC, TX, TY>::MINB)
    k_split_collide2(const LatDesc *__restrict__ lats, const Tile *__restrict__ tiles, int ntiles,
                     float *f0, float *f1, float *db0, float *db1, const uint8_t *__restrict__ rock,
                     unsigned S, const float4 *__restrict__ Mf) {
  using G = Collide2Geom<NC, TX, TY>;
  constexpr int NT = G::NT, AW = G::AW, AN = G::AN, RS = G::RS;
  extern __shared__ __align__(16) unsigned char smraw[];
  float4 *ringP4 = reinterpret_cast<float4 *>(smraw);          // ternary psi ring
  float2 *ringP2 = reinterpret_cast<float2 *>(smraw);          // binary psi ring
  float *ringB = reinterpret_cast<float *>(smraw + G::P_BYTES);  // [RS][3][AN]
  float *stage = reinterpret_cast<float *>(smraw + G::P_BYTES + G::B_BYTES);
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  float *mystage = stage + tid;

  // the tile's lattice descriptor, copied to shared memory once per tile:
  // the per-site physics constants are then shared loads, not global ones
  __shared__ LatDesc sLat;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    if (tid == 0) sLat = lats[T.lat];
    __syncthreads();
    const LatDesc &Lg = sLat;
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    const int base = (int)Lg.base;
    const int par = Lg.parity;
    const float *__restrict__ F = (par ? f1 : f0) + base;
    float *__restrict__ Fo = (par ? f0 : f1) + base;
    const float *__restrict__ DBn = (NC == 3) ? (par ? db0 : db1) + base : nullptr;  // new dipoles
    const float4 *__restrict__ Mb = Mf + base;
    const uint8_t *__restrict__ RK = rock + base;
    const float rho0 = Lg.rho0, psi0 = Lg.psi0;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool act = gx < nx && gy < ny;

    // the in-plane offsets of this thread's ring entries, once per tile
    constexpr int RE = (AN + NT - 1) / NT;
    int rxy[RE];
#pragma unroll
    for (int e = 0; e < RE; ++e) {
      const int s = tid + e * NT;
      rxy[e] = s < AN ? wrapz(x0 - 1 + s % AW, nx) + nx * wrapz(y0 - 1 + s / AW, ny) : 0;
    }
    // ring index r holds plane z0 - 1 + r in slot r % RS
    auto load_ring = [&](int r) {
      const int gz = wrapz(z0 - 1 + r, nz);
      const int sl = (r % RS) * AN;
#pragma unroll
      for (int e = 0; e < RE; ++e) {
        const int s = tid + e * NT;
        if (s >= AN) break;
        const int vx = x0 - 1 + s % AW;                       // Lees-Edwards halo
        const int iy = LE ? wrapz(y0 - 1 + s / AW, ny) : 0;   // entries only
        const int i = rxy[e] + nx * ny * gz;
        if (NC == 3) {
          cp_async16(ringP4 + sl + s, Mb + S + i);  // {drho_s, dpsi_r, dpsi_b, dpsi_s}
          float *b = ringB + 3 * sl + s;
          cp_async4(b, DBn + i);
          cp_async4(b + AN, DBn + S + i);
          cp_async4(b + 2 * AN, DBn + 2 * S + i);
        } else if (LE && vx == -1) {  // sheared halo below x = 0
          cp_async8(ringP2 + sl + s, Lg.le_p[0] + iy + ny * gz);
        } else if (LE && vx == nx) {  // sheared halo above x = nx - 1
          cp_async8(ringP2 + sl + s, Lg.le_p[1] + iy + ny * gz);
        } else {
          cp_async8(ringP2 + sl + s, reinterpret_cast<const float2 *>(Mb) + i);
        }
      }
    };
    // own-site pulls of compute plane k into the stage; returns the own rock flag
    auto issue_pulls = [&](int k) -> bool {
      if (!act) return true;
      Nbr nb;
      const int gz = wrapz(z0 + k, nz);
      make_nbr(nb, gx, gy, gz, nx, ny, nz);
      const int self = noff<18, 1>(nb);
      if (ROCK && __ldg(RK + self) != 0) return true;
      if constexpr (LE) {
        LeYZ lw;
        make_leyz(lw, gy, gz, ny, nz);
#pragma unroll
        for (int c = 0; c < NC; ++c)
          pull_async_le<NT, ROCK>(F, S, c, nb, self, gx, nx, lw, Lg, ny * nz, mystage + c * 19 * NT, RK);
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) pull_async<ROCK, NT>(F, S, c, nb, self, RK, mystage + c * 19 * NT);
      }
      return false;
    };

    load_ring(0);
    load_ring(1);
    load_ring(2);
    cp_async_commit();
    bool skip = issue_pulls(0);
    cp_async_commit();

    for (int k = 0; k < zc; ++k) {
      if (k + 3 <= zc + 1) load_ring(k + 3);
      cp_async_commit();
      cp_async_wait<2>();  // ring planes up to k + 2 landed (this thread's copies)
      __syncthreads();     // ... and everybody's
      const int gzc = wrapz(z0 + k, nz);
      float Fx[NC][3];
      Nbr nb;
      int self = 0;
      if (act && !skip) {
        make_nbr(nb, gx, gy, gzc, nx, ny, nz);
        self = noff<18, 1>(nb);
        const int as = (tx + 1) + AW * (ty + 1);
        if constexpr (NC == 3) {
          force_ternary<AW, AW>(ringP4 + (k % RS) * AN, ringP4 + ((k + 1) % RS) * AN,
                                ringP4 + ((k + 2) % RS) * AN, DipAxes{ringB + 3 * (k % RS) * AN, AN},
                                DipAxes{ringB + 3 * ((k + 1) % RS) * AN, AN},
                                DipAxes{ringB + 3 * ((k + 2) % RS) * AN, AN}, as, as, Lg, psi0,
                                reinterpret_cast<float(*)[3]>(Fx));
        } else {
          // binary rings hold {dpsi_r, dpsi_b}
          const float2 *Qm = ringP2 + (k % RS) * AN, *Q0 = ringP2 + ((k + 1) % RS) * AN,
                       *Qp = ringP2 + ((k + 2) % RS) * AN;
          force_binary<AW, ROCK, float2, LE>(Qm, Q0, Qp, as, nb, RK, Lg, psi0,
                                             reinterpret_cast<float(*)[3]>(Fx), gx, gy, gzc);
        }
      }
      cp_async_wait<1>();  // this thread's pulls of plane k landed
      bool next_skip = true;
      if (act && !skip) {
        // the staged pulls, read once: red/blue on paired lanes, the surfactant alone
        float2 d01[19];
        float ds[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
          d01[q] = make_float2(mystage[q * NT], mystage[(19 + q) * NT]);
          if (NC == 3) ds[q] = mystage[(38 + q) * NT];
        }
        // the stage column is free again: the next plane's pulls fly during
        // this site's moments and BGK update
        if (k + 1 < zc) next_skip = issue_pulls(k + 1);
        float dr[NC], rho[NC], j[NC][3];
        {
          float2 r2, a0, a1, a2;
          own_moments2_reg(d01, r2, a0, a1, a2);
          dr[0] = r2.x, dr[1] = r2.y;
          j[0][0] = a0.x, j[1][0] = a0.y;
          j[0][1] = a1.x, j[1][1] = a1.y;
          j[0][2] = a2.x, j[1][2] = a2.y;
          if (NC == 3) own_moments<1>(ds, dr[NC - 1], j[NC - 1][0], j[NC - 1][1], j[NC - 1][2]);
#pragma unroll
          for (int c = 0; c < NC; ++c) rho[c] = rho0 + dr[c];
        }
        // stage-8 inflow boundaries act on the populations, not on the moments
        if constexpr (INF) inflow_site<NC>(d01, ds, Lg, gzc, nz);
        if (BODY) {
          const int x1 = gx + 1, y1 = gy + 1, z1 = gzc + 1;
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
        float vx[NC], vy[NC], vz[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float kf = Lg.tau[c] / (Lg.amass[c] * fmaxf(rho[c], 1.0e-8f));
          vx[c] = fmaf(kf, Fx[c][0], u0);
          vy[c] = fmaf(kf, Fx[c][1], u1);
          vz[c] = fmaf(kf, Fx[c][2], u2);
        }
        {
          bgk_update2(d01, make_float2(rho[0], rho[1]), make_float2(dr[0], dr[1]),
                      make_float2(vx[0], vx[1]), make_float2(vy[0], vy[1]), make_float2(vz[0], vz[1]),
                      make_float2(Lg.omega[0], Lg.omega[1]));
          float *fo = Fo + self;
#pragma unroll
          for (int q = 0; q < 19; ++q) {
            __stcs(fo + q * S, d01[q].x);
            __stcs(fo + (19 + q) * S, d01[q].y);
          }
          if constexpr (LE) {
            // the next step's pre-stream populations of the x boundary
            // planes, for its stage-6 halo kernel
            if (gx == 0 || gx == nx - 1) {
              float v0[19], v1[19];
#pragma unroll
              for (int q = 0; q < 19; ++q) v0[q] = d01[q].x, v1[q] = d01[q].y;
              le_store_boundary(Lg, 0, 0, gx, gy, gzc, v0);
              le_store_boundary(Lg, 0, 1, gx, gy, gzc, v1);
            }
          }
        }
        if (NC == 3) {
          bgk_update(ds, rho[NC - 1], dr[NC - 1], vx[NC - 1], vy[NC - 1], vz[NC - 1], Lg.omega[NC - 1]);
          float *fo = Fo + (size_t)38 * S + self;
#pragma unroll
          for (int q = 0; q < 19; ++q) __stcs(fo + q * S, ds[q]);
        }
      } else if (k + 1 < zc) {
        next_skip = issue_pulls(k + 1);
      }
      skip = next_skip;
      cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();  // the next tile refills ring slots 0..2
  }
}


// ---------------------------------------------------------------------------
// Lees-Edwards x-halos of the FP32 path (binary single lattices), two
// threads per (y, z), one per halo side, in FP64 from the FP32 deviations
// with the FP64 path's adjustment (le_adjust: the equilibrium shift by -/+
// 2 shear_u along z,
// the clipping rule and the top halo's reading of the adjusted bottom site,
// code/lb3d_bc_leesedwards.F90:147-1315).
//   k_le_pre32  (stage 6): pre-stream populations at x = nx - 1 / x = 0,
//               interpolated between z + e, z + e + 1 / z - e - 1, z - e,
//               written to le_h[0/1] as deviations; the pulls across the
//               x boundary read them.
//   k_le_post32 (stage 8): the same for the post-stream populations (each
//               pulled as the moments pass pulls it), reduced to the halo
//               densities and written to le_p[0/1] as psi deviations; the
//               collide pass's force stencil reads them.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double wq64(int q) { return q == 18 ? 1.0 / 3.0 : 1.0 / 36.0; }

template <int NC>
__global__ void k_le_pre32(DevParams P, LEStep L, const LatDesc *__restrict__ lat,
                           const float *__restrict__ f0, const float *__restrict__ f1, unsigned S) {
  const LatDesc &Lg = *lat;
  const int ny = Lg.ny, nz = Lg.nz, NP = ny * nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * NP) return;
  // threads [0, NP) build the bottom halo site of (y, z), threads [NP, 2 NP)
  // the top one (consecutive threads read consecutive y)
  const bool top = t >= NP;
  const int u = top ? t - NP : t;
  const int y = u % ny, z = u / ny;
  const double rho0 = (double)Lg.rho0, f = L.lefrac;
  (void)f0;
  (void)f1;
  (void)S;
  // the pre-stream populations of x = nx - 1 and x = 0 come from the compact
  // boundary planes
  double hb[NC][19];
  auto bottom = [&]() {
    const int ia = y + ny * wrapz(z + L.eoff, nz), ib = y + ny * wrapz(z + L.eoff + 1, nz);
    const float *B = Lg.le_b[0];
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q) {
        const double w = __dmul_rn(wq64(q), rho0);
        hb[c][q] = (1.0 - f) * ((double)B[(c * 19 + q) * NP + ia] + w) +
                   f * ((double)B[(c * 19 + q) * NP + ib] + w);
      }
    le_adjust<NC>(P, hb, hb, L.shear_u, -1.0);
  };
  if (!top) {
    bottom();
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q)
        Lg.le_h[0][(c * 19 + q) * NP + u] = (float)(hb[c][q] - __dmul_rn(wq64(q), rho0));
    return;
  }
  double ht[NC][19], df[NC][19];
  {
    const int ia = y + ny * wrapz(z - L.eoff - 1, nz), ib = y + ny * wrapz(z - L.eoff, nz);
    const float *B = Lg.le_b[1];
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q) {
        const double w = __dmul_rn(wq64(q), rho0);
        ht[c][q] = f * ((double)B[(c * 19 + q) * NP + ia] + w) +
                   (1.0 - f) * ((double)B[(c * 19 + q) * NP + ib] + w);
      }
  }
  // the top site's clipping rule reads the adjusted bottom site, which this
  // thread builds only when the rule applies
  const bool neg = le_adjust_df<NC>(P, ht, L.shear_u, +1.0, df);
  if (neg) bottom();
  le_adjust_apply<NC>(ht, hb, df, neg);
  for (int c = 0; c < NC; ++c)
    for (int q = 0; q < 19; ++q)
      Lg.le_h[1][(c * 19 + q) * NP + u] = (float)(ht[c][q] - __dmul_rn(wq64(q), rho0));
}

template <int NC>
__global__ void k_le_post32(DevParams P, LEStep L, const LatDesc *__restrict__ lat,
                            const float *__restrict__ f0, const float *__restrict__ f1, unsigned S) {
  const LatDesc &Lg = *lat;
  const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz, NP = ny * nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * NP) return;
  const bool top = t >= NP;
  const int u = top ? t - NP : t;
  const int y = u % ny, z = u / ny;
  const double rho0 = (double)Lg.rho0, f = L.lefrac;
  (void)f0;
  (void)f1;
  (void)S;
  // post-stream population q of component c at (x, yy, zz), x = nx - 1 or
  // 0: the moments pass left them in the compact boundary planes, pulled as
  // it pulls every site (across x from the stage-6 halo planes)
  auto post = [&](int c, int q, int x, int yy, int zz) -> double {
    const float v = Lg.le_b[x == 0 ? 3 : 2][(c * 19 + q) * NP + yy + ny * zz];
    return (double)v + __dmul_rn(wq64(q), rho0);
  };
  double hb[NC][19];
  auto bottom = [&]() {
    const int za = wrapz(z + L.eoff, nz), zb = wrapz(z + L.eoff + 1, nz);
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q)
        hb[c][q] = (1.0 - f) * post(c, q, nx - 1, y, za) + f * post(c, q, nx - 1, y, zb);
    le_adjust<NC>(P, hb, hb, L.shear_u, -1.0);
  };
  // psi(rho) - psi(rho0) = -e^{-rho0} expm1(-(rho - rho0)) of each
  // component's density at the halo site h
  const double em0 = exp(-rho0);
  auto dpsi = [&](const double h[NC][19], double d[NC]) {
    for (int c = 0; c < NC; ++c) {
      double a = 0.0;
#pragma unroll
      for (int q = 0; q < 19; ++q) a = a + h[c][q] * (double)gw(q);
      d[c] = -em0 * expm1(-(a - rho0));
    }
  };
  double d[NC];
  if (!top) {
    bottom();
    dpsi(hb, d);
    Lg.le_p[0][u] = make_float2((float)d[0], (float)d[1]);
    return;
  }
  double ht[NC][19], df[NC][19];
  {
    const int za = wrapz(z - L.eoff - 1, nz), zb = wrapz(z - L.eoff, nz);
    for (int c = 0; c < NC; ++c)
      for (int q = 0; q < 19; ++q)
        ht[c][q] = f * post(c, q, 0, y, za) + (1.0 - f) * post(c, q, 0, y, zb);
  }
  // the top site's clipping rule reads the adjusted bottom site, built here
  // only when the rule applies
  const bool neg = le_adjust_df<NC>(P, ht, L.shear_u, +1.0, df);
  if (neg) bottom();
  le_adjust_apply<NC>(ht, hb, df, neg);
  dpsi(ht, d);
  Lg.le_p[1][u] = make_float2((float)d[0], (float)d[1]);
}

// Fills the compact pre-stream boundary planes from the state (after an
// upload or a restored state); the collide passes keep them current after
// every step.
__global__ void k_le_gather32(const LatDesc *__restrict__ lat, const float *__restrict__ f0,
                              const float *__restrict__ f1, unsigned S) {
  const LatDesc &Lg = *lat;
  const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz, NP = ny * nz;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)Lg.nc * 19 * NP) return;
  const int cq = (int)(t / NP), yz = (int)(t % NP);
  const float *__restrict__ F = (Lg.parity ? f1 : f0) + Lg.base + (size_t)cq * S;
  const int row = nx * yz;  // y + ny * z
  Lg.le_b[0][t] = F[row + nx - 1];
  Lg.le_b[1][t] = F[row];
}
