// fp32_mfield.cuh -- the moment-field strategy (strategy 3) of the FP32
// deviation path, included by fp32_path.cu after fp32_split.cuh.
//
// Passes per step (binary lattices skip the second):
//
//   k_mf_moments: the pulls of every fluid site's 19*nc post-stream
//       deviations (code/lb3d_advection.F90:109-151 with the half-way
//       bounce-back of code/lb3d_bc_bounce.F90:53-90), read once from HBM,
//       reduced to the site's moment entries and written to halo-padded
//       moment fields:
//         ternary  MF1 = {drho_r, drho_b, drho_s, P_x}
//                  MF2 = {rho_b - rho_r, da}
//                  plain MFp = {P_y, P_z}, plain DS = drho_s
//         binary   MF1 = {drho_r, drho_b, P_x, P_y}, plain MFp = {P_z, 0}
//       where P = sum_c amass_c omega_c j_c is the weighted momentum of
//       code/lb3d_collision.F90:560-587 and da the advected dipole flux
//       (code/lb3d_advection.F90:137-148).
//   k_mf_dipole (ternary): the dipole relaxation (code/lb3d_collision.F90:
//       296-403) of every site from MF2 with a one-site halo, written to the
//       dipole state, and the site's force-stencil entry DD = {a, dpsi_s}
//       with a = d psi(rho_s) (the product every neighbour's force term
//       uses, code/lb3d_force_shanchen.F90:283) to a halo-padded field.
//   k_mf_collide: psi deviations of red and blue on the tile plus a
//       one-site halo from MF1, the Shan-Chen force
//       (code/lb3d_force_shanchen.F90:127-330) from them and (ternary) DD and
//       the own dipole, the body force and the velocities, and the
//       populations of the next step.
//
// Lees-Edwards lattices (binary, no walls) run the same passes between the
// FP32 path's halo kernels: the moments pass pulls across the sheared x
// boundary from the stage-6 halo planes and the collide pass takes the psi
// deviations of the x-halo columns from the stage-8 planes
// (code/lb3d_bc_leesedwards.F90:147-1315).
//
// The padded fields carry two extra sites on each side in x and y; the
// sites on an x or y boundary also write their periodic image into the
// padding, so a tile plus its one-site halo is one dense box.  The dipole and
// collide passes march a column tile in z and receive every plane of their
// input fields as one TMA box per field (cp.async.bulk.tensor), two planes
// ahead of use, on one mbarrier per ring slot, with one CTA barrier per plane.
//
// The populations are read once per step, by the moments pass: the collide
// pass writes the equilibrium, which is the BGK update
// (code/lb3d_collision.F90:258-284) when every component relaxes fully
// (omega_c = 1, tau_c = 1: the populations' own values drop out); the
// strategy is offered for such lattices only.  Every quantity is evaluated
// with the expressions and in the order of the split strategies, so strategy
// 3 equals them bit for bit (up to the sign of zero).
//
// The tensor maps cover this GPU's own moment field only and the loads do
// not multicast.

// ---- TMA and mbarrier primitives (PTX) -----------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on one phase of an mbarrier: false if it did not complete
// within the iteration limit (each try_wait suspends for a bounded time).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
  for (int i = 0; i < (1 << 21); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// One 4-D tiled box global -> shared, completing on `bar` (no multicast).
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tmap, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const void *tmap) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// Programmatic dependent launch between the passes: each pass lets the next
// one launch once all its CTAs are running (the next pass's CTAs then take
// the SM resources its finished CTAs free and run their set-up), and waits
// for the previous grid to complete, with its memory visible, before it
// reads anything that grid or an earlier one wrote (the lattice
// descriptors, the fields, the populations).  Without the launch attribute
// both are no-ops.
__device__ __forceinline__ void pdl_launch_next() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
__device__ __forceinline__ void pdl_wait_previous() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Geometry shared by the passes: padded fields with MF_PAD extra sites on
// each side in x and y (one of them used as the periodic image), ring boxes
// of the tile plus a one-site halo.
constexpr int MF_PAD = 2;
template <int NC, int TX, int TY>
struct MfGeom {
  static constexpr int NT = TX * TY;
  static constexpr int AW = TX + 2, AN = AW * (TY + 2);  // ring box, one-site halo
  static constexpr int BOX_BYTES = 16 * AN;
  // a TMA destination in shared memory starts on a 128-byte boundary: the
  // boxes of one slot sit FIELD bytes apart
  static constexpr int FIELD = (BOX_BYTES + 127) / 128 * 128;
  // dipole pass: one MF2 box per slot, 5 slots
  static constexpr int D_SLOT = (FIELD + 1023) / 1024 * 1024;
  static constexpr int D_RS = 8;
  static constexpr int D_SMEM = D_RS * D_SLOT + 1024;
  // collide pass: MF1 (+ DD) boxes per slot, 6 slots; psi ring of 4 planes
  static constexpr int NF = NC == 3 ? 2 : 1;
  static constexpr int C_SLOT = (NF * FIELD + 1023) / 1024 * 1024;
  static constexpr int C_RS = 8, PR = 4;  // powers of two: cheap slot indices
  static constexpr int PSI_BYTES = PR * AN * 8;
  static constexpr int C_SMEM = C_RS * C_SLOT + PSI_BYTES + 1024;
  static constexpr int AHEAD = 2;  // planes loaded ahead of use
  static constexpr int C_MINB = NT >= 256 ? 2 : 3;
};

static_assert(MfGeom<3, 32, 8>::FIELD % 128 == 0 && MfGeom<3, 32, 8>::D_SLOT % 1024 == 0 &&
                  MfGeom<3, 32, 8>::C_SLOT % 1024 == 0 && MfGeom<3, 32, 8>::C_SLOT >= 2 * MfGeom<3, 32, 8>::FIELD,
              "TMA destinations of the ring slots must be 128-byte aligned");

// Writes a float4 entry of site (gx, gy, gz) to a padded field, and its
// periodic image when the site lies on an x or y boundary (nx, ny >= 2).
__device__ __forceinline__ void mf_put(float4 *__restrict__ M, float4 e, int gx, int gy, int gz, int nx,
                                       int ny) {
  const int XP = nx + 2 * MF_PAD, YP = ny + 2 * MF_PAD;
  const int xi = gx == 0 ? nx : (gx == nx - 1 ? -1 : gx);
  const int yi = gy == 0 ? ny : (gy == ny - 1 ? -1 : gy);
  const size_t zoff = (size_t)XP * YP * gz;
  M[zoff + (gx + MF_PAD) + (size_t)XP * (gy + MF_PAD)] = e;
  if (xi != gx) M[zoff + (xi + MF_PAD) + (size_t)XP * (gy + MF_PAD)] = e;
  if (yi != gy) M[zoff + (gx + MF_PAD) + (size_t)XP * (yi + MF_PAD)] = e;
  if (xi != gx && yi != gy) M[zoff + (xi + MF_PAD) + (size_t)XP * (yi + MF_PAD)] = e;
}

// ---------------------------------------------------------------------------
// Moments pass: one thread per tile site, marching the tile's z range; the
// previous dipoles (ternary) stream through a four-plane ring with a
// one-site halo, refilled with cp.async one plane ahead, for the advected
// flux.  Binary lattices need no ring and their threads never wait on each
// other.
// ---------------------------------------------------------------------------
template <int NC, int TX, int TY, bool ROCK, bool NARROW, bool LE = false>
__global__ void __launch_bounds__(TX *TY, 1024 / (TX * TY))
    k_mf_moments(const LatDesc *__restrict__ lats, const Tile *__restrict__ tiles, int ntiles,
                 const float *f0, const float *f1, const float *db0, const float *db1,
                 const uint8_t *__restrict__ rock, unsigned S, float4 *__restrict__ MF1,
                 float4 *__restrict__ MF2, float2 *__restrict__ MFp, float *__restrict__ DS) {
  constexpr int NT = TX * TY, DW = TX + 2, DN = DW * (TY + 2), DR = 4;
  extern __shared__ float4 smd[];  // previous dipoles [DR][DN] (ternary)
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  pdl_launch_next();
  pdl_wait_previous();
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    const LatDesc &Lg = lats[T.lat];
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    const int par = Lg.parity;
    const float *__restrict__ F = par ? f1 : f0;
    const float *__restrict__ DBi = (NC == 3) ? (par ? db1 : db0) : nullptr;
    const float rho0 = Lg.rho0;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool act = gx < nx && gy < ny;
    const bool le_edge = x0 == 0 || x0 + TX >= nx;  // the tile holds x = 0 or x = nx - 1
    // the ring of previous dipoles: plane z0 - 1 + j in slot j % DR
    auto load_db_plane = [&](int j) {
      const int gz = wrapz(z0 - 1 + j, nz);
      float *dst = reinterpret_cast<float *>(smd + (j % DR) * DN);
      for (int s = tid; s < DN; s += NT) {
        const int ix = wrapz(x0 - 1 + s % DW, nx), iy = wrapz(y0 - 1 + s / DW, ny);
        const int i = ix + nx * (iy + ny * gz);
        cp_async4(dst + 4 * s, DBi + i);
        cp_async4(dst + 4 * s + 1, DBi + S + i);
        cp_async4(dst + 4 * s + 2, DBi + 2 * S + i);
      }
    };
    if (NC == 3) {
      load_db_plane(0);
      load_db_plane(1);
      load_db_plane(2);
      cp_async_commit();
    }
    for (int it = 0; it < zc; ++it) {
      if (NC == 3) {
        if (it + 3 <= zc + 1) load_db_plane(it + 3);
        cp_async_commit();
        cp_async_wait<1>();  // planes up to it + 2 landed (this thread's copies)
        __syncthreads();     // ... and everybody's
      }
      bool fluid = act;
      Nbr nb;
      int self = 0, gz = 0;
      if (act) {
        gz = wrapz(z0 + it, nz);
        make_nbr(nb, gx, gy, gz, nx, ny, nz);
        self = noff<18, 1>(nb);
        // rock sites are never collided and their entries are never read
        // (the force stencil takes the rock colour there): no pulls
        if (ROCK) fluid = __ldg(rock + self) == 0;
      }
      if (LE && ROCK && act && !fluid && le_edge) {
        // a rock site on the sheared boundary keeps its (zero) populations:
        // they go to the post-stream boundary plane as they are
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          float d[19];
#pragma unroll
          for (int q = 0; q < 19; ++q) d[q] = __ldg(F + (size_t)(c * 19 + q) * S + self);
          le_store_boundary(Lg, 2, c, gx, gy, gz, d);
        }
      }
      if (fluid) {
        float dr[NC], jm[NC][3];
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
        const float4 *Dm = smd + (it % DR) * DN, *D0 = smd + ((it + 1) % DR) * DN,
                     *Dp = smd + ((it + 2) % DR) * DN;
        LeYZ lw;
        if constexpr (LE) make_leyz(lw, gy, gz, ny, nz);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          float d[19];
          // Lees-Edwards lattices pull across x = 0 and x = nx - 1 from the
          // sheared halo planes of this step; tiles away from those planes
          // pull as periodic lattices do
          if (LE && le_edge) {
            pull_comp_le<NARROW, ROCK>(F, S, c, nb, self, gx, nx, lw, Lg, ny * nz, d, rock);
            le_store_boundary(Lg, 2, c, gx, gy, gz, d);  // for the stage-8 halo kernel
          } else {
            pull_comp<ROCK, false, NARROW>(F, S, c, nb, self, rock, d);
          }
          own_moments<1>(d, dr[c], jm[c][0], jm[c][1], jm[c][2]);
          if (NC == 3 && c == 2) {
            // da = sum_q (n_s(x - c_q, q) g_q) db(x - c_q) + n_s(x, rest) db(x)
            const int ds0 = (tx + 1) + DW * (ty + 1);
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
        // the weighted momentum of the common velocity, summed as the
        // collide passes sum it
        float p0 = 0.f, p1 = 0.f, p2 = 0.f;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float am = Lg.amass[c] * Lg.omega[c];
          p0 = fmaf(am, jm[c][0], p0);
          p1 = fmaf(am, jm[c][1], p1);
          p2 = fmaf(am, jm[c][2], p2);
        }
        if (NC == 3) {
          MFp[self] = make_float2(p1, p2);
          DS[self] = dr[NC - 1];
          mf_put(MF1, make_float4(dr[0], dr[1], dr[NC - 1], p0), gx, gy, gz, nx, ny);
          mf_put(MF2, make_float4(dr[1] - dr[0], a0, a1, a2), gx, gy, gz, nx, ny);
        } else {
          MFp[self] = make_float2(p2, 0.0f);
          mf_put(MF1, make_float4(dr[0], dr[1], p0, p1), gx, gy, gz, nx, ny);
        }
      }
      if (NC == 3) __syncthreads();  // the next iteration refills a ring slot read here
    }
    if (NC == 3) cp_async_wait<0>();
  }
}

// Issues the TMA boxes of one plane into a ring slot (1024-byte aligned):
// one or two float4 fields of the tile plus a one-site halo, at padded
// coordinates (x0 + 1, y0 + 1), the second box `field` bytes (a multiple of
// 128) after the first, on the slot's mbarrier.
__device__ __forceinline__ void mf_issue(unsigned char *slot, int box_bytes, int field, const CUtensorMap *ma,
                                         const CUtensorMap *mb, int x0, int y0, int zw, uint64_t *bar) {
  mbar_expect_tx(bar, (mb ? 2 : 1) * box_bytes);
  tma_load_4d(slot, ma, 0, x0 + MF_PAD - 1, y0 + MF_PAD - 1, zw, bar);
  if (mb) tma_load_4d(slot + field, mb, 0, x0 + MF_PAD - 1, y0 + MF_PAD - 1, zw, bar);
}

// 1024-byte aligned start of the dynamic shared memory (TMA destinations).
__device__ __forceinline__ unsigned char *mf_smem_base(unsigned char *raw) {
  return reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(raw) + 1023) &
                                           ~static_cast<uintptr_t>(1023));
}

// ---------------------------------------------------------------------------
// Dipole pass (ternary).  Plane m of a tile is moment-field plane z0 - 1 + m
// (m = 0 .. zc + 1); iteration j waits for plane j of MF2 and relaxes the
// dipoles of plane j - 1 on the tile, dipole_site's arithmetic on the
// {rho_b - rho_r, da} entries as the split strategies run it.  *err receives
// LB3DC_ETIMEOUT if a plane never arrives.
// ---------------------------------------------------------------------------
template <int TX, int TY>
__global__ void __launch_bounds__(TX *TY, 1024 / (TX * TY))
    k_mf_dipole(const __grid_constant__ CUtensorMap tm2, const LatDesc *__restrict__ lats,
                const Tile *__restrict__ tiles, int ntiles, float *db0, float *db1,
                const float *__restrict__ DS, float4 *__restrict__ DD, int *err) {
  using G = MfGeom<3, TX, TY>;
  constexpr int AW = G::AW, RS = G::D_RS, AHEAD = G::AHEAD;
  extern __shared__ unsigned char smraw_[];
  unsigned char *ring = mf_smem_base(smraw_);
  __shared__ __align__(8) uint64_t bars[RS];
  __shared__ LatDesc sLat;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  if (tid == 0) {
    for (int s = 0; s < RS; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    tma_prefetch_desc(&tm2);
  }
  __syncthreads();
  pdl_launch_next();
  pdl_wait_previous();
  auto box = [&](unsigned g) { return reinterpret_cast<const float4 *>(ring + (g % RS) * G::D_SLOT); };
  unsigned gbase = 0, issued = 0, waited = 0;
  bool failed = false;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    if (tid == 0) sLat = lats[T.lat];
    __syncthreads();
    const LatDesc &Lg = sLat;
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    float *__restrict__ DBo = Lg.parity ? db0 : db1;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    const int npl = zc + 2;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool act = gx < nx && gy < ny;
    auto issue = [&](int m) {
      const unsigned g = gbase + (unsigned)m;
      mf_issue(ring + (g % RS) * G::D_SLOT, G::BOX_BYTES, G::FIELD, &tm2, nullptr, x0, y0,
               wrapz(z0 - 1 + m, nz), &bars[g % RS]);
    };
    if (tid == 0)
      for (int m = 0; m < AHEAD && m < npl; ++m) issue(m);
    issued = gbase + (unsigned)(AHEAD < npl ? AHEAD : npl);
    // the own surfactant density deviation of the plane relaxed next,
    // loaded one iteration ahead
    float drs = 0.0f, drs_next = 0.0f;
    for (int j = 0; j < npl; ++j) {
      const unsigned g = gbase + (unsigned)j;
      const bool ok = mbar_wait_bounded(&bars[g % RS], (g / RS) & 1u);
      // every thread is past iteration j - 1, which last read the slot
      // refilled below, and plane j has landed
      if (__syncthreads_or(!ok)) {
        failed = true;
        waited = g;
        break;
      }
      if (j + AHEAD < npl) {
        if (tid == 0) issue(j + AHEAD);
        issued = g + AHEAD + 1;
      }
      if (act && j >= 1 && j <= zc) drs_next = __ldg(DS + gx + nx * (gy + ny * wrapz(z0 + j - 1, nz)));
      if (j >= 2 && act) {
        const int as = (tx + 1) + AW * (ty + 1);
        const int gz = wrapz(z0 + j - 2, nz);
        const float3 d = dipole_site<AW>(box(g - 2), box(g - 1), box(g), as, Lg, Lg.rho0, drs);
        const int i = gx + nx * (gy + ny * gz);
        __stcs(DBo + i, d.x);
        __stcs(DBo + (size_t)Lg.nx * Lg.ny * Lg.nz + i, d.y);
        __stcs(DBo + 2 * (size_t)Lg.nx * Lg.ny * Lg.nz + i, d.z);
        const float pse = -Lg.em0 * expm1f(-drs);
        const float ps = Lg.psi0 + pse;
        const float2 a01 = mul2(make_float2(d.x, d.y), f2(ps));
        mf_put(DD, make_float4(a01.x, a01.y, d.z * ps, pse), gx, gy, gz, nx, ny);
      }
      drs = drs_next;
    }
    if (failed) break;
    gbase += (unsigned)npl;
    __syncthreads();  // sLat and the ring are reused by the next tile
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, LB3DC_ETIMEOUT);
      for (unsigned g = waited; g < issued; ++g) mbar_wait_bounded(&bars[g % RS], (g / RS) & 1u);
    }
    __syncthreads();
  }
}

// force_ternary with the neighbours' a = d (psi0 + dpsi_s) precomputed by the
// dipole pass: psi entries {dpsi_r, dpsi_b}, a entries {a, dpsi_s}; the own
// dipole d given.  The same operations in the same order as force_ternary.
template <int W>
__device__ __forceinline__ void force_ternary_pre(const float2 *Pm, const float2 *P0, const float2 *Pp,
                                                  const float4 *Am, const float4 *A0, const float4 *Ap,
                                                  int ap, float3 dd, const LatDesc &Lg, float psi0,
                                                  float Fx[3][3]) {
  float2 FB[3] = {f2(0.f), f2(0.f), f2(0.f)}, M01[3] = {f2(0.f), f2(0.f), f2(0.f)};
  float2 TQ[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};
  float2 SA01 = f2(0.f);
  float SA2 = 0.f, V[3] = {0, 0, 0}, M2[3] = {0, 0, 0}, SG = 0.f;
#pragma unroll
  for (int q = 0; q < 18; ++q) {
    const float2 *Pq = cz(q) == 1 ? Pp : (cz(q) == -1 ? Pm : P0);
    const float4 *Aq = cz(q) == 1 ? Ap : (cz(q) == -1 ? Am : A0);
    const float g = (float)gw(q);
    const int c[3] = {cx(q), cy(q), cz(q)};
    const float2 e = Pq[ap + cx(q) + W * cy(q)];
    const float4 av = Aq[ap + cx(q) + W * cy(q)];
    const float2 a01 = make_float2(av.x, av.y);
    const float a2 = av.z;
    const float a[3] = {a01.x, a01.y, a2};
    float ac = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (c[k]) ac = fmaf((float)c[k], a[k], ac);
    const float Gq = g * (e.y - e.x);
    const float g8 = 8.0f * g;
    SG += Gq;
    SA01 = fma2(f2(g), a01, SA01);
    SA2 = fmaf(g, a2, SA2);
    const float2 ezy = make_float2(e.y, e.x);
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
  const float d[3] = {dd.x, dd.y, dd.z};
  const float2 own = P0[ap];
  const float psr = psi0 + own.x, psb = psi0 + own.y, pss = psi0 + A0[ap].w;
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

// ---------------------------------------------------------------------------
// Collide pass.  Plane m of a tile is field plane z0 - 1 + m (m = 0 ..
// zc + 1).  Iteration j (0 .. zc + 2) waits for plane j, computes its psi
// deviations on the tile plus a one-site halo into the psi ring, and the
// force and equilibrium of plane j - 2 on the tile (whose psi planes were
// computed in earlier iterations), so one CTA barrier per plane separates
// the ring's writers from its readers.  *err receives LB3DC_ETIMEOUT if a
// plane never arrives.
// ---------------------------------------------------------------------------
template <int NC, int TX, int TY, bool ROCK, bool BODY, bool LE = false>
__global__ void __launch_bounds__(TX *TY, MfGeom<NC, TX, TY>::C_MINB)
    k_mf_collide(const __grid_constant__ CUtensorMap tm1, const __grid_constant__ CUtensorMap tmd,
                 const LatDesc *__restrict__ lats, const Tile *__restrict__ tiles, int ntiles, float *f0,
                 float *f1, const float *db0, const float *db1, const uint8_t *__restrict__ rock, unsigned S,
                 const float2 *__restrict__ MFp, int *err) {
  using G = MfGeom<NC, TX, TY>;
  constexpr int AW = G::AW, AN = G::AN, RS = G::C_RS, PR = G::PR, AHEAD = G::AHEAD;
  extern __shared__ unsigned char smraw_[];
  unsigned char *ring = mf_smem_base(smraw_);
  unsigned char *psiring = ring + RS * G::C_SLOT;
  __shared__ __align__(8) uint64_t bars[RS];
  __shared__ LatDesc sLat;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  constexpr int NT = G::NT;
  if (tid == 0) {
    for (int s = 0; s < RS; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    tma_prefetch_desc(&tm1);
    if (NC == 3) tma_prefetch_desc(&tmd);
  }
  __syncthreads();
  pdl_launch_next();
  pdl_wait_previous();
  auto box = [&](unsigned g, int f) {
    return reinterpret_cast<const float4 *>(ring + (g % RS) * G::C_SLOT + f * G::FIELD);
  };
  unsigned gbase = 0, issued = 0, waited = 0;
  bool failed = false;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile T = tiles[t];
    if (tid == 0) sLat = lats[T.lat];
    __syncthreads();
    const LatDesc &Lg = sLat;
    const int nx = Lg.nx, ny = Lg.ny, nz = Lg.nz;
    float *__restrict__ Fo = Lg.parity ? f0 : f1;
    const float *__restrict__ DBn = Lg.parity ? db0 : db1;
    const float psi0 = Lg.psi0, em0 = Lg.em0;
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0, zc = T.zc;
    const int npl = zc + 2;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool act = gx < nx && gy < ny;
    const bool le_edge = x0 == 0 || x0 + TX >= nx;  // the tile holds x = 0 or x = nx - 1
    auto issue = [&](int m) {
      const unsigned g = gbase + (unsigned)m;
      mf_issue(ring + (g % RS) * G::C_SLOT, G::BOX_BYTES, G::FIELD, &tm1, NC == 3 ? &tmd : nullptr, x0,
               y0, wrapz(z0 - 1 + m, nz), &bars[g % RS]);
    };
    if (tid == 0)
      for (int m = 0; m < AHEAD && m < npl; ++m) issue(m);
    issued = gbase + (unsigned)(AHEAD < npl ? AHEAD : npl);
    // the own plain momentum entry of the plane collided next, loaded one
    // iteration ahead
    float2 op = make_float2(0.0f, 0.0f), op_next = op;
    float3 dnow = make_float3(0.f, 0.f, 0.f), dnext = dnow;
    for (int j = 0; j <= npl; ++j) {
      const unsigned g = gbase + (unsigned)j;
      bool ok = true;
      if (j < npl) ok = mbar_wait_bounded(&bars[g % RS], (g / RS) & 1u);
      // every thread is past iteration j - 1 (the psi slot written below and
      // the ring slot refilled below were last read there) and plane j landed
      if (__syncthreads_or(!ok)) {
        failed = true;
        waited = g;
        break;
      }
      if (j + AHEAD < npl) {
        if (tid == 0) issue(j + AHEAD);
        issued = g + AHEAD + 1;
      }
      // ---- psi deviations of plane j on the tile plus a one-site halo
      if (j < npl) {
        const float4 *M1 = box(g, 0);
        for (int s = tid; s < AN; s += NT) {
          if (LE && le_edge) {
            // the sheared halo columns take the psi deviations of the
            // stage-8 halo planes (binary lattices)
            const int vx = x0 - 1 + s % AW;
            if (vx == -1 || vx == nx) {
              const int iy = wrapz(y0 - 1 + s / AW, ny), iz = wrapz(z0 - 1 + j, nz);
              reinterpret_cast<float2 *>(psiring)[(j % PR) * AN + s] = Lg.le_p[vx < 0 ? 0 : 1][iy + ny * iz];
              continue;
            }
          }
          const float4 e = M1[s];
          reinterpret_cast<float2 *>(psiring)[(j % PR) * AN + s] =
              make_float2(-em0 * expm1f(-e.x), -em0 * expm1f(-e.y));
        }
      }
      // ---- force and equilibrium of plane mc = j - 2 on the tile
      const int mc = j - 2;
      if (act && mc + 1 >= 1 && mc + 1 <= zc) {
        const int in = gx + nx * (gy + ny * wrapz(z0 + mc, nz));
        op_next = __ldg(MFp + in);
        if (NC == 3) dnext = make_float3(__ldg(DBn + in), __ldg(DBn + S + in), __ldg(DBn + 2 * S + in));
      }
      if (mc >= 1 && mc <= zc && act) {
        const int gz = wrapz(z0 - 1 + mc, nz);
        Nbr nb;
        make_nbr(nb, gx, gy, gz, nx, ny, nz);
        const int self = noff<18, 1>(nb);
        bool own_rock = false;
        if (ROCK) own_rock = __ldg(rock + self) != 0;
        if (!own_rock) {
          const int ap = (tx + 1) + AW * (ty + 1);
          const unsigned gc = gbase + (unsigned)mc;
          float Fx[NC][3];
          if constexpr (NC == 3) {
            const float2 *P2 = reinterpret_cast<const float2 *>(psiring);
            force_ternary_pre<AW>(P2 + ((mc + PR - 1) % PR) * AN, P2 + (mc % PR) * AN,
                                  P2 + ((mc + 1) % PR) * AN, box(gc - 1, 1), box(gc, 1), box(gc + 1, 1), ap,
                                  dnow, Lg, psi0, reinterpret_cast<float(*)[3]>(Fx));
          } else {
            const float2 *P2 = reinterpret_cast<const float2 *>(psiring);
            force_binary<AW, ROCK, float2, LE>(P2 + ((mc + PR - 1) % PR) * AN, P2 + (mc % PR) * AN,
                                               P2 + ((mc + 1) % PR) * AN, ap, nb, rock, Lg, psi0,
                                               reinterpret_cast<float(*)[3]>(Fx), gx, gy, gz);
          }
          // own densities and weighted momentum
          const float4 o1 = box(gc, 0)[ap];
          float dr[NC], rho[NC], pp[3];
          if constexpr (NC == 3) {
            dr[0] = o1.x, dr[1] = o1.y, dr[NC - 1] = o1.z;
            pp[0] = o1.w, pp[1] = op.x, pp[2] = op.y;
          } else {
            dr[0] = o1.x, dr[1] = o1.y;
            pp[0] = o1.z, pp[1] = o1.w, pp[2] = op.x;
          }
#pragma unroll
          for (int c = 0; c < NC; ++c) rho[c] = Lg.rho0 + dr[c];
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
          float rt = 0.f;
#pragma unroll
          for (int c = 0; c < NC; ++c) rt = fmaf(Lg.amass[c] * Lg.omega[c], rho[c], rt);
          const float irt = 1.0f / fmaxf(rt, 1.0e-8f);
          const float u0 = pp[0] * irt, u1 = pp[1] * irt, u2 = pp[2] * irt;
          float vx[NC], vy[NC], vz[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const float kf = Lg.tau[c] / (Lg.amass[c] * fmaxf(rho[c], 1.0e-8f));
            vx[c] = fmaf(kf, Fx[c][0], u0);
            vy[c] = fmaf(kf, Fx[c][1], u1);
            vz[c] = fmaf(kf, Fx[c][2], u2);
          }
          float *fo = Fo + self;
          // a site on the sheared x boundary also writes the next step's
          // pre-stream boundary plane for its stage-6 halo kernel, with the
          // same equilibrium values (one store sequence for every lane; at
          // x = 0 and x = nx - 1 both when the lattice is one site wide)
          float *b0 = nullptr;
          int NP = 0;
          if (LE && (gx == 0 || gx == nx - 1)) {
            NP = ny * nz;
            b0 = Lg.le_b[gx == nx - 1 ? 0 : 1] + gy + ny * gz;
          }
          eq_store2(fo, fo + (size_t)19 * S, S, make_float2(rho[0], rho[1]), make_float2(dr[0], dr[1]),
                    make_float2(vx[0], vx[1]), make_float2(vy[0], vy[1]), make_float2(vz[0], vz[1]),
                    make_float2(Lg.omega[0], Lg.omega[1]), b0, b0 ? b0 + 19 * NP : nullptr, (unsigned)NP);
          if (LE && gx == 0 && gx == nx - 1) {
            float *b1 = Lg.le_b[1] + gy + ny * gz;
            eq_store2(b1, b1 + 19 * NP, (unsigned)NP, make_float2(rho[0], rho[1]), make_float2(dr[0], dr[1]),
                      make_float2(vx[0], vx[1]), make_float2(vy[0], vy[1]), make_float2(vz[0], vz[1]),
                      make_float2(Lg.omega[0], Lg.omega[1]));
          }
          if (NC == 3)
            eq_store(fo + (size_t)38 * S, S, rho[NC - 1], dr[NC - 1], vx[NC - 1], vy[NC - 1], vz[NC - 1],
                     Lg.omega[NC - 1]);
        }
      }
      op = op_next;
      dnow = dnext;
    }
    if (failed) break;
    gbase += (unsigned)npl;
    __syncthreads();  // sLat and the rings are reused by the next tile
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, LB3DC_ETIMEOUT);
      for (unsigned g = waited; g < issued; ++g) mbar_wait_bounded(&bars[g % RS], (g / RS) & 1u);
    }
    __syncthreads();
  }
}
