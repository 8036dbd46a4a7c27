// hancock_kernel.cuh -- the 2D MUSCL-Hancock variant of the step
// (pmhd_config.order = PMHD_ORDER_HANCOCK): one predictor-corrector stage per
// step instead of the two SSPRK2 stages, so one pass over HBM per step.
//
// No 2D reference exists.  The scheme is the unsplit 2D extension of the
// reference's 1D Hancock predictor (src/mhd/mhd1d_cpu.cpp:203-235) on the
// 2D GLM solver's reconstruction, Riemann fluxes and update
// (src/mhd/mhd2d_glm_cpu.cpp:231-287): a cell's four reconstructed faces
// advance by half a step with its GLM flux differences in x and y and half a
// step of psi damping (a face whose evolved state is unusable keeps its
// unevolved state), one HLLD/HLL + GLM flux per interface from the evolved
// states, U += dt * rhs.  The oracle's or_run_hancock is the same sequence.
//
// A CTA owns a 32 x TYH tile: it loads the 36 x (TYH+4) ghosted region
// (plain coalesced loads; the SoA buffers keep ghost cells current), forms
// primitives, the evolved faces of the (34 x (TYH+2)) box around the tile,
// the tile's interface fluxes and the update, all staged in shared memory,
// and stores the tile with its ghost copies into the other buffer (the step
// of parity p reads buffer p, writes buffer p^1).  Policies as in the stage
// kernel: fp64, fp32, and mixed (binary64 storage, recovery and update;
// binary32 faces, predictor and fluxes).
// Included by kernels.cu after stage_kernels.cuh.

// Tile of one CTA.  The primitives are dead once the evolved faces exist,
// so the interface fluxes reuse their storage.  Binary64 faces use 32 x 4
// tiles: with 32 x 8 the tile needs ~200 KB and one CTA of 8 warps per SM
// (latency-bound); at 32 x 4 two CTAs fit (98 KB; binary32 faces: 98 KB or
// 82 KB at 32 x 8).  Registers are sized for two CTAs (128 per thread).
template <class S, class R>
struct HancockTile {
  static constexpr int TYH = sizeof(R) == 8 ? 4 : 8;
  static constexpr int MINB = 2;                   // resident CTAs the registers are sized for
  static constexpr int RW = TX + 4, RH = TYH + 4;  // region 36 x (TYH + 4)
  static constexpr int NR = RW * RH;
  static constexpr int BW = TX + 2, BH = TYH + 2;  // evolved-face box 34 x (TYH + 2)
  static constexpr int NB = BW * BH;
  static constexpr int NFX = (TX + 1) * TYH;       // x-interfaces of the tile
  static constexpr int NGY = TX * (TYH + 1);       // y-interfaces
  struct Fluxes {
    R Fx[NVAR][NFX];                               // interface fluxes
    R Gy[NVAR][NGY];
  };
  S U[NVAR][NR];
  union {
    R P[NVAR][NR];                                 // primitives
    Fluxes f;                                      // after the evolved faces
  };
  R H[4][NVAR][NB];                                // evolved faces: x-left, x-right, y-bottom, y-top
};
template <class Pol>
using HancockTileOf = HancockTile<typename Pol::S, typename Pol::R>;

// The binary32-face policies run the persistent TMA kernel; binary64 the
// one-tile-per-CTA kernel.
template <class Pol>
struct HancockPersistent {
  static constexpr bool on = sizeof(typename Pol::R) == 4;
};

// Prologue of a step: the stage-1 control update (zeroes the next step's
// speed slot when the step runs, carries the slots forward when it does not).
template <class Pol>
__global__ void hancock_begin_kernel(const __grid_constant__ Member m, const int p) {
  if (threadIdx.x != 0) return;
  const StepVals<Pol> v = step_values<Pol, 1>(m, p);
  member_bookkeeping<Pol, 1>(m, v, p);
}

// Scalars of one Hancock step: in the time type, and the predictor's in the
// face precision.
template <class Pol>
struct HancockScalars {
  typename Pol::TT dt, dx, dy, damping;
  typename Pol::R ch, hx, hy, hdamp;
  __device__ __forceinline__ HancockScalars(const Member& m, const StepVals<Pol>& v) {
    using TT = typename Pol::TT;
    using R = typename Pol::R;
    dt = v.dt;
    dx = (TT)m.dx;
    dy = (TT)m.dy;
    ch = v.ch;
    damping = (TT)ch / vmax((TT)m.alpha, (TT)1.0e-12);
    hx = (R)((TT)0.5 * dt / dx);
    hy = (R)((TT)0.5 * dt / dy);
    hdamp = (R)((TT)0.5 * dt * damping);
  }
};

// Primitives of region cells first, first + step, ... from the region's
// conserved states in shared memory, in the storage precision (the mixed
// policy's binary64 recovery), kept in the face precision.
template <class Pol>
__device__ __forceinline__ void hancock_recover(HancockTileOf<Pol>& s, const Phys<typename Pol::S>& phS, int first,
                                                int step) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  for (int q = first; q < HancockTileOf<Pol>::NR; q += step) {
    S U9[NVAR], P9[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) U9[k] = s.U[k][q];
    recover_cell<Pol>(U9, P9, phS);
#pragma unroll
    for (int k = 0; k < NVAR; k++) s.P[k][q] = (R)P9[k];
  }
}

// Evolved faces of the box cells (region rows 1..TYH+2, columns 1..34; the
// four box corners feed no interface of the tile).
template <class Pol>
__device__ __forceinline__ void hancock_faces(HancockTileOf<Pol>& s, const HancockScalars<Pol>& c0,
                                              const Phys<typename Pol::R>& ph, int first, int step) {
  using R = typename Pol::R;
  using HT = HancockTileOf<Pol>;
  constexpr int RW = HT::RW, BW = HT::BW, BH = HT::BH, NB = HT::NB;
  const R ch = c0.ch, hx = c0.hx, hy = c0.hy, hdamp = c0.hdamp;
  for (int q = first; q < NB; q += step) {
    const int br = q / BW, bc = q % BW;
    if ((br == 0 || br == BH - 1) && (bc == 0 || bc == BW - 1)) continue;
    const int c = (br + 1) * RW + (bc + 1);
    R P0[NVAR], Pw[NVAR], Pe[NVAR], Ps[NVAR], Pn[NVAR], Pl[NVAR], Pr[NVAR];
    R F[4][NVAR], Uf[4][NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      P0[k] = s.P[k][c];
      Pw[k] = s.P[k][c - 1];
      Pe[k] = s.P[k][c + 1];
      Ps[k] = s.P[k][c - RW];
      Pn[k] = s.P[k][c + RW];
    }
#if PMHD_FAST_FLUX
    // Performance build: the predictor's fluxes from the face primitives
    // (glm_phys_flux_prim), no recovery from the conserved faces.
    const R ch2 = ch * ch;
    recon_cell<R>(Pw, P0, Pe, Pl, Pr);
    prim9_to_state<R>(Pl, Uf[0], ph);
    prim9_to_state<R>(Pr, Uf[1], ph);
    glm_phys_flux_prim<R, 0>(Pl, Uf[0][EN], ch2, F[0]);
    glm_phys_flux_prim<R, 0>(Pr, Uf[1][EN], ch2, F[1]);
    recon_cell<R>(Ps, P0, Pn, Pl, Pr);
    prim9_to_state<R>(Pl, Uf[2], ph);
    prim9_to_state<R>(Pr, Uf[3], ph);
    glm_phys_flux_prim<R, 1>(Pl, Uf[2][EN], ch2, F[2]);
    glm_phys_flux_prim<R, 1>(Pr, Uf[3][EN], ch2, F[3]);
#else
    recon_cell<R>(Pw, P0, Pe, Pl, Pr);
    prim9_to_state<R>(Pl, Uf[0], ph);
    prim9_to_state<R>(Pr, Uf[1], ph);
    recon_cell<R>(Ps, P0, Pn, Pl, Pr);
    prim9_to_state<R>(Pl, Uf[2], ph);
    prim9_to_state<R>(Pr, Uf[3], ph);
    glm_phys_flux<R, 0>(Uf[0], ch, F[0], ph);
    glm_phys_flux<R, 0>(Uf[1], ch, F[1], ph);
    glm_phys_flux<R, 1>(Uf[2], ch, F[2], ph);
    glm_phys_flux<R, 1>(Uf[3], ch, F[3], ph);
#endif
    R corr[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) corr[k] = hx * (F[1][k] - F[0][k]) + hy * (F[3][k] - F[2][k]);
#pragma unroll
    for (int f = 0; f < 4; f++) {
      R h[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) h[k] = Uf[f][k] - corr[k];
      h[PSI] = h[PSI] - hdamp * Uf[f][PSI];
      const bool ok = PMHD_FAST_FLUX ? state_usable_fast<R>(h, ph) : state_usable<R>(h, ph);
#pragma unroll
      for (int k = 0; k < NVAR; k++) s.H[f][k][q] = ok ? h[k] : Uf[f][k];
    }
  }
}

// Interface fluxes of the tile at (i0, j0): x-interface (r, c) = between
// tile columns c-1 and c (c = 0..32) of tile row r; y-interface (r, c) =
// between tile rows r-1 and r (r = 0..TYH) of tile column c.  Stored over
// the (dead) primitives.  Adds the HLLD fallbacks of the domain's interfaces
// this tile counts to n_deg / n_np.
template <class Pol, bool HLLD>
__device__ __forceinline__ void hancock_fluxes(HancockTileOf<Pol>& s, const Member& m, int i0, int j0,
                                               typename Pol::R ch, const Phys<typename Pol::R>& ph, int first,
                                               int step, unsigned& n_deg, unsigned& n_np) {
  using R = typename Pol::R;
  using HT = HancockTileOf<Pol>;
  constexpr int BW = HT::BW, TYH = HT::TYH;
  R* Fx = &s.f.Fx[0][0];
  R* Gy = &s.f.Gy[0][0];
  const GlmK<R> gk = GlmK<R>::make(ch);
  for (int q = first; q < HT::NFX + HT::NGY; q += step) {
    R a[NVAR], b[NVAR], F[NVAR];
    int st;
    if (q < HT::NFX) {
      const int r = q / (TX + 1), c = q % (TX + 1);
      const int bl = (r + 1) * BW + c, br = bl + 1;  // box cells left / right of the interface
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        a[k] = s.H[1][k][bl];
        b[k] = s.H[0][k][br];
      }
      st = PMHD_FAST_FLUX ? glm_flux_fast_cons<R, 0>(a, b, gk, HLLD, F, ph) : glm_flux<R, 0>(a, b, ch, HLLD, F, ph);
#pragma unroll
      for (int k = 0; k < NVAR; k++) Fx[k * HT::NFX + q] = F[k];
    } else {
      const int g = q - HT::NFX, r = g / TX, c = g % TX;
      const int bb = r * BW + (c + 1), bt = bb + BW;  // box cells below / above
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        a[k] = s.H[3][k][bb];
        b[k] = s.H[2][k][bt];
      }
      st = PMHD_FAST_FLUX ? glm_flux_fast_cons<R, 1>(a, b, gk, HLLD, F, ph) : glm_flux<R, 1>(a, b, ch, HLLD, F, ph);
#pragma unroll
      for (int k = 0; k < NVAR; k++) Gy[k * HT::NGY + g] = F[k];
    }
    if (HLLD) {
      // Count each interface of the domain once: interface I (between
      // cells I-1 and I) by the tile with i0 <= I < i0 + 32, and I = nx by
      // the last tile; likewise in y.
      bool inside;
      if (q < HT::NFX) {
        const int r = q / (TX + 1), c = q % (TX + 1), I = i0 + c;
        inside = j0 + r < m.ny && I <= m.nx && (c < TX || I == m.nx);
      } else {
        const int g = q - HT::NFX, r = g / TX, c = g % TX, J = j0 + r;
        inside = i0 + c < m.nx && J <= m.ny && (r < TYH || J == m.ny);
      }
      if (inside) {
        n_deg += st == HLLD_FALLBACK_DEGENERATE ? 1u : 0u;
        n_np += st == HLLD_FALLBACK_NONPHYSICAL ? 1u : 0u;
      }
    }
  }
}

// Update of the tile cells first, first + step, ...: U += dt * rhs, store
// with ghost copies, usability (stateIsUsable with the policy's recovery)
// and the next step's signal speed into sp.  The cell's old state comes from
// the region in shared memory (UIN_SMEM) or from global memory.
template <class Pol, bool UIN_SMEM>
__device__ __forceinline__ void hancock_update(const HancockTileOf<Pol>& s, const Member& m, const StepVals<Pol>& v,
                                               const HancockScalars<Pol>& c0, const typename Pol::S* uin,
                                               typename Pol::S* uout, int i0, int j0,
                                               const Phys<typename Pol::S>& phS, const Phys<typename Pol::R>& ph,
                                               int first, int step, unsigned long long& sp) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using HT = HancockTileOf<Pol>;
  constexpr int RW = HT::RW, TYH = HT::TYH;
  const R* Fx = &s.f.Fx[0][0];
  const R* Gy = &s.f.Gy[0][0];
  for (int q = first; q < TX * TYH; q += step) {
    const int r = q / TX, c = q % TX;
    const int i = i0 + c, j = j0 + r;
    if (i >= m.nx || j >= m.ny) continue;
    const int rc = (r + 2) * RW + (c + 2);
    const size_t g = (size_t)(j + GHOST) * m.pitch + (i + GHOST);
    auto old = [&](int k) { return UIN_SMEM ? s.U[k][rc] : uin[(size_t)k * m.plane + g]; };
    S Un[NVAR];
    if constexpr (!Pol::kMixed) {
      const R idx = (R)m.inv_dx, idy = (R)m.inv_dy;
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        const R dfx = Fx[k * HT::NFX + r * (TX + 1) + c + 1] - Fx[k * HT::NFX + r * (TX + 1) + c];
        const R dgy = Gy[k * HT::NGY + (r + 1) * TX + c] - Gy[k * HT::NGY + r * TX + c];
        // The performance build multiplies by 1 / dx, 1 / dy (Member).
        R rhs = PMHD_FAST_FLUX ? -dfx * idx - dgy * idy : -dfx / c0.dx - dgy / c0.dy;
        const S u = old(k);
        if (k == PSI) rhs -= c0.damping * u;
        Un[k] = u + c0.dt * rhs;
      }
    } else {
      // Binary32 flux differences, binary64 scaling and accumulation (as
      // the mixed stage kernel).
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        const float dfx = Fx[k * HT::NFX + r * (TX + 1) + c + 1] - Fx[k * HT::NFX + r * (TX + 1) + c];
        const float dgy = Gy[k * HT::NGY + (r + 1) * TX + c] - Gy[k * HT::NGY + r * TX + c];
        double rhs = -(double)dfx * m.inv_dx - (double)dgy * m.inv_dy;
        const S u = old(k);
        if (k == PSI) rhs -= c0.damping * u;
        Un[k] = u + c0.dt * rhs;
      }
    }
    store_cell<S>(uout, m.plane, m.pitch, i, j, m.nx, m.ny, m.bc, Un);
    S P9[NVAR];
    recover_cell<Pol>(Un, P9, phS);
    if (!(Un[RHO] > rho_floor<S>()) || !prim9_usable<S>(P9)) {
      atomicMin(&m.ctrl->bad1, j * m.nx + i);
      m.ctrl->bad_step = v.step;
      m.ctrl->t_bad = (double)v.t;
    } else {
      R Pr[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) Pr[k] = (R)P9[k];
      const unsigned long long b =
          speed_bits((double)(PMHD_FAST_FLUX ? cell_speed_fast<R>(Pr, ph) : cell_speed<R>(Pr, ph)));
      sp = b > sp ? b : sp;
    }
  }
}

// Copies the tile cells first, first + step, ... (with their ghost copies)
// into the output buffer: a step past the stop condition.
template <class Pol>
__device__ __forceinline__ void hancock_carry(const Member& m, const typename Pol::S* uin, typename Pol::S* uout,
                                              int i0, int j0, int first, int step) {
  using S = typename Pol::S;
  for (int q = first; q < TX * HancockTileOf<Pol>::TYH; q += step) {
    const int i = i0 + q % TX, j = j0 + q / TX;
    if (i < m.nx && j < m.ny) {
      S c[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) c[k] = uin[(size_t)k * m.plane + (size_t)(j + GHOST) * m.pitch + (i + GHOST)];
      store_cell<S>(uout, m.plane, m.pitch, i, j, m.nx, m.ny, m.bc, c);
    }
  }
}

// Reduces a CTA's speed and fallback counts into the control block.
template <bool HLLD>
__device__ __forceinline__ void hancock_flush(const Member& m, int p, int lane, unsigned long long sp,
                                              unsigned n_deg, unsigned n_np) {
  sp = warp_max_u64(sp);
  if (HLLD) {
    n_deg = warp_sum_u32(n_deg);
    n_np = warp_sum_u32(n_np);
  }
  if (lane == 0) {
    if (sp) atomicMax(&m.ctrl->chbits[p ^ 1], sp);
    if (HLLD && n_deg) atomicAdd(&m.ctrl->degenerate, (unsigned long long)n_deg);
    if (HLLD && n_np) atomicAdd(&m.ctrl->nonphysical, (unsigned long long)n_np);
  }
}

// One CTA per tile, plain coalesced loads (the binary64 policy, whose 32 x 4
// tiles have no TMA descriptor).
template <class Pol, bool HLLD>
__global__ void __launch_bounds__(256, HancockTileOf<Pol>::MINB) hancock_kernel(const __grid_constant__ Member m, const int p) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using HT = HancockTileOf<Pol>;
  constexpr int RW = HT::RW, NR = HT::NR, TYH = HT::TYH;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  HT& s = *reinterpret_cast<HT*>(smem_raw);
  const Phys<S> phS = Phys<S>::make(m.gamma, m.tol);
  const Phys<R> ph = Phys<R>::make(m.gamma, m.tol);
  const S* __restrict__ uin = static_cast<const S*>(p ? m.u1 : m.u);
  S* __restrict__ uout = static_cast<S*>(p ? m.u : m.u1);
  const int ntx = (m.nx + TX - 1) / TX;
  const int i0 = (blockIdx.x % ntx) * TX, j0 = (blockIdx.x / ntx) * TYH;
  const StepVals<Pol> v = step_values<Pol, 2>(m, p);
  const int tid = threadIdx.x, lane = tid & 31;
  if (!v.active) {
    hancock_carry<Pol>(m, uin, uout, i0, j0, tid, blockDim.x);
    if (blockIdx.x == 0 && tid == 0) member_bookkeeping<Pol, 2>(m, v, p);
    return;
  }
  // Region: ghosted rows j0 .. j0+TYH+3, columns i0 .. i0+35 (clamped to the
  // allocation; cells past the domain's ghost ring feed no in-domain update).
  for (int q = tid; q < NR; q += blockDim.x) {
    int gj = j0 + q / RW, gi = i0 + q % RW;
    gj = gj < m.ny + 2 * GHOST ? gj : m.ny + 2 * GHOST - 1;
    gi = gi < m.nx + 2 * GHOST ? gi : m.nx + 2 * GHOST - 1;
#pragma unroll
    for (int k = 0; k < NVAR; k++) s.U[k][q] = uin[(size_t)k * m.plane + (size_t)gj * m.pitch + gi];
  }
  hancock_recover<Pol>(s, phS, tid, blockDim.x);  // each thread recovers the cells it loaded
  __syncthreads();
  const HancockScalars<Pol> c0(m, v);
  hancock_faces<Pol>(s, c0, ph, tid, blockDim.x);
  __syncthreads();
  unsigned n_deg = 0, n_np = 0;
  hancock_fluxes<Pol, HLLD>(s, m, i0, j0, c0.ch, ph, tid, blockDim.x, n_deg, n_np);
  __syncthreads();
  unsigned long long sp = 0;
  hancock_update<Pol, true>(s, m, v, c0, uin, uout, i0, j0, phS, ph, tid, blockDim.x, sp);
  hancock_flush<HLLD>(m, p, lane, sp, n_deg, n_np);
  if (blockIdx.x == 0 && tid == 0) member_bookkeeping<Pol, 2>(m, v, p);
}

// Persistent CTAs (the binary32-face policies): a tile's region arrives by
// TMA (the 36 x 12 x 9 box of the stage kernel's 32 x 8 descriptor, no
// multicast) and the next tile's load is started as soon as the region is
// recovered, so it lands while the faces, fluxes and update run; the update
// reads a cell's old state from global memory (an L2 hit).  Waits on the
// mbarrier are bounded and report a timeout instead of hanging.
template <class Pol, bool HLLD>
__global__ void __launch_bounds__(256, HancockTileOf<Pol>::MINB)
    hancock_persistent_kernel(const __grid_constant__ Member m, const int p) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using HT = HancockTileOf<Pol>;
  constexpr int TYH = HT::TYH;
  static_assert(TYH == 8, "the region box is the 32 x 8 stage-kernel descriptor's");
  constexpr int TI = kTileHeights[0] == 8 ? 0 : 1;  // index of the 32 x 8 descriptors in Member::tm
  extern __shared__ __align__(128) unsigned char smem_raw[];
  HT& s = *reinterpret_cast<HT*>(smem_raw);
  __shared__ __align__(8) uint64_t bar;
  const Phys<S> phS = Phys<S>::make(m.gamma, m.tol);
  const Phys<R> ph = Phys<R>::make(m.gamma, m.tol);
  const S* __restrict__ uin = static_cast<const S*>(p ? m.u1 : m.u);
  S* __restrict__ uout = static_cast<S*>(p ? m.u : m.u1);
  const int ntx = (m.nx + TX - 1) / TX;
  const int ntiles = ntx * ((m.ny + TYH - 1) / TYH);
  const StepVals<Pol> v = step_values<Pol, 2>(m, p);
  const int tid = threadIdx.x, lane = tid & 31;
  if (!v.active) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
      hancock_carry<Pol>(m, uin, uout, (t % ntx) * TX, (t / ntx) * TYH, tid, blockDim.x);
    if (blockIdx.x == 0 && tid == 0) member_bookkeeping<Pol, 2>(m, v, p);
    return;
  }
  const CUtensorMap* tm = &m.tm[TI][p ? 1 : 0];
  auto issue = [&](int t) {
    mbar_arrive_expect_tx(&bar, (uint32_t)(sizeof(S) * NVAR * HT::NR));
    tma_load_3d(&s.U[0][0], tm, &bar, (t % ntx) * TX, (t / ntx) * TYH, 0);
  };
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x);
  const HancockScalars<Pol> c0(m, v);
  unsigned n_deg = 0, n_np = 0;
  unsigned long long sp = 0;
  for (int t = blockIdx.x, it = 0; t < ntiles; t += gridDim.x, it++) {
    const int i0 = (t % ntx) * TX, j0 = (t / ntx) * TYH;
    // Also orders the previous tile's update (which reads the fluxes stored
    // over the primitives) before this tile's recovery.
    const bool got = __syncthreads_and(mbar_wait_bounded(&bar, (uint32_t)it & 1, kWaitIters));
    if (!got) {
      if (tid == 0) atomicExch(&m.ctrl->err, (int)DERR_TMA_TIMEOUT);
      mbar_wait_bounded(&bar, (uint32_t)it & 1, kWaitIters);  // let the copy land before leaving
      return;
    }
    hancock_recover<Pol>(s, phS, tid, blockDim.x);
    __syncthreads();
    if (tid == 0 && t + (int)gridDim.x < ntiles) {
      fence_proxy_async_smem();  // order the reads of the region before the async overwrite
      issue(t + gridDim.x);
    }
    hancock_faces<Pol>(s, c0, ph, tid, blockDim.x);
    __syncthreads();
    hancock_fluxes<Pol, HLLD>(s, m, i0, j0, c0.ch, ph, tid, blockDim.x, n_deg, n_np);
    __syncthreads();
    hancock_update<Pol, false>(s, m, v, c0, uin, uout, i0, j0, phS, ph, tid, blockDim.x, sp);
  }
  hancock_flush<HLLD>(m, p, lane, sp, n_deg, n_np);
  if (blockIdx.x == 0 && tid == 0) member_bookkeeping<Pol, 2>(m, v, p);
}
