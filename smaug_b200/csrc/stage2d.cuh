// stage2d.cuh -- fused 2D stage kernel, included by stage2d.cu.
//
// One launch evaluates the reference's whole spatial operator for a 32x8
// tile of interior cells and writes the stage result, its ghost images and
// the per-dimension fast-speed maxima.  Term by term it follows the launch
// order of the reference's step (src/iosmaug.c:631-835); the arithmetic of
// each term is the reference's, with divisions by rho_t and by the cell
// width replaced by multiplications with per-cell / per-line reciprocals
// (agreement with the reference stays at rounding level, ~1e-16 relative).
//
// Two precision forms share the code (template MIX):
//   FP64   every value and every operation in double;
//   mixed  perturbation fields stored in float (stage buffers, and the base
//          state as a float high/low pair), backgrounds in double; fluxes,
//          the pressure recovery p_t = (g-1)(e - m^2/2rho_t) - ..., the
//          CFL speeds, the stage sums and the RK4 accumulator in double;
//          the hyperdiffusion coefficient and sources (q, nu, their
//          differences) in float, with q itself formed in double.
//
// Shared memory: the tile's state (6 perturbation fields in the storage
// type, the background fields in double) on the tile + 3-cell halo, 1/rho_t,
// the tile's cell widths and their reciprocals, then one union of phase
// scratch:
//   flux phase:  5 flux arrays on the tile +-2 cells along the direction
//                (+ 2 velocity arrays when background fields are present)
//   hyperdiffusion phase: q of one field on the whole region (shared by the
//                passes of both directions), the nu ratio on the tile
//                extended by one cell along the direction, two cross-term
//                arrays on the tile +-1 across.
#pragma once

// (included inside namespace smaug)
namespace s2 {
// flux arrays: the tile +-2 along the direction (+-3 along dim 0 for the
// 6th-order derivative, which a 2D build of the reference applies along dim 0
// only: its dir-1 USE_DORDER3 branch is overwritten by the 4th-order form,
// src/gradops.cu:536-544)
template <bool O6>
__host__ __device__ constexpr int fsz() {
  return (TX + (O6 ? 6 : 4)) * TY > TX * (TY + 4) ? (TX + (O6 ? 6 : 4)) * TY : TX * (TY + 4);
}
constexpr int RSZ = (TX + 1) * (TY + 2) > (TX + 2) * (TY + 1) ? (TX + 1) * (TY + 2) : (TX + 2) * (TY + 1);
constexpr int NSZ = TX * (TY + 2) > (TX + 2) * TY ? TX * (TY + 2) : (TX + 2) * TY;
constexpr int HYP = RC + RSZ + 2 * NSZ;  // q, ratio, two cross-term arrays
template <bool MIX, bool O6 = false>
__host__ __device__ constexpr size_t union_bytes() {
  return (5 * fsz<O6>() * sizeof(double)) > HYP * sizeof(typename Form<MIX>::H)
             ? 5 * fsz<O6>() * sizeof(double)
             : HYP * sizeof(typename Form<MIX>::H);
}
template <bool BG, bool MIX, bool O6 = false>
__host__ __device__ constexpr size_t smem_bytes() {
  return 6 * RC * sizeof(typename Form<MIX>::S) +
         sizeof(double) * ((BG ? 6 : 0) * RC + RC + 2 * (RX + RY)) + union_bytes<MIX, O6>();
}
}  // namespace s2

template <bool BG, bool MIX>
struct T2 {
  using ST = typename Form<MIX>::S;
  ST* S;         // [6][RC] perturbation state
  double* G;     // [4][RC] background fields (BG only)
  double* R;     // [RC] 1/rho_t
  double* V;     // [2][RC] velocities (BG only)
  double* dl0;   // [RX] widths along x of the region columns
  double* dl1;   // [RY]
  double* rd0;   // [RX] reciprocals
  double* rd1;   // [RY]
  void* U;       // union scratch
  int x0, y0;
  bool inner;    // the staged region lies inside the grid and off its pads
  // field f of the reference numbering at region cell l, in double
  __device__ __forceinline__ double v(int f, int l) const {
    if (f < 6) return (double)S[f * RC + l];
    return BG ? G[(f - 6) * RC + l] : 0.0;
  }
};

// fluxes along D of rho, m1, m2, e and the B component across D at region
// cell l (src/centdiff1.cu:51-197, src/centdiff2.cu:203-323):
//   F_rho = m_D (= m_D rho'/rho_t + rho_b m_D/rho_t)
//   F_m_c = v_D m_c + delta_cD p_t - (B'_c Bb_D + Bb_c B'_D) - B'_c B'_D
//   F_e   = v_D (e + p_t + e_b) - (B'_D (Bb.m) + Bb_D (B'.m) + B'_D (B'.m)) / rho_t
//   F_B_c = v_D (B'_c + Bb_c) - v_c (B'_D + Bb_D)
template <bool BG, bool MIX, int D>
__device__ __forceinline__ void flux_at(const T2<BG, MIX>& T, double gamma, int l, double* F) {
  const double m1 = T.v(M1, l), m2 = T.v(M2, l);
  const double e = T.v(EN, l), b1 = T.v(B1, l), b2 = T.v(B2, l);
  double eb = 0, bb1 = 0, bb2 = 0;
  if (BG) {
    eb = T.v(EB, l);
    bb1 = T.v(BB1, l);
    bb2 = T.v(BB2, l);
  }
  const double r = T.R[l];
  const double md = D == 0 ? m1 : m2;
  const double vd = md * r;
  // computept3 (src/dervfields.cu:107-153)
  const double pt = (gamma - 1.0) * (e - 0.5 * (m1 * m1 + m2 * m2) * r) -
                    (gamma - 2.0) * ((b1 * bb1 + b2 * bb2) + 0.5 * (b1 * b1 + b2 * b2));
  const double bd = D == 0 ? b1 : b2, bbd = D == 0 ? bb1 : bb2;
  F[0] = md;
  // momentum components
  F[1] = vd * m1 + (D == 0 ? pt : 0.0) - (b1 * bbd + bb1 * bd) - b1 * bd;
  F[2] = vd * m2 + (D == 1 ? pt : 0.0) - (b2 * bbd + bb2 * bd) - b2 * bd;
  // energy
  const double bbm = bb1 * m1 + bb2 * m2, bm = b1 * m1 + b2 * m2;
  F[3] = vd * (e + pt + eb) - (bd * bbm + bbd * bm + bd * bm) * r;
  // B component across D
  if (D == 0)
    F[4] = vd * (b2 + bb2) - (m2 * r) * (b1 + bb1);
  else
    F[4] = vd * (b1 + bb1) - (m1 * r) * (b2 + bb2);
}

// q of a hyperdiffusion pass at region cell l (src/hyperdifvisc1r.cu:1225-1253),
// formed in double
template <bool BG, bool MIX, int KIND, int COMP>
__device__ __forceinline__ double hq_at(const T2<BG, MIX>& T, int l) {
  if (KIND == 0) return T.v(RHO, l);
  if (KIND == 1) {
    const double m1 = T.v(M1, l), m2 = T.v(M2, l);
    const double b1 = T.v(B1, l), b2 = T.v(B2, l);
    return T.v(EN, l) - 0.5 * ((b1 * b1 + b2 * b2) + (m1 * m1 + m2 * m2) * T.R[l]);
  }
  if (KIND == 2) return T.v(M1 + COMP, l) * T.R[l];
  return T.v(B1 + COMP, l);
}

// the same q from global memory (stray pad source cell)
template <typename ST, int KIND, int COMP, bool CG = false>
__device__ __forceinline__ double hq_global(const ST* u, const double* bg, long nc, long c) {
  auto ld = [&](long i) { return CG ? (double)__ldcg(u + i) : (double)u[i]; };
  const double rho = ld(0 * nc + c), rhob = bg[1 * nc + c];
  if (KIND == 0) return rho;
  const double r = 1.0 / (rho + rhob);
  if (KIND == 1) {
    const double m1 = ld(1 * nc + c), m2 = ld(2 * nc + c);
    const double b1 = ld(4 * nc + c), b2 = ld(5 * nc + c);
    return ld(3 * nc + c) - 0.5 * ((b1 * b1 + b2 * b2) + (m1 * m1 + m2 * m2) * r);
  }
  if (KIND == 2) return ld((1 + COMP) * nc + c) * r;
  return ld((4 + COMP) * nc + c);
}

// (A) q of one hyperdiffusion field on the whole staged region, with the
// reference's pads: index -1 along an axis holds the copy of index 5
// (bc_hyperdifl), index n the stray tmp6 store of hyperdifvisc1r_parallel
// (source table B.padsrc).  The passes of both directions read it.
template <bool BG, bool MIX, int KIND, int COMP, bool CG = false>
__device__ __forceinline__ void stage_q2(const T2<BG, MIX>& T, const KParams& P, const KBufs& B,
                                         int tid) {
  using HT = typename Form<MIX>::H;
  using ST = typename Form<MIX>::S;
  HT* Q = static_cast<HT*>(T.U);
  const int n0 = P.n0, n1 = P.n1;
  const long nc = P.ncell;
  if (T.inner) {
    for (int u = tid; u < RXU * RY; u += NTHREADS) {
      const int r = RXU == RX ? u : (u / RXU) * RX + u % RXU;
      Q[r] = (HT)hq_at<BG, MIX, KIND, COMP>(T, r);
    }
    __syncthreads();
    return;
  }
  for (int u = tid; u < RXU * RY; u += NTHREADS) {
    const int lx = u % RXU, ly = u / RXU, r = ly * RX + lx;
    const int ci = T.x0 - HALO + lx, cj = T.y0 - HALO + ly;
    const bool inx = ci >= 0 && ci < n0, iny = cj >= 0 && cj < n1;
    double q = 0.0;
    if (inx && iny) {
      q = hq_at<BG, MIX, KIND, COMP>(T, r);
    } else if (iny) {
      if (ci == -1) {
        q = hq_at<BG, MIX, KIND, COMP>(T, r + 6);
      } else if (ci == n0) {
        const int src = B.padsrc[0][cj];
        if (src >= 0) q = hq_global<ST, KIND, COMP, CG>(static_cast<const ST*>(B.uin), B.bg, nc, src);
      }
    } else if (inx) {
      if (cj == -1) {
        q = hq_at<BG, MIX, KIND, COMP>(T, r + 6 * RX);
      } else if (cj == n1) {
        const int src = B.padsrc[1][ci];
        if (src >= 0) q = hq_global<ST, KIND, COMP, CG>(static_cast<const ST*>(B.uin), B.bg, nc, src);
      }
    }
    Q[r] = (HT)q;
  }
  __syncthreads();
}

// One hyperdiffusion pass on staged q: field kind (0 rho, 1 energy,
// 2 momentum, 3 B), component COMP, direction DIM.
//
// nu_r and nu_l (hyperdifvisc2-4) are ratios of windowed maxima of the third
// differences D3 and first differences D1 of q:
//   nu_r(i) = dl(i) cmax chyp max D3(i-1..i+1) / max D1(i-2..i+2)
//   nu_l(i) = dl(i) cmax chyp max D3(i-2..i)   / max D1(i-3..i+1)
// (0 where the denominator is 0, and 0 outside [2, n-3] in every
// dimension).  The windows of nu_l(i) are those of nu_r(i-1), so one ratio
// R(i) = max D3 / max D1 per cell serves both: nu_r(i) = c(i) R(i),
// nu_l(i) = c(i) R(i-1).
template <bool BG, bool MIX, int KIND, int COMP, int DIM>
__device__ __forceinline__ void hyper_pass(const T2<BG, MIX>& T, const KParams& P, const KBufs& B,
                                           int tid, bool active, int lxo, int lyo, int gi, int gj,
                                           double dt, const double* cin, double* out) {
  using HT = typename Form<MIX>::H;
  constexpr int SX = (DIM == 0), SY = (DIM == 1);
  constexpr int QFIELD = (KIND == 0) ? RHO : (KIND == 1) ? EN : (KIND == 2) ? M1 + COMP : B1 + COMP;
  constexpr bool CROSS = (KIND == 2 && COMP != DIM) || (KIND == 3);
  const int n0 = P.n0, n1 = P.n1;
  const int nd = DIM == 0 ? n0 : n1;
  const HT* Q = static_cast<const HT*>(T.U);  // region-indexed q
  HT* RR = static_cast<HT*>(T.U) + RC;         // ratio area
  HT* C3 = RR + s2::RSZ;                       // cross-term arrays (nu area)
  HT* C4 = C3 + s2::NSZ;
  constexpr int SQ = DIM == 0 ? 1 : RX;        // stride along DIM in Q
  // ratio area: the tile along DIM extended by one cell below, the tile
  // across (+-1 when cross terms need it)
  constexpr int exR = DIM == 0 ? TX + 1 : (CROSS ? TX + 2 : TX);
  constexpr int eyR = DIM == 0 ? (CROSS ? TY + 2 : TY) : TY + 1;
  constexpr int oxR = DIM == 0 ? HALO - 1 : (CROSS ? HALO - 1 : HALO);
  constexpr int oyR = DIM == 0 ? (CROSS ? HALO - 1 : HALO) : HALO - 1;
  constexpr int SR = DIM == 0 ? 1 : exR;       // stride along DIM in RR
  // nu area: the tile along DIM, +-1 across
  constexpr int exN = (DIM == 0) ? TX : TX + 2, eyN = (DIM == 0) ? TY + 2 : TY;
  constexpr int oxN = (DIM == 0) ? HALO : HALO - 1, oyN = (DIM == 0) ? HALO - 1 : HALO;
  auto ri = [&](int lx, int ly) { return (ly - oyR) * exR + (lx - oxR); };
  auto ni = [&](int lx, int ly) { return (ly - oyN) * exN + (lx - oxN); };
  const HT coef = (HT)(cin[DIM] * P.chyp[QFIELD]);

  // (B) R = max D3(i-1..i+1) / max D1(i-2..i+2) from q(i-2..i+3)
  for (int r = tid; r < exR * eyR; r += NTHREADS) {
    const int lx = oxR + r % exR, ly = oyR + r / exR;
    const int l = ly * RX + lx;
    HT q[6];
#pragma unroll
    for (int s = 0; s < 6; s++) q[s] = Q[l + (s - 2) * SQ];
    HT t4 = 0, t5 = 0;
#pragma unroll
    for (int k = 0; k < 3; k++)
      t4 = hmax0(t4, (HT)fabs((HT)3 * (q[k + 2] - q[k + 1]) - (q[k + 3] - q[k])));
#pragma unroll
    for (int k = 0; k < 5; k++) t5 = hmax0(t5, (HT)fabs(q[k + 1] - q[k]));
    RR[r] = (t5 > 0) ? hdiv(t4, t5) : (HT)0;
  }
  __syncthreads();
  // (C) cross-term arrays (hyperdifmomsourcene2-4 / hyperdifbsourcene1b-4)
  if (CROSS) {
    for (int r = tid; r < exN * eyN; r += NTHREADS) {
      const int lx = oxN + r % exN, ly = oyN + r / exN;
      const int ci = T.x0 - HALO + lx, cj = T.y0 - HALO + ly;
      HT c3 = 0, c4 = 0;
      if (T.inner || (ci > 0 && ci < n0 - 1 && cj > 0 && cj < n1 - 1)) {
        const int a = DIM == 0 ? ci : cj;
        const int l = ly * RX + lx;
        // grad13n along DIM of q
        HT g = ((Q[l + SQ] - Q[l - SQ]) * (HT)(DIM == 0 ? T.rd0[lx] : T.rd1[ly])) * (HT)0.5;
        if ((P.bt[DIM] != 0) && zero1n(a, nd)) g = 0;
        HT nsum = 0;
        if (T.inner || (ci >= 2 && ci <= n0 - 3 && cj >= 2 && cj <= n1 - 3)) {
          const int rr = ri(lx, ly);
          const HT c = (HT)(DIM == 0 ? T.dl0[lx] : T.dl1[ly]) * coef;
          nsum = c * RR[rr] + c * RR[rr - SR];
        }
        if (KIND == 2) {
          const HT tau = (g * nsum) * (HT)0.25;
          c3 = (HT)(T.v(RHO, l) + T.v(RHOB, l)) * tau;
          c4 = tau * (HT)T.v(M1 + DIM, l);
        } else {
          const HT t3 = (g * nsum) * (HT)0.5;
          c3 = t3;
          c4 = t3 * (HT)T.v(B1 + DIM, l);
        }
      }
      C3[r] = c3;
      C4[r] = c4;
    }
    __syncthreads();
  }
  // (D) sources at the tile cells (all inside [2, n-3])
  if (active) {
    const int a = DIM == 0 ? gi : gj;
    const int l = lyo * RX + lxo;
    const int rr = ri(lxo, lyo);
    const int nidx = ni(lxo, lyo);
    const HT c = (HT)(DIM == 0 ? T.dl0[lxo] : T.dl1[lyo]) * coef;
    const HT nur = c * RR[rr], nul = c * RR[rr - SR];
    const HT rdl = (HT)(DIM == 0 ? T.rd0[lxo] : T.rd1[lyo]);
    const HT qc = Q[l], qp = Q[l + SQ], qm = Q[l - SQ];
    HT gr = (qp - qc) * rdl;   // grad1r3n
    HT gl = (qc - qm) * rdl;   // grad1l3n
    if ((P.bt[DIM] != 0) && zero1n(a, nd)) { gr = 0; gl = 0; }
    constexpr int SL = SX + SY * RX;  // region stride along DIM
    if (KIND == 0) {
      out[RHO] = out[RHO] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 1) {
      out[EN] = out[EN] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 2) {
      // hyperdifmomsource1-3a (src/hyperdifmomsource1.cu:17-511), ii0 = COMP
      const double rb0 = T.v(RHOB, l), rbm = T.v(RHOB, l - SL), rbp = T.v(RHOB, l + SL);
      const double r0 = T.v(RHO, l);
      const HT t2 = (HT)((r0 + rb0 + T.v(RHO, l - SL) + rbm) * 0.5);
      const HT t3 = (HT)((r0 + rb0 + T.v(RHO, l + SL) + rbp) * 0.5);
      const double mf = T.v(M1 + COMP, l);
      const HT t5 = (HT)((mf + T.v(M1 + COMP, l - SL)) * 0.5);
      const HT t6 = (HT)((mf + T.v(M1 + COMP, l + SL)) * 0.5);
      const double dm = (double)(((t3 * nur * gr - t2 * nul * gl) * rdl) * (HT)0.5);
      const double de = (double)(((t6 * nur * gr - t5 * nul * gl) * rdl) * (HT)0.5);
      out[M1 + COMP] = out[M1 + COMP] + dt * dm;
      out[EN] = out[EN] + dt * de;
      if (COMP == DIM) {
        out[M1 + COMP] = out[M1 + COMP] + dt * dm;
        out[EN] = out[EN] + dt * de;
      } else {
        // hyperdifmomsourcene5-6a: d/dx_COMP of (rho_t tau) and (tau m_DIM)
        constexpr int FS = (COMP == 0) ? 1 : exN;  // stride across in the nu area
        const int af = COMP == 0 ? gi : gj;
        const HT rdf = (HT)(COMP == 0 ? T.rd0[lxo] : T.rd1[lyo]);
        HT g7 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
        HT g8 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
        if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) { g7 = 0; g8 = 0; }
        out[M1 + DIM] = out[M1 + DIM] + dt * (double)g7;
        out[EN] = out[EN] + dt * (double)g8;
      }
    } else {
      // B component COMP diffused along DIM: hyperdifbsourcene (sb=-1) then
      // hyperdifbsource (sb=+1)
      constexpr int FS = (COMP == 0) ? 1 : exN;
      const int af = COMP == 0 ? gi : gj;
      const HT rdf = (HT)(COMP == 0 ? T.rd0[lxo] : T.rd1[lyo]);
      HT g4 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
      HT g6 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
      if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) { g4 = 0; g6 = 0; }
      out[B1 + DIM] = out[B1 + DIM] - dt * (double)g4;
      out[EN] = out[EN] - dt * (double)g6;
      const HT t2 = (qc + qm) * (HT)0.5, t3 = (qc + qp) * (HT)0.5;
      const double dB = (double)((gr * nur - gl * nul) * rdl);
      const double de = (double)((t3 * gr * nur - t2 * gl * nul) * rdl);
      out[B1 + COMP] = out[B1 + COMP] + dt * dB;
      out[EN] = out[EN] + dt * de;
    }
  }
  __syncthreads();
}

// Bulk tensor copy of the staged state of tile (bx, by) -- the 6 fields in
// the storage type into s, and (gdst non-null) the 4 background fields
// (with background fields) or rho_b alone (without) into gdst -- completing
// on tt.bar.  Cells outside the grid read 0.  The region starts at column
// x0 - HALO = XORG - HALO + bx TX, which the TMA-staged kernel's tile origin
// makes a multiple of 32 cells (the copy's x offset must be 16-byte aligned).
template <bool BG, bool MIX>
__device__ __forceinline__ void tma_stage_issue(void* s, void* gdst, const TmaTile& tt, int bx, int by) {
  using ST = typename Form<MIX>::S;
  const unsigned bytes = (s ? 6 * RC * sizeof(ST) : 0) + (gdst ? (BG ? 4 : 1) * RC * sizeof(double) : 0);
  const int x = XORG - HALO + bx * TX, y = 2 - HALO + by * TY;
  fence_proxy_async_smem();
  mbar_expect_tx(tt.bar, bytes);
  if (s) tma_load_3d(s, tt.ms, x, y, 0, tt.bar);
  if (gdst) tma_load_3d(gdst, tt.mg, x, y, BG ? 0 : 1, tt.bar);
}

// The stage for tile (bx, by) of one grid; the single-run kernels below and
// in stage2d_tma.cu and the batched kernel (batch.cu) call it.  TMA = 1: the
// state arrives by bulk tensor copy (tt: the block's copy schedule), and the
// copy of the block's next tile is issued once this tile's staged arrays
// are dead, so that it overlaps the stores.  TMA = 2 (no background
// fields): two state buffers; the copy of the next tile's state goes to the
// other buffer as soon as this tile's copy has arrived, so that it overlaps
// the whole tile, and its rho_b (into 1/rho_t's array, dead by then) during
// the stores -- two arrivals on the barrier per phase.  Returns false when a copy did
// not complete in time (FLAG_TMA_TIMEOUT set; the block must stop).
template <int MODE, bool BG, bool MIX, bool O6 = false, bool CG = false, int TMA = 0>
__device__ __forceinline__ bool stage2d_body(const KParams& P, const KBufs& B, int bx, int by,
                                             const TmaTile* tt = nullptr) {
  using ST = typename Form<MIX>::S;
  extern __shared__ double smem[];
  T2<BG, MIX> T;
  unsigned char* sp = reinterpret_cast<unsigned char*>(smem);
  // the copy boxes land on 128-byte boundaries (the launch adds the slack);
  // an offset added to the shared array itself, so that the compiler still
  // addresses the tile arrays as shared memory (a pointer rebuilt from an
  // integer would make every tile access a generic one)
  if constexpr (TMA != 0) sp += (128u - (smem_u32(sp) & 127u)) & 127u;
  static_assert(TMA != 2 || !BG, "double-buffered staging without background fields only");
  T.S = reinterpret_cast<ST*>(sp);
  sp += 6 * RC * sizeof(ST);
  ST* const s_other = reinterpret_cast<ST*>(sp);  // TMA = 2: the second state buffer
  if constexpr (TMA == 2) {
    if (tt->parity) T.S = s_other;
    sp += 6 * RC * sizeof(ST);
  }
  T.G = reinterpret_cast<double*>(sp);
  sp += (BG ? 4 * RC : 0) * sizeof(double);
  T.R = reinterpret_cast<double*>(sp);
  T.V = T.R + RC;
  T.dl0 = T.V + (BG ? 2 * RC : 0);
  T.dl1 = T.dl0 + RX;
  T.rd0 = T.dl1 + RY;
  T.rd1 = T.rd0 + RX;
  T.U = T.rd1 + RY;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  T.x0 = XORG + bx * TX;
  T.y0 = 2 + by * TY;
  const int n0 = P.n0, n1 = P.n1;
  // region columns x0-3 .. x0-3+RX-1 (rows y0-3 .. y0+TY+2) inside
  // [0, n-1]: no bounds or pad checks in the staging, flux and cross-term
  // loops
  T.inner = bx >= 1 && by >= 1 && T.x0 - HALO + RX <= n0 && T.y0 + TY + HALO <= n1;
  const long nc = P.ncell;
  const ST* uin = static_cast<const ST*>(B.uin);

  // ---- stage the tile, 1/rho_t, the metric -------------------------------
  if constexpr (TMA) {
    // every thread waits on the barrier (one waiter and a block barrier
    // measured 2.5 % slower at 4096^2)
    void* const gdst = BG ? static_cast<void*>(T.G) : static_cast<void*>(T.R);
    if (tt->issue_self && tid == 0) {
      tma_stage_issue<BG, MIX>(T.S, gdst, *tt, bx, by);
      if (TMA == 2) mbar_arrive(tt->bar);  // the phase's second arrival
    }
    const bool ok = mbar_wait(tt->bar, tt->parity, TMA_WAIT_NS);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(B.flags, FLAG_TMA_TIMEOUT);
        mbar_wait(tt->bar, tt->parity, TMA_WAIT_NS);  // the copy in flight
      }
      __syncthreads();
      return false;
    }
    if constexpr (TMA == 2) {
      // the other buffer's last reader, the previous tile, is done
      if (tid == 0 && tt->nbx >= 0) {
        ST* const s0 = reinterpret_cast<ST*>(reinterpret_cast<unsigned char*>(s_other) - 6 * RC * sizeof(ST));
        tma_stage_issue<BG, MIX>(tt->parity ? s0 : s_other, nullptr, *tt, tt->nbx, tt->nby);
      }
    }
    for (int u = tid; u < RXU * RY; u += NTHREADS) {
      const int lx = u % RXU, ly = u / RXU, r = ly * RX + lx;
      const int gi = T.x0 - HALO + lx, gj = T.y0 - HALO + ly;
      const bool in = T.inner || (gi >= 0 && gi < n0 && gj >= 0 && gj < n1);
      const double rho = (double)T.S[r];  // 0 outside the grid (the copy's fill)
      double rhob;
      if (BG) {
        if (!in) T.G[1 * RC + r] = 1.0;
        rhob = T.G[1 * RC + r];
      } else {
        rhob = in ? T.R[r] : 1.0;
      }
      const double rinv = 1.0 / (rho + rhob);
      T.R[r] = rinv;
      if (BG) {
        T.V[r] = (double)T.S[M1 * RC + r] * rinv;
        T.V[RC + r] = (double)T.S[M2 * RC + r] * rinv;
      }
    }
  } else {
  for (int u = tid; u < RXU * RY; u += NTHREADS) {
    const int lx = u % RXU, ly = u / RXU, r = ly * RX + lx;
    const int gi = T.x0 - HALO + lx, gj = T.y0 - HALO + ly;
    const bool in = T.inner || (gi >= 0 && gi < n0 && gj >= 0 && gj < n1);
    const long c = (long)gj * n0 + gi;
    double rho = 0.0, rhob = 1.0;
#pragma unroll
    for (int f = 0; f < 6; f++) {
      const ST v = in ? ldin<CG>(uin + f * nc + c) : (ST)0;
      T.S[f * RC + r] = v;
      if (f == 0) rho = v;
    }
    if (BG) {
#pragma unroll
      for (int f = 0; f < 4; f++) {
        const double v = in ? __ldg(B.bg + f * nc + c) : (f == 1 ? 1.0 : 0.0);
        T.G[f * RC + r] = v;
        if (f == 1) rhob = v;
      }
    } else {
      rhob = in ? __ldg(B.bg + 1 * nc + c) : 1.0;
      if (!in) rho = 0.0;
    }
    const double rinv = 1.0 / (rho + rhob);
    T.R[r] = rinv;
    if (BG) {
      T.V[r] = (double)T.S[M1 * RC + r] * rinv;
      T.V[RC + r] = (double)T.S[M2 * RC + r] * rinv;
    }
  }
  }
  for (int r = tid; r < RX + RY; r += NTHREADS) {
    if (r < RX) {
      const int gi = T.x0 - HALO + r;
      const double d = (gi >= 0 && gi < n0) ? B.delx[0][gi] : 1.0;
      T.dl0[r] = d;
      T.rd0[r] = 1.0 / d;
    } else {
      const int gj = T.y0 - HALO + (r - RX);
      const double d = (gj >= 0 && gj < n1) ? B.delx[1][gj] : 1.0;
      T.dl1[r - RX] = d;
      T.rd1[r - RX] = 1.0 / d;
    }
  }

  // ---- dt of this step and stage time ----------------------------------
  const double cin[2] = {ldsc<CG>(B.cmax_in), ldsc<CG>(B.cmax_in + 1)};
  double dt, tstage;
  if (B.stage == 0) {
    dt = device_dt(P, cin, ldsc<CG>(B.dt_prev), 2);
    if (bx == 0 && by == 0 && tid == 0) {
      *B.dt_new = dt;
      *B.t_new = ldsc<CG>(B.t_prev) + dt;
      B.cmax_clear[0] = B.cmax_clear[1] = B.cmax_clear[2] = 0ull;
    }
    tstage = ldsc<CG>(B.t_prev);
  } else {
    dt = ldsc<CG>(B.dt_new);
    tstage = ldsc<CG>(B.t_prev) + (B.stage == 3 ? dt : 0.5 * dt);
    if (bx == 0 && by == 0 && tid == 0)
      B.cmax_clear[0] = B.cmax_clear[1] = B.cmax_clear[2] = 0ull;
  }
  __syncthreads();

  const int lxo = tx + HALO, lyo = ty + HALO, lo = lyo * RX + lxo;
  const int gi = T.x0 + tx, gj = T.y0 + ty;
  const bool active = (XORG >= 2 || gi >= 2) && gi <= n0 - 3 && gj <= n1 - 3;
  const long co = active ? (long)gj * n0 + gi : 0;

  double out[6];
#pragma unroll
  for (int f = 0; f < 6; f++) {
    if (MODE != SMAUG_INT_EULER)
      out[f] = 0.0;
    else if (MIX)
      out[f] = active ? base_value<MIX, CG>(B, f * nc + co) : 0.0;
    else
      out[f] = T.v(f, lo);
  }

  // ---- fluxes and divergence (centdiff1 / centdiff2), direction 0 then 1 --
  constexpr int FSZ = s2::fsz<O6>();
#pragma unroll
  for (int d = 0; d < 2; d++) {
    const bool o6d = O6 && d == 0;  // 6th order along dim 0 only (see s2::fsz)
    const int fh = o6d ? 3 : 2;     // flux halo along the direction
    const int ex = (d == 0) ? TX + 2 * fh : TX, ey = (d == 0) ? TY : TY + 2 * fh;
    const int ox = (d == 0) ? HALO - fh : HALO, oy = (d == 0) ? HALO : HALO - fh;
    double* F = static_cast<double*>(T.U);
    for (int r = tid; r < ex * ey; r += NTHREADS) {
      const int lx = ox + r % ex, ly = oy + r / ex;
      const int ci = T.x0 - HALO + lx, cj = T.y0 - HALO + ly;
      double f5[5] = {0, 0, 0, 0, 0};
      if (T.inner || (ci >= 0 && ci < n0 && cj >= 0 && cj < n1)) {
        if (d == 0)
          flux_at<BG, MIX, 0>(T, P.gamma, ly * RX + lx, f5);
        else
          flux_at<BG, MIX, 1>(T, P.gamma, ly * RX + lx, f5);
      }
#pragma unroll
      for (int k = 0; k < 5; k++) F[k * FSZ + r] = f5[k];
    }
    __syncthreads();
    if (active) {
      const int a = d == 0 ? gi : gj, n = d == 0 ? n0 : n1;
      const bool z = ((P.bt[d] != 0) && zero3dn(a, n)) || (o6d && edge6(a, n));
      const double rdl2 = 0.5 * (d == 0 ? T.rd0[lxo] : T.rd1[lyo]);
      const int fo = (lyo - oy) * ex + (lxo - ox);
      const int fs = d == 0 ? 1 : ex;
      const int fld[5] = {RHO, M1, M2, EN, d == 0 ? B2 : B1};
#pragma unroll
      for (int k = 0; k < 5; k++) {
        double g = o6d ? d6(F + k * FSZ, fo, fs, rdl2) : d4(F + k * FSZ, fo, fs, rdl2);
        if (z) g = 0;
        out[fld[k]] = out[fld[k]] - dt * g;
      }
      if (BG) {
        // addenergyterms_cd2 (src/centdiff2.cu:80-115)
        const double eb = T.v(EB, lo), bb1 = T.v(BB1, lo), bb2 = T.v(BB2, lo);
        const double ptb = (P.gamma - 1) * eb - 0.5 * (P.gamma - 2) * (bb1 * bb1 + bb2 * bb2);
        const double* v = T.V + d * RC;
        double gv = o6d ? d6(v, lo, 1, rdl2) : d4(v, lo, d == 0 ? 1 : RX, rdl2);
        if (z) gv = 0;
        out[EN] -= dt * ptb * gv;
        const double bbd = d == 0 ? bb1 : bb2;
        double g0 = dflux<O6>(v, lo, 1, 0.5 * T.rd0[lxo]);
        if (((P.bt[0] != 0) && zero3dn(gi, n0)) || (O6 && edge6(gi, n0))) g0 = 0;
        out[EN] += dt * bb1 * bbd * g0;
        double g1 = d4(v, lo, RX, 0.5 * T.rd1[lyo]);
        if ((P.bt[1] != 0) && zero3dn(gj, n1)) g1 = 0;
        out[EN] += dt * bb2 * bbd * g1;
      }
    }
    __syncthreads();
  }

  // ---- gravity (addgrav_cd2, src/centdiff2.cu:118-154) --------------------
  if (P.has_grav && active) {
    const double rho = T.v(RHO, lo);
    out[M1] += dt * P.g[0] * rho;
    out[M2] += dt * P.g[1] * rho;
    const double rr = rho * T.R[lo];
    out[EN] += (dt * P.g[0] * T.v(M1, lo)) * rr;
    out[EN] += (dt * P.g[1] * T.v(M2, lo)) * rr;
  }

  // ---- hyperdiffusion, in the driver's order -------------------------------
  if (P.hyperdif == 1) {
#define HP(K, C, D) hyper_pass<BG, MIX, K, C, D>(T, P, B, tid, active, lxo, lyo, gi, gj, dt, cin, out)
#define SQ(K, C) stage_q2<BG, MIX, K, C, CG>(T, P, B, tid)
    SQ(0, 0); HP(0, 0, 0); HP(0, 0, 1);
    SQ(1, 0); HP(1, 0, 0); HP(1, 0, 1);
    SQ(2, 0); HP(2, 0, 0); HP(2, 0, 1);
    SQ(2, 1); HP(2, 1, 0); HP(2, 1, 1);
    SQ(3, 1); HP(3, 1, 0);
    SQ(3, 0); HP(3, 0, 1);
#undef SQ
#undef HP
  }

  // ---- user driver (source_parallel + addsourceterms2) ---------------------
  if (P.driver == SMAUG_DRIVER_GAUSS && active) {
    double v = P.drv_amp;
    if (P.drv_period > 0) v *= sin(tstage * 2.0 * M_PI / P.drv_period);
    if (P.drv_sigma[0] > 0) {
      const double x = B.pos[0][gi] - P.drv_x0[0];
      v *= exp(-x * x / (P.drv_sigma[0] * P.drv_sigma[0]));
    }
    if (P.drv_sigma[1] > 0) {
      const double x = B.pos[1][gj] - P.drv_x0[1];
      v *= exp(-x * x / (P.drv_sigma[1] * P.drv_sigma[1]));
    }
    const double rhob = BG ? T.v(RHOB, lo) : B.bg[1 * nc + co];
    const double rr = (MODE == SMAUG_INT_EULER) ? out[RHO] : T.v(RHO, lo);
    out[M1] = out[M1] + dt * v * (rr + rhob);
  }

  // ---- combine, write, ghost images, CFL maxima -----------------------------
  double cm0 = P.cmax_floor[0], cm1 = P.cmax_floor[1];
  double res[6] = {0, 0, 0, 0, 0, 0};
  const bool is_base = (MODE == SMAUG_INT_EULER) || B.stage == 3;
  double gb[4] = {0, 0, 0, 0};  // background fields at the tile cell
  if (active) {
    if (MODE == SMAUG_INT_EULER) {
#pragma unroll
      for (int f = 0; f < 6; f++) res[f] = out[f];
    } else {
      const double wgt = (B.stage == 0 || B.stage == 3) ? 1.0 / 6.0 : 1.0 / 3.0;
      const double cst = (B.stage == 2) ? 1.0 : 0.5;
#pragma unroll
      for (int f = 0; f < 6; f++) {
        const double dl = out[f];
        if (B.stage == 0) {
          const double u = MIX ? base_value<MIX, CG>(B, f * nc + co) : T.v(f, lo);
          B.acc[f * nc + co] = u + wgt * dl;
          res[f] = u + cst * dl;
        } else if (B.stage < 3) {
          B.acc[f * nc + co] = ldsc<CG>(B.acc + f * nc + co) + wgt * dl;
          res[f] = base_value<MIX, CG>(B, f * nc + co) + cst * dl;
        } else {
          res[f] = ldsc<CG>(B.acc + f * nc + co) + wgt * dl;
        }
      }
    }
    bool bad = false;
#pragma unroll
    for (int f = 0; f < 6; f++) bad |= !isfinite(res[f]);
    if (bad) atomicOr(B.flags, 1);
    if (BG) {
      gb[0] = T.v(EB, lo);
      gb[1] = T.v(RHOB, lo);
      gb[2] = T.v(BB1, lo);
      gb[3] = T.v(BB2, lo);
    }
  }
  if constexpr (TMA != 0) {
    // the staged arrays are dead: copy the block's next tile (TMA = 2: its
    // rho_b) during the stores
    __syncthreads();
    if (tid == 0 && tt->nbx >= 0)
      tma_stage_issue<BG, MIX>(TMA == 2 ? nullptr : static_cast<void*>(T.S),
                               BG ? static_cast<void*>(T.G) : static_cast<void*>(T.R), *tt, tt->nbx, tt->nby);
  }
  if (active) {
    int ix[3], iy[3];
    ix[0] = gi;
    iy[0] = gj;
    const int nx = 1 + ghost_images(gi, n0, P.bc[0], ix + 1);
    const int ny = 1 + ghost_images(gj, n1, P.bc[1], iy + 1);
    bool negated = false;  // res holds the negated values
    for (int b = 0; b < ny; b++)
      for (int a2 = 0; a2 < nx; a2++) {
        const long cc = (long)iy[b] * n0 + ix[a2];
        // antisymmetric images carry the opposite sign (negation is exact)
        const bool neg = ((a2 > 0) && P.gneg[0]) != ((b > 0) && P.gneg[1]);
        if (neg != negated) {
#pragma unroll
          for (int f = 0; f < 6; f++) res[f] = -res[f];
          negated = neg;
        }
        const double* r = res;
#pragma unroll
        for (int f = 0; f < 6; f++) store_value<MIX>(B, f * nc + cc, r[f], is_base);
        double eb, rb, b1b, b2b;
        if (BG && a2 == 0 && b == 0) {
          eb = gb[0]; rb = gb[1]; b1b = gb[2]; b2b = gb[3];
        } else {
          eb = B.bg[0 * nc + cc]; rb = B.bg[1 * nc + cc]; b1b = B.bg[2 * nc + cc]; b2b = B.bg[3 * nc + cc];
        }
        double c0, c1;
        cfast2_both(P.gamma, r[RHO], r[M1], r[M2], r[EN], r[B1], r[B2], eb, rb, b1b, b2b, c0, c1);
        cm0 = dmax0(cm0, c0);
        cm1 = dmax0(cm1, c1);
      }
  }
  __shared__ double red[NTHREADS / 32][2];
  for (int o = 16; o > 0; o >>= 1) {
    cm0 = dmax0(cm0, __shfl_xor_sync(0xffffffffu, cm0, o));
    cm1 = dmax0(cm1, __shfl_xor_sync(0xffffffffu, cm1, o));
  }
  if ((tid & 31) == 0) {
    red[tid >> 5][0] = cm0;
    red[tid >> 5][1] = cm1;
  }
  __syncthreads();
  if (tid < 2) {
    double v = 0.0;
    for (int w = 0; w < NTHREADS / 32; w++) v = dmax0(v, red[w][tid]);
    atomicMax(&B.cmax_out[tid], (unsigned long long)__double_as_longlong(v));
  }
  return true;
}

template <int MODE, bool BG, bool MIX, bool O6>
__global__ void __launch_bounds__(NTHREADS, SMAUG_MINB2D) stage2d_fast(const KParams P, const KBufs B) {
  stage2d_body<MODE, BG, MIX, O6>(P, B, blockIdx.x, blockIdx.y);
}

// launch helper: picks the background and stencil-order specialisations
template <int MODE, bool MIX, bool O6>
static cudaError_t launch_stage2d_o(const KParams& K, const KBufs& B, cudaStream_t st) {
  dim3 block(TX, TY);
  dim3 grid((K.n0 - 4 + TX - 1) / TX, (K.n1 - 4 + TY - 1) / TY);
  if (K.has_bg) {
    stage2d_fast<MODE, true, MIX, O6><<<grid, block, s2::smem_bytes<true, MIX, O6>(), st>>>(K, B);
  } else {
    stage2d_fast<MODE, false, MIX, O6><<<grid, block, s2::smem_bytes<false, MIX, O6>(), st>>>(K, B);
  }
  return cudaGetLastError();
}
template <int MODE, bool MIX>
static cudaError_t launch_stage2d(const KParams& K, const KBufs& B, cudaStream_t st) {
  return K.order6 ? launch_stage2d_o<MODE, MIX, true>(K, B, st) : launch_stage2d_o<MODE, MIX, false>(K, B, st);
}

template <int MODE, bool BG, bool MIX, bool O6>
static cudaError_t stage2d_attr() {
  return cudaFuncSetAttribute(stage2d_fast<MODE, BG, MIX, O6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)s2::smem_bytes<BG, MIX, O6>());
}
