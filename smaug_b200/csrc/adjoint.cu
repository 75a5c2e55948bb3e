// adjoint.cu -- hand-written adjoint (vector-Jacobian product) of the 2D
// stage operator, FP64.
//
// The stage operator F maps a ghost-filled stage input X to the increment
// k = F(X) of the interior cells (the quantity the forward stage kernel adds
// with its RK weights); F depends on X, on the per-dimension CFL maxima cmax
// of X (through the hyperdiffusion coefficient) and on the driver parameters
// (amplitude, period, centre along dim 1).  With dt held fixed, the adjoint of
// one classical RK4 step needs, for a given k-bar,
//   X-bar += (dF/dX)^T k-bar,   cmax-bar += (dF/dcmax)^T k-bar,
//   theta-bar += (dF/dtheta)^T k-bar.
// adj_stage2d computes them term by term, in the reverse of the forward
// kernel's arithmetic (stage2d.cuh):
//   flux divergence       -dt d4(F_f)         (src/centdiff1.cu, centdiff2.cu)
//   background coupling   e terms of addenergyterms_cd2 (src/centdiff2.cu:80-115)
//   gravity               (src/centdiff2.cu:118-154)
//   hyperdiffusion        nu = c R with R = max D3 / max D1 differentiated
//                         through the stored argmax faces (a max with ties
//                         keeps the first maximum, as the forward does)
//   driver                m_1 += dt v(theta, t, x) (rho + rho_b)
// One thread per output cell of a 32x8 tile recomputes what its outputs need
// from the tile's staged state and scatters the products into a shared
// accumulator over the tile + 3-cell region (shared-memory atomics), flushed
// to global memory with one atomic add per region cell and field.  Pads of the
// hyperdiffusion windows route their adjoints to their source cells (index 5,
// or the stray-store source).  cmax-bar is returned as two scalars; the caller
// sends it to the cell that attains the maximum (adj_cmax2d).
#include <vector>

#include "engine_internal.h"
#include "kernels.cuh"

#define CUDA_TRY(call)                                                                  \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess)                                                              \
      return smaug::set_error(SMAUG_E_CUDA, "%s failed: %s (%s:%d)", #call,             \
                              cudaGetErrorString(_e), __FILE__, __LINE__);              \
  } while (0)

namespace smaug {

namespace {

constexpr int ANT = TX * TY;  // threads per adjoint block (tile 32x8 as the forward)
#ifndef SMAUG_ADJ_MINB
#define SMAUG_ADJ_MINB 2  // resident blocks per SM the adjoint stage is compiled for
#endif

struct A2 {
  double* S;   // [6][RC] state
  double* G;   // [4][RC] background fields
  double* R;   // [RC] 1/rho_t
  double* A;   // [6][RC] adjoint accumulator
  double* dl0;
  double* dl1;
  double* rd0;
  double* rd1;
  int x0, y0;
  __device__ __forceinline__ double v(int f, int l) const { return f < 6 ? S[f * RC + l] : G[(f - 6) * RC + l]; }
};

struct AdjIn {
  const double* X;       // [6][ncell] stage input, ghosts filled
  const double* bg;      // [4][ncell]
  const double* lam;     // [6][ncell] k-bar (interior cells)
  double* Xb;            // [6][ncell] X-bar (accumulated)
  double* sbar;          // [2] cmax-bar (accumulated)
  double* thbar;         // [3] d/d(amp, period, x0 along dim 1) (accumulated)
  const double* cmax;    // [2] the stage's CFL maxima
  const double* delx[2];
  const double* pos[2];
  const int* padsrc[2];
  double dt, tstage;
};

__device__ __forceinline__ void sadd(double* a, double v) {
  if (v != 0.0) atomicAdd(a, v);
}

// ---- q of the hyperdiffusion fields and its adjoint -------------------------
// (src/hyperdifvisc1r.cu:1225-1253): rho; e - (B^2 + m^2/rho_t)/2; m_c/rho_t; B_c
template <int KIND, int COMP>
__device__ __forceinline__ double q_loc(const A2& T, int l) {
  if (KIND == 0) return T.v(RHO, l);
  if (KIND == 1) {
    const double m1 = T.v(M1, l), m2 = T.v(M2, l), b1 = T.v(B1, l), b2 = T.v(B2, l);
    return T.v(EN, l) - 0.5 * ((b1 * b1 + b2 * b2) + (m1 * m1 + m2 * m2) * T.R[l]);
  }
  if (KIND == 2) return T.v(M1 + COMP, l) * T.R[l];
  return T.v(B1 + COMP, l);
}

template <int KIND, int COMP>
__device__ __forceinline__ void qbar_loc(const A2& T, int l, double qb) {
  if (qb == 0.0) return;
  double* A = T.A;
  if (KIND == 0) {
    sadd(A + RHO * RC + l, qb);
  } else if (KIND == 1) {
    const double m1 = T.v(M1, l), m2 = T.v(M2, l), b1 = T.v(B1, l), b2 = T.v(B2, l), r = T.R[l];
    sadd(A + EN * RC + l, qb);
    sadd(A + B1 * RC + l, -qb * b1);
    sadd(A + B2 * RC + l, -qb * b2);
    sadd(A + M1 * RC + l, -qb * m1 * r);
    sadd(A + M2 * RC + l, -qb * m2 * r);
    sadd(A + RHO * RC + l, qb * 0.5 * (m1 * m1 + m2 * m2) * r * r);
  } else if (KIND == 2) {
    const double r = T.R[l], m = T.v(M1 + COMP, l);
    sadd(A + (M1 + COMP) * RC + l, qb * r);
    sadd(A + RHO * RC + l, -qb * m * r * r);
  } else {
    sadd(A + (B1 + COMP) * RC + l, qb);
  }
}

template <int KIND, int COMP>
__device__ __forceinline__ double q_glob(const AdjIn& I, long nc, long c) {
  const double rho = I.X[c], r = 1.0 / (rho + I.bg[1 * nc + c]);
  if (KIND == 0) return rho;
  if (KIND == 1) {
    const double m1 = I.X[1 * nc + c], m2 = I.X[2 * nc + c], b1 = I.X[4 * nc + c], b2 = I.X[5 * nc + c];
    return I.X[3 * nc + c] - 0.5 * ((b1 * b1 + b2 * b2) + (m1 * m1 + m2 * m2) * r);
  }
  if (KIND == 2) return I.X[(1 + COMP) * nc + c] * r;
  return I.X[(4 + COMP) * nc + c];
}

template <int KIND, int COMP>
__device__ __forceinline__ void qbar_glob(const AdjIn& I, long nc, long c, double qb) {
  if (qb == 0.0) return;
  double* Xb = I.Xb;
  const double rho = I.X[c], r = 1.0 / (rho + I.bg[1 * nc + c]);
  if (KIND == 0) {
    atomicAdd(Xb + c, qb);
  } else if (KIND == 1) {
    const double m1 = I.X[1 * nc + c], m2 = I.X[2 * nc + c], b1 = I.X[4 * nc + c], b2 = I.X[5 * nc + c];
    atomicAdd(Xb + 3 * nc + c, qb);
    atomicAdd(Xb + 4 * nc + c, -qb * b1);
    atomicAdd(Xb + 5 * nc + c, -qb * b2);
    atomicAdd(Xb + 1 * nc + c, -qb * m1 * r);
    atomicAdd(Xb + 2 * nc + c, -qb * m2 * r);
    atomicAdd(Xb + c, qb * 0.5 * (m1 * m1 + m2 * m2) * r * r);
  } else if (KIND == 2) {
    atomicAdd(Xb + (1 + COMP) * nc + c, qb * r);
    atomicAdd(Xb + c, -qb * I.X[(1 + COMP) * nc + c] * r * r);
  } else {
    atomicAdd(Xb + (4 + COMP) * nc + c, qb);
  }
}

// ---- the nu ratio and its adjoint ------------------------------------------
// R = max(0, D3(f), f = o-1..o+1) / max(0, D1(f), f = o-2..o+2) from
// qv[k] = q(o - 2 + k), k = 0..5; the argmax faces and the signs of the
// differences there are kept for the adjoint.
struct RInfo {
  double R, T4, T5, s3, s1;
  int f3, f1;
};

__device__ __forceinline__ RInfo ratio_of(const double* qv) {
  RInfo r{0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double w = 3.0 * (qv[k + 2] - qv[k + 1]) - (qv[k + 3] - qv[k]);
    const double d = fabs(w);
    if (d > r.T4) {
      r.T4 = d;
      r.f3 = k;
      r.s3 = w > 0 ? 1.0 : -1.0;
    }
  }
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const double w = qv[k + 1] - qv[k];
    const double d = fabs(w);
    if (d > r.T5) {
      r.T5 = d;
      r.f1 = k;
      r.s1 = w > 0 ? 1.0 : -1.0;
    }
  }
  r.R = (r.T5 > 0) ? r.T4 / r.T5 : 0.0;
  return r;
}

// adds (dR/dqv)^T Rb into qvb[0..5]
__device__ __forceinline__ void ratio_bwd(const RInfo& r, double Rb, double* qvb) {
  if (!(r.T5 > 0) || Rb == 0.0) return;
  const double T4b = Rb / r.T5, T5b = -Rb * r.R / r.T5;
  if (r.T4 > 0) {
    const double wb = r.s3 * T4b;
    const int k = r.f3;
    qvb[k + 2] += 3.0 * wb;
    qvb[k + 1] -= 3.0 * wb;
    qvb[k + 3] -= wb;
    qvb[k] += wb;
  }
  const double wb = r.s1 * T5b;
  qvb[r.f1 + 1] += wb;
  qvb[r.f1] -= wb;
}

// ---- flux Jacobian, transposed ----------------------------------------------
// x = (rho, m1, m2, e, b1, b2) at one cell, g = (eb, rhob, bb1, bb2);
// F = (F_rho, F_m1, F_m2, F_e, F_B across D) as in flux_at (stage2d.cuh);
// adds J^T Fb into xb.
template <int D>
__device__ __forceinline__ void flux_vjp(const double* x, const double* g, double gamma, const double* Fb,
                                         double* xb) {
  const double rt = x[0] + g[1], r = 1.0 / rt;
  const double m[2] = {x[1], x[2]}, b[2] = {x[4], x[5]}, bb[2] = {g[2], g[3]};
  const double e = x[3], eb = g[0];
  constexpr int c = 1 - D;
  const double md = m[D], vd = md * r, bd = b[D], bbd = bb[D];
  const double M2 = m[0] * m[0] + m[1] * m[1];
  const double pt = (gamma - 1.0) * (e - 0.5 * M2 * r) -
                    (gamma - 2.0) * ((b[0] * bb[0] + b[1] * bb[1]) + 0.5 * (b[0] * b[0] + b[1] * b[1]));
  const double bbm = bb[0] * m[0] + bb[1] * m[1], bm = b[0] * m[0] + b[1] * m[1];
  double mb[2] = {0, 0}, bbar[2] = {0, 0}, eb_ = 0, vdb = 0, ptb = 0, rb = 0;
  // F_rho = m_D
  mb[D] += Fb[0];
  // F_m1, F_m2
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const double F = Fb[1 + k];
    vdb += F * m[k];
    mb[k] += F * vd;
    if (k == D) ptb += F;
    bbar[k] -= F * (bbd + bd);
    bbar[D] -= F * (bb[k] + b[k]);
  }
  // F_e = vd (e + pt + eb) - W r, W = bd bbm + bbd bm + bd bm
  {
    const double F = Fb[3];
    vdb += F * (e + pt + eb);
    eb_ += F * vd;
    ptb += F * vd;
    const double W = bd * bbm + bbd * bm + bd * bm;
    const double Wb = -F * r;
    rb -= F * W;
    bbar[D] += Wb * (bbm + bm);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      mb[k] += Wb * bd * bb[k];
      bbar[k] += Wb * (bbd + bd) * m[k];
      mb[k] += Wb * (bbd + bd) * b[k];
    }
  }
  // F_B = vd (b_c + bb_c) - (m_c r)(b_D + bb_D)
  {
    const double F = Fb[4];
    vdb += F * (b[c] + bb[c]);
    bbar[c] += F * vd;
    mb[c] -= F * r * (bd + bbd);
    rb -= F * m[c] * (bd + bbd);
    bbar[D] -= F * m[c] * r;
  }
  // vd = m_D r
  mb[D] += vdb * r;
  rb += vdb * md;
  // pt
  eb_ += ptb * (gamma - 1.0);
#pragma unroll
  for (int k = 0; k < 2; k++) {
    mb[k] -= ptb * (gamma - 1.0) * m[k] * r;
    bbar[k] -= ptb * (gamma - 2.0) * (bb[k] + b[k]);
  }
  rb -= ptb * (gamma - 1.0) * 0.5 * M2;
  xb[0] -= rb * r * r;
  xb[1] += mb[0];
  xb[2] += mb[1];
  xb[3] += eb_;
  xb[4] += bbar[0];
  xb[5] += bbar[1];
}

// ---- fast speed, transposed (computec3, src/dervfields.cu:241-309) ----------
// adds s * d cfast_dir / dx into xb for x = (rho, m1, m2, e, b1, b2)
__device__ __forceinline__ void cfast_vjp(double gamma, const double* x, const double* g, int dir, double s,
                                          double* xb) {
  const double rho = x[0], m1 = x[1], m2 = x[2], e = x[3], b1 = x[4], b2 = x[5];
  const double eb = g[0], rhob = g[1], bb1 = g[2], bb2 = g[3];
  const double m2s = m1 * m1 + m2 * m2, b2s = b1 * b1 + b2 * b2, bbb = bb1 * b1 + bb2 * b2;
  const double bb2s = bb1 * bb1 + bb2 * bb2, rt = rho + rhob;
  const double pk = (gamma - 1) * (e - 0.5 * (m2s / rt) - 0.5 * b2s - bbb);
  const double K = (gamma - 1) * (eb - 0.5 * bb2s);
  const double cs2 = (gamma * (pk + K)) / rt;
  const double cf = (b2s + bb2s + 2.0 * bbb) / rt + cs2;
  const double bd = (dir == 0) ? (bb1 + b1) : (bb2 + b2);
  const double md = (dir == 0) ? m1 : m2;
  const double disc = cf * cf - 4.0 * cs2 * (bd * bd) / rt;
  const double sq = disc > 0 ? sqrt(disc) : 0.0;
  const double cfasti = 0.5 * (cf + sq);
  double cfb = 0, cs2b = 0, bdb = 0, rtb = 0, mdb = 0;
  if (cfasti > 0) {
    const double cib = s / (2.0 * sqrt(cfasti));
    cfb += 0.5 * cib;
    if (sq > 0) {
      const double db = 0.5 * cib / (2.0 * sq);
      cfb += db * 2.0 * cf;
      cs2b -= db * 4.0 * (bd * bd) / rt;
      bdb -= db * 8.0 * cs2 * bd / rt;
      rtb += db * 4.0 * cs2 * (bd * bd) / (rt * rt);
    }
  }
  const double w = md / rt;
  const double wb = s * (w > 0 ? 1.0 : (w < 0 ? -1.0 : 0.0));
  mdb += wb / rt;
  rtb -= wb * md / (rt * rt);
  // cf = (b2s + bb2s + 2 bbb)/rt + cs2
  cs2b += cfb;
  double b2sb = cfb / rt, bbbb = 2.0 * cfb / rt;
  rtb -= cfb * (b2s + bb2s + 2.0 * bbb) / (rt * rt);
  // cs2 = gamma (pk + K) / rt
  const double pkb = cs2b * gamma / rt;
  rtb -= cs2b * cs2 / rt;
  // pk
  double eb_ = pkb * (gamma - 1);
  double m2sb = -pkb * (gamma - 1) * 0.5 / rt;
  rtb += pkb * (gamma - 1) * 0.5 * m2s / (rt * rt);
  b2sb -= pkb * (gamma - 1) * 0.5;
  bbbb -= pkb * (gamma - 1);
  xb[0] += rtb;
  xb[1] += 2.0 * m2sb * m1 + (dir == 0 ? mdb : 0.0);
  xb[2] += 2.0 * m2sb * m2 + (dir == 1 ? mdb : 0.0);
  xb[3] += eb_;
  xb[4] += 2.0 * b2sb * b1 + bbbb * bb1 + (dir == 0 ? bdb : 0.0);
  xb[5] += 2.0 * b2sb * b2 + bbbb * bb2 + (dir == 1 ? bdb : 0.0);
}

// ---- one hyperdiffusion pass, transposed ------------------------------------
// Block-cooperative, in the phases of the forward pass (hyper_pass in
// stage2d.cuh): (A) q of the pass on the staged region, (B) the nu ratio R with
// its argmax faces on the ratio area, then the adjoint: (C) the cross-term
// arrays at each nu-area cell j, gathered from the two tile cells whose
// outputs difference them, and (D) the diagonal terms at each tile cell,
// both accumulating R-bar (RB) and q-bar (QB); (E) R-bar through the argmax
// faces into q-bar; (F) q-bar into the field adjoints, pads routed to their
// sources.  All threads of the block call it.
constexpr int ARSZ = (TX + 1) * (TY + 2) > (TX + 2) * (TY + 1) ? (TX + 1) * (TY + 2) : (TX + 2) * (TY + 1);

struct PassScratch {
  double* Q;    // [RC] q of the pass (pads included)
  double* QB;   // [RC] q-bar
  double* RR;   // [ARSZ] ratio R
  double* T5;   // [ARSZ] its denominator max D1
  double* RB;   // [ARSZ] R-bar
  int* code;    // [ARSZ] argmax faces and signs
};

__device__ __forceinline__ int pack_code(const RInfo& r) {
  return r.f3 | (r.f1 << 2) | ((r.s3 > 0) << 5) | ((r.s1 > 0) << 6);
}
__device__ __forceinline__ RInfo unpack(double R, double T5, int c) {
  RInfo r;
  r.R = R;
  r.T5 = T5;
  r.T4 = R * T5;  // only its sign is used (R > 0 iff T4 > 0 where T5 > 0)
  r.f3 = c & 3;
  r.f1 = (c >> 2) & 7;
  r.s3 = (c & 32) ? 1.0 : -1.0;
  r.s1 = (c & 64) ? 1.0 : -1.0;
  return r;
}

// (A) q of the pass field on the region with the reference's pads; q-bar
// cleared.  The passes of both directions of one field share q and q-bar; the
// caller places the barrier (the next field's staging runs beside the
// previous field's flush, on the other q-bar buffer).
template <int KIND, int COMP>
__device__ __forceinline__ void adj_stage_q(const A2& T, const AdjIn& I, const KParams& P,
                                            const PassScratch& W, int tid) {
  const long nc = P.ncell;
  const int n0 = P.n0, n1 = P.n1;
  // (A) q on the region with the reference's pads; q-bar cleared
  for (int r = tid; r < RC; r += ANT) {
    const int lx = r % RX, ly = r / RX;
    const int ci = T.x0 - HALO + lx, cj = T.y0 - HALO + ly;
    const bool inx = ci >= 0 && ci < n0, iny = cj >= 0 && cj < n1;
    double q = 0.0;
    if (inx && iny) {
      q = q_loc<KIND, COMP>(T, r);
    } else if (iny) {
      if (ci == -1) {
        q = q_loc<KIND, COMP>(T, r + 6);
      } else if (ci == n0) {
        const int src = I.padsrc[0][cj];
        if (src >= 0) q = q_glob<KIND, COMP>(I, nc, src);
      }
    } else if (inx) {
      if (cj == -1) {
        q = q_loc<KIND, COMP>(T, r + 6 * RX);
      } else if (cj == n1) {
        const int src = I.padsrc[1][ci];
        if (src >= 0) q = q_glob<KIND, COMP>(I, nc, src);
      }
    }
    W.Q[r] = q;
    W.QB[r] = 0.0;
  }
}

// (B)-(E) of one pass on the staged q: R-bar and q-bar accumulated
template <int KIND, int COMP, int DIM>
__device__ __forceinline__ void hyp_pass_adj(const A2& T, const AdjIn& I, const KParams& P,
                                             const PassScratch& W, int tid, bool active, int lxo,
                                             int lyo, int gi, int gj, const double* Lam, double* sb) {
  constexpr bool CROSS = (KIND == 2 && COMP != DIM) || (KIND == 3);
  constexpr int QF = (KIND == 0) ? RHO : (KIND == 1) ? EN : (KIND == 2) ? M1 + COMP : B1 + COMP;
  constexpr int SQ = DIM == 0 ? 1 : RX;  // stride along DIM in the region
  constexpr int SL = SQ;
  // ratio area: the tile along DIM extended by one cell below, +-1 across
  // when cross terms need it (as the forward)
  constexpr int exR = DIM == 0 ? TX + 1 : (CROSS ? TX + 2 : TX);
  constexpr int eyR = DIM == 0 ? (CROSS ? TY + 2 : TY) : TY + 1;
  constexpr int oxR = DIM == 0 ? HALO - 1 : (CROSS ? HALO - 1 : HALO);
  constexpr int oyR = DIM == 0 ? (CROSS ? HALO - 1 : HALO) : HALO - 1;
  constexpr int SR = DIM == 0 ? 1 : exR;  // stride along DIM in the ratio area
  // nu area: the tile along DIM, +-1 across
  constexpr int exN = DIM == 0 ? TX : TX + 2, eyN = DIM == 0 ? TY + 2 : TY;
  constexpr int oxN = DIM == 0 ? HALO : HALO - 1, oyN = DIM == 0 ? HALO - 1 : HALO;
  const int n0 = P.n0, n1 = P.n1, nd = DIM == 0 ? n0 : n1;
  const double dt = I.dt;
  const double chyp = P.chyp[QF], coef = I.cmax[DIM] * chyp;
  auto ri = [&](int lx, int ly) { return (ly - oyR) * exR + (lx - oxR); };

  // (B) R = max D3(i-1..i+1) / max D1(i-2..i+2) and its argmax faces
  for (int r = tid; r < exR * eyR; r += ANT) {
    const int lx = oxR + r % exR, ly = oyR + r / exR;
    const int l = ly * RX + lx;
    double qv[6];
#pragma unroll
    for (int k = 0; k < 6; k++) qv[k] = W.Q[l + (k - 2) * SQ];
    const RInfo Ri = ratio_of(qv);
    W.RR[r] = Ri.R;
    W.T5[r] = Ri.T5;
    W.code[r] = pack_code(Ri);
    W.RB[r] = 0.0;
  }
  __syncthreads();
  // (C) cross terms: d/dx_COMP of C3 = rho_t tau, C4 = tau m_DIM (momentum) or
  // C3 = t3, C4 = t3 B_DIM (field; the outputs take them with a minus sign),
  // tau = g nsum / 4, t3 = g nsum / 2, at the nu-area cells j
  if (CROSS) {
    for (int r = tid; r < exN * eyN; r += ANT) {
      const int lx = oxN + r % exN, ly = oyN + r / exN;
      const int jx = T.x0 - HALO + lx, jy = T.y0 - HALO + ly;
      if (!(jx >= 2 && jx <= n0 - 3 && jy >= 2 && jy <= n1 - 3)) continue;  // nsum = 0 there
      // C3-bar, C4-bar from the tile cells i = j -+ e_COMP
      double C3b = 0.0, C4b = 0.0;
#pragma unroll
      for (int s = -1; s <= 1; s += 2) {
        const int ix = lx - HALO - (COMP == 0 ? s : 0), iy = ly - HALO - (COMP == 1 ? s : 0);
        if (ix < 0 || ix >= TX || iy < 0 || iy >= TY) continue;
        const int ci = T.x0 + ix, cj = T.y0 + iy;
        if (!(ci <= n0 - 3 && cj <= n1 - 3)) continue;  // not an output cell
        const int af = COMP == 0 ? ci : cj;
        if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) continue;
        const int it = iy * TX + ix;
        const double rdf = COMP == 0 ? T.rd0[ix + HALO] : T.rd1[iy + HALO];
        const double sgn = (KIND == 2) ? 1.0 : -1.0;
        const double lx_ = (KIND == 2) ? Lam[(M1 + DIM) * ANT + it] : Lam[(B1 + DIM) * ANT + it];
        C3b += sgn * s * lx_ * dt * rdf * 0.5;
        C4b += sgn * s * Lam[EN * ANT + it] * dt * rdf * 0.5;
      }
      if (C3b == 0.0 && C4b == 0.0) continue;
      const int l = ly * RX + lx;
      const int a = DIM == 0 ? jx : jy;
      const double dl = DIM == 0 ? T.dl0[lx] : T.dl1[ly];
      const double rdl = DIM == 0 ? T.rd0[lx] : T.rd1[ly];
      const double c = dl * coef;
      const int rr = ri(lx, ly);
      const double Rj = W.RR[rr], Rjm = W.RR[rr - SR];
      const double nsum = c * Rj + c * Rjm;
      const bool zj = (P.bt[DIM] != 0) && zero1n(a, nd);
      const double g = zj ? 0.0 : ((W.Q[l + SQ] - W.Q[l - SQ]) * rdl) * 0.5;
      double tb;
      if (KIND == 2) {
        const double tau = (g * nsum) * 0.25;
        tb = C3b * (T.v(RHO, l) + T.v(RHOB, l)) + C4b * T.v(M1 + DIM, l);
        sadd(T.A + RHO * RC + l, C3b * tau);
        sadd(T.A + (M1 + DIM) * RC + l, C4b * tau);
        tb *= 0.25;
      } else {
        const double t3 = (g * nsum) * 0.5;
        tb = C3b + C4b * T.v(B1 + DIM, l);
        sadd(T.A + (B1 + DIM) * RC + l, C4b * t3);
        tb *= 0.5;
      }
      const double gb = tb * nsum, nsb = tb * g;
      if (!zj) {
        sadd(W.QB + l + SQ, gb * rdl * 0.5);
        sadd(W.QB + l - SQ, -gb * rdl * 0.5);
      }
      sb[DIM] += nsb * dl * chyp * (Rj + Rjm);
      sadd(W.RB + rr, nsb * c);
      sadd(W.RB + rr - SR, nsb * c);
    }
  }
  // (D) the diagonal terms at the tile cells
  if (active) {
    const int l = lyo * RX + lxo;
    const int a = DIM == 0 ? gi : gj;
    const double dl = DIM == 0 ? T.dl0[lxo] : T.dl1[lyo];
    const double rdl = DIM == 0 ? T.rd0[lxo] : T.rd1[lyo];
    const double c = dl * coef;
    const int rr = ri(lxo, lyo);
    const double Ri = W.RR[rr], Rm = W.RR[rr - SR];
    const double nur = c * Ri, nul = c * Rm;
    const double qc = W.Q[l], qp = W.Q[l + SQ], qm = W.Q[l - SQ];
    const bool z = (P.bt[DIM] != 0) && zero1n(a, nd);
    const double gr = z ? 0.0 : (qp - qc) * rdl, gl = z ? 0.0 : (qc - qm) * rdl;
    const int tid_ = tid;
    auto lam = [&](int f) { return Lam[f * ANT + tid_]; };
    double nurb = 0, nulb = 0, grb = 0, glb = 0;
    double qb0 = 0, qbm = 0, qbp = 0;  // q-bar at i, i-1, i+1
    if (KIND == 0 || KIND == 1) {
      const double ab = lam(QF) * dt * rdl;
      nurb += ab * gr;
      nulb -= ab * gl;
      grb += ab * nur;
      glb -= ab * nul;
    } else if (KIND == 2) {
      const double mult = (COMP == DIM) ? 2.0 : 1.0;
      const double r0 = T.v(RHO, l) + T.v(RHOB, l);
      const double t2 = (r0 + T.v(RHO, l - SL) + T.v(RHOB, l - SL)) * 0.5;
      const double t3 = (r0 + T.v(RHO, l + SL) + T.v(RHOB, l + SL)) * 0.5;
      const double mf = T.v(M1 + COMP, l);
      const double t5 = (mf + T.v(M1 + COMP, l - SL)) * 0.5;
      const double t6 = (mf + T.v(M1 + COMP, l + SL)) * 0.5;
      const double am = lam(M1 + COMP) * dt * mult * rdl * 0.5;
      const double ae = lam(EN) * dt * mult * rdl * 0.5;
      const double t3b = am * nur * gr, t2b = -am * nul * gl;
      const double t6b = ae * nur * gr, t5b = -ae * nul * gl;
      nurb += am * t3 * gr + ae * t6 * gr;
      grb += am * t3 * nur + ae * t6 * nur;
      nulb -= am * t2 * gl + ae * t5 * gl;
      glb -= am * t2 * nul + ae * t5 * nul;
      sadd(T.A + RHO * RC + l, 0.5 * (t2b + t3b));
      sadd(T.A + RHO * RC + l - SL, 0.5 * t2b);
      sadd(T.A + RHO * RC + l + SL, 0.5 * t3b);
      sadd(T.A + (M1 + COMP) * RC + l, 0.5 * (t5b + t6b));
      sadd(T.A + (M1 + COMP) * RC + l - SL, 0.5 * t5b);
      sadd(T.A + (M1 + COMP) * RC + l + SL, 0.5 * t6b);
    } else {
      // diagonal B term (hyperdifbsource, sb = +1), q = B_COMP
      const double aB = lam(B1 + COMP) * dt * rdl;
      const double ae = lam(EN) * dt * rdl;
      const double t2 = (qc + qm) * 0.5, t3 = (qc + qp) * 0.5;
      grb += aB * nur + ae * t3 * nur;
      nurb += aB * gr + ae * t3 * gr;
      glb -= aB * nul + ae * t2 * nul;
      nulb -= aB * gl + ae * t2 * gl;
      const double t3b = ae * gr * nur, t2b = -ae * gl * nul;
      qb0 += 0.5 * (t2b + t3b);
      qbm += 0.5 * t2b;
      qbp += 0.5 * t3b;
    }
    if (!z) {
      qbp += grb * rdl;
      qb0 -= grb * rdl;
      qb0 += glb * rdl;
      qbm -= glb * rdl;
    }
    sadd(W.QB + l, qb0);
    sadd(W.QB + l - SQ, qbm);
    sadd(W.QB + l + SQ, qbp);
    sb[DIM] += nurb * dl * chyp * Ri + nulb * dl * chyp * Rm;
    sadd(W.RB + rr, nurb * c);
    sadd(W.RB + rr - SR, nulb * c);
  }
  __syncthreads();
  // (E) R-bar through the argmax faces into q-bar
  for (int r = tid; r < exR * eyR; r += ANT) {
    const double Rb = W.RB[r];
    if (Rb == 0.0) continue;
    const int lx = oxR + r % exR, ly = oyR + r / exR;
    const int l = ly * RX + lx;
    const RInfo Ri = unpack(W.RR[r], W.T5[r], W.code[r]);
    double qvb[6] = {0, 0, 0, 0, 0, 0};
    ratio_bwd(Ri, Rb, qvb);
#pragma unroll
    for (int k = 0; k < 6; k++) sadd(W.QB + l + (k - 2) * SQ, qvb[k]);
  }
  __syncthreads();
}

// (F) q-bar of the field into the field adjoints; pads routed to the cells
// they copy (the caller places the barrier)
template <int KIND, int COMP>
__device__ __forceinline__ void adj_flush_q(const A2& T, const AdjIn& I, const KParams& P,
                                            const PassScratch& W, int tid) {
  const long nc = P.ncell;
  const int n0 = P.n0, n1 = P.n1;
  for (int r = tid; r < RC; r += ANT) {
    const double qb = W.QB[r];
    if (qb == 0.0) continue;
    const int lx = r % RX, ly = r / RX;
    const int ci = T.x0 - HALO + lx, cj = T.y0 - HALO + ly;
    const bool inx = ci >= 0 && ci < n0, iny = cj >= 0 && cj < n1;
    if (inx && iny) {
      qbar_loc<KIND, COMP>(T, r, qb);
    } else if (iny) {
      if (ci == -1) {
        qbar_loc<KIND, COMP>(T, r + 6, qb);
      } else if (ci == n0) {
        const int src = I.padsrc[0][cj];
        if (src >= 0) qbar_glob<KIND, COMP>(I, nc, src, qb);
      }
    } else if (inx) {
      if (cj == -1) {
        qbar_loc<KIND, COMP>(T, r + 6 * RX, qb);
      } else if (cj == n1) {
        const int src = I.padsrc[1][ci];
        if (src >= 0) qbar_glob<KIND, COMP>(I, nc, src, qb);
      }
    }
  }
}

// d4 weights: d4(a)(i) = sum_k W4(k) a(i+k) * rdl2, k = -2..2 (k = 0 unused)
__device__ __forceinline__ double w4(int k) {
  return k == 1 ? 8.0 / 6.0 : (k == -1 ? -8.0 / 6.0 : (k == -2 ? 1.0 / 6.0 : (k == 2 ? -1.0 / 6.0 : 0.0)));
}

__global__ void __launch_bounds__(ANT, SMAUG_ADJ_MINB) adj_stage2d(const KParams P, const AdjIn I) {
  extern __shared__ double smem[];
  A2 T;
  T.S = smem;
  T.G = T.S + 6 * RC;
  T.R = T.G + 4 * RC;
  T.A = T.R + RC;
  double* Lam = T.A + 6 * RC;  // [6][ANT] k-bar of the tile's cells
  T.dl0 = Lam + 6 * ANT;
  T.dl1 = T.dl0 + RX;
  T.rd0 = T.dl1 + RY;
  T.rd1 = T.rd0 + RX;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  T.x0 = 2 + blockIdx.x * TX;
  T.y0 = 2 + blockIdx.y * TY;
  const int n0 = P.n0, n1 = P.n1;
  const long nc = P.ncell;
  const double dt = I.dt;
  const int gi = T.x0 + tx, gj = T.y0 + ty;
  const bool active = gi <= n0 - 3 && gj <= n1 - 3;
  const long co = (long)gj * n0 + gi;
  double lam[6];
  bool nonzero = false;
#pragma unroll
  for (int f = 0; f < 6; f++) {
    lam[f] = active ? I.lam[f * nc + co] : 0.0;
    nonzero |= lam[f] != 0.0;
  }
  // every term below is linear in the tile's k-bar: a tile without any adds
  // nothing (sparse adjoints: a loss on part of the domain)
  if (!__syncthreads_or(nonzero)) return;
#pragma unroll
  for (int f = 0; f < 6; f++) Lam[f * ANT + tid] = lam[f];

  // ---- stage X, backgrounds, 1/rho_t, zero the accumulator ---------------
  for (int r = tid; r < RC; r += ANT) {
    const int lx = r % RX, ly = r / RX;
    const int gi = T.x0 - HALO + lx, gj = T.y0 - HALO + ly;
    const bool in = gi >= 0 && gi < n0 && gj >= 0 && gj < n1;
    const long c = (long)gj * n0 + gi;
#pragma unroll
    for (int f = 0; f < 6; f++) {
      T.S[f * RC + r] = in ? I.X[f * nc + c] : 0.0;
      T.A[f * RC + r] = 0.0;
    }
#pragma unroll
    for (int f = 0; f < 4; f++) T.G[f * RC + r] = in ? I.bg[f * nc + c] : (f == 1 ? 1.0 : 0.0);
    T.R[r] = 1.0 / (T.S[RHO * RC + r] + T.G[1 * RC + r]);
  }
  for (int r = tid; r < RX + RY; r += ANT) {
    if (r < RX) {
      const int gi = T.x0 - HALO + r;
      const double d = (gi >= 0 && gi < n0) ? I.delx[0][gi] : 1.0;
      T.dl0[r] = d;
      T.rd0[r] = 1.0 / d;
    } else {
      const int gj = T.y0 - HALO + (r - RX);
      const double d = (gj >= 0 && gj < n1) ? I.delx[1][gj] : 1.0;
      T.dl1[r - RX] = d;
      T.rd1[r - RX] = 1.0 / d;
    }
  }
  __syncthreads();

  // ---- fluxes, background energy coupling, gravity (gather per cell) -----
  // the adjoint of -dt d4(F_f) at the tile cells collected at each flux cell
  // j; then the pointwise flux Jacobian, transposed, at j
  const bool bgon = P.has_bg != 0;
  for (int r = tid; r < RC; r += ANT) {
    const int lx = r % RX, ly = r / RX;
    const int tj = lx - HALO, tk = ly - HALO;  // tile coordinates of j
    const int cj0 = T.x0 - HALO + lx, cj1 = T.y0 - HALO + ly;
    if (cj0 < 0 || cj0 >= n0 || cj1 < 0 || cj1 >= n1) continue;
    const bool inrow = tk >= 0 && tk < TY, incol = tj >= 0 && tj < TX;
    double xb[6] = {0, 0, 0, 0, 0, 0};
    double vb[2] = {0, 0};
    const double x[6] = {T.S[r], T.S[RC + r], T.S[2 * RC + r], T.S[3 * RC + r], T.S[4 * RC + r], T.S[5 * RC + r]};
    const double g[4] = {T.G[r], T.G[RC + r], T.G[2 * RC + r], T.G[3 * RC + r]};
#pragma unroll
    for (int d = 0; d < 2; d++) {
      if (d == 0 ? !inrow : !incol) continue;
      double Fb[5] = {0, 0, 0, 0, 0};
      bool any = false;
#pragma unroll
      for (int k = -2; k <= 2; k++) {
        if (k == 0) continue;
        // output cell i = j - k e_d
        const int ti = d == 0 ? tj - k : tj, tk2 = d == 0 ? tk : tk - k;
        if (ti < 0 || ti >= TX || tk2 < 0 || tk2 >= TY) continue;
        const int it = tk2 * TX + ti;
        const int ci = T.x0 + ti, cjj = T.y0 + tk2;
        const int ai = d == 0 ? ci : cjj, ni = d == 0 ? n0 : n1;
        if ((P.bt[d] != 0) && zero3dn(ai, ni)) continue;
        const double rdl2 = 0.5 * (d == 0 ? T.rd0[ti + HALO] : T.rd1[tk2 + HALO]);
        const double wk = -dt * w4(k) * rdl2;
        const int fld[5] = {RHO, M1, M2, EN, d == 0 ? B2 : B1};
#pragma unroll
        for (int q = 0; q < 5; q++) Fb[q] += wk * Lam[fld[q] * ANT + it];
        any = true;
        if (bgon) {
          // e += dt (Bb_d' Bb_d - [d' == d] p_tb) d4_d(v_d') for d' = 0, 1
          const int li = (tk2 + HALO) * RX + ti + HALO;
          const double bb1 = T.G[2 * RC + li], bb2 = T.G[3 * RC + li];
          const double ptb = (P.gamma - 1) * T.G[li] - 0.5 * (P.gamma - 2) * (bb1 * bb1 + bb2 * bb2);
          const double bbk = d == 0 ? bb1 : bb2;
          const double le = Lam[EN * ANT + it] * (-wk);  // dt w4 rdl2 lam_e
          vb[0] += le * (bbk * bb1 - (d == 0 ? ptb : 0.0));
          vb[1] += le * (bbk * bb2 - (d == 1 ? ptb : 0.0));
        }
      }
      if (any) {
        if (d == 0)
          flux_vjp<0>(x, g, P.gamma, Fb, xb);
        else
          flux_vjp<1>(x, g, P.gamma, Fb, xb);
      }
    }
    if (bgon) {
      // v_d = m_d / rho_t
      const double rr = T.R[r];
      xb[M1] += vb[0] * rr;
      xb[M2] += vb[1] * rr;
      xb[RHO] -= (vb[0] * x[M1] + vb[1] * x[M2]) * rr * rr;
    }
    if (P.has_grav && inrow && incol) {
      const int it = tk * TX + tj;
      const double lm1 = Lam[M1 * ANT + it], lm2 = Lam[M2 * ANT + it], le = Lam[EN * ANT + it];
      const double rr = T.R[r], rho = x[RHO];
      xb[RHO] += lm1 * dt * P.g[0] + lm2 * dt * P.g[1] +
                 le * dt * (P.g[0] * x[M1] + P.g[1] * x[M2]) * (rr - rho * rr * rr);
      xb[M1] += le * dt * P.g[0] * rho * rr;
      xb[M2] += le * dt * P.g[1] * rho * rr;
    }
#pragma unroll
    for (int f = 0; f < 6; f++) T.A[f * RC + r] += xb[f];
  }
  __syncthreads();

  // ---- hyperdiffusion (block-cooperative passes) and driver ---------------
  double sb[2] = {0, 0}, th[3] = {0, 0, 0};
  const int lxo = tx + HALO, lyo = ty + HALO, lo = lyo * RX + lxo;
  if (P.hyperdif == 1) {
    // the passes grouped by field (their contributions add up, in any order)
    PassScratch Wa, Wb;
    Wa.Q = T.rd1 + RY;
    Wa.QB = Wa.Q + RC;
    Wa.RR = Wa.QB + 2 * RC;
    Wa.T5 = Wa.RR + ARSZ;
    Wa.RB = Wa.T5 + ARSZ;
    Wa.code = reinterpret_cast<int*>(Wa.RB + ARSZ);
    Wb = Wa;
    Wb.QB = Wa.QB + RC;
#define HPA(W, K, C, D) hyp_pass_adj<K, C, D>(T, I, P, W, tid, active, lxo, lyo, gi, gj, Lam, sb)
    adj_stage_q<0, 0>(T, I, P, Wa, tid);
    __syncthreads();
    HPA(Wa, 0, 0, 0); HPA(Wa, 0, 0, 1);
    adj_flush_q<0, 0>(T, I, P, Wa, tid);
    adj_stage_q<1, 0>(T, I, P, Wb, tid);
    __syncthreads();
    HPA(Wb, 1, 0, 0); HPA(Wb, 1, 0, 1);
    adj_flush_q<1, 0>(T, I, P, Wb, tid);
    adj_stage_q<2, 0>(T, I, P, Wa, tid);
    __syncthreads();
    HPA(Wa, 2, 0, 0); HPA(Wa, 2, 0, 1);
    adj_flush_q<2, 0>(T, I, P, Wa, tid);
    adj_stage_q<2, 1>(T, I, P, Wb, tid);
    __syncthreads();
    HPA(Wb, 2, 1, 0); HPA(Wb, 2, 1, 1);
    adj_flush_q<2, 1>(T, I, P, Wb, tid);
    adj_stage_q<3, 1>(T, I, P, Wa, tid);
    __syncthreads();
    HPA(Wa, 3, 1, 0);
    adj_flush_q<3, 1>(T, I, P, Wa, tid);
    adj_stage_q<3, 0>(T, I, P, Wb, tid);
    __syncthreads();
    HPA(Wb, 3, 0, 1);
    adj_flush_q<3, 0>(T, I, P, Wb, tid);
    __syncthreads();
#undef HPA
  }
  if (active) {
    if (P.driver == SMAUG_DRIVER_GAUSS) {
      // m_1 += dt v (rho + rho_b), v = amp sin(2 pi t/P) prod_d exp(-(x_d-x0_d)^2/s_d^2)
      const double tt = I.tstage;
      double E = 1.0, dEx0 = 0.0;
      if (P.drv_sigma[0] > 0) {
        const double xx = I.pos[0][gi] - P.drv_x0[0];
        E *= exp(-xx * xx / (P.drv_sigma[0] * P.drv_sigma[0]));
      }
      if (P.drv_sigma[1] > 0) {
        const double xx = I.pos[1][gj] - P.drv_x0[1];
        E *= exp(-xx * xx / (P.drv_sigma[1] * P.drv_sigma[1]));
        dEx0 = 2.0 * xx / (P.drv_sigma[1] * P.drv_sigma[1]);
      }
      double sn = 1.0, dsdP = 0.0;
      if (P.drv_period > 0) {
        const double w = 2.0 * M_PI / P.drv_period;
        sn = sin(tt * w);
        dsdP = cos(tt * w) * (-2.0 * M_PI * tt / (P.drv_period * P.drv_period));
      }
      const double rt = T.v(RHO, lo) + T.v(RHOB, lo);
      const double a = lam[M1] * dt;
      const double v = P.drv_amp * sn * E;
      sadd(T.A + RHO * RC + lo, a * v);
      th[0] += a * sn * E * rt;
      th[1] += a * P.drv_amp * E * dsdP * rt;
      th[2] += a * v * dEx0 * rt;
    }
  }
  __syncthreads();

  // ---- flush: one atomic add per region cell and field --------------------
  for (int r = tid; r < RC; r += ANT) {
    const int lx = r % RX, ly = r / RX;
    const int cx = T.x0 - HALO + lx, cy = T.y0 - HALO + ly;
    if (cx < 0 || cx >= n0 || cy < 0 || cy >= n1) continue;
    const long c = (long)cy * n0 + cx;
#pragma unroll
    for (int f = 0; f < 6; f++) {
      const double v = T.A[f * RC + r];
      if (v != 0.0) atomicAdd(I.Xb + f * nc + c, v);
    }
  }
  // block sums of cmax-bar and theta-bar
  double vals[5] = {sb[0], sb[1], th[0], th[1], th[2]};
#pragma unroll
  for (int k = 0; k < 5; k++)
    for (int o = 16; o > 0; o >>= 1) vals[k] += __shfl_xor_sync(0xffffffffu, vals[k], o);
  if ((tid & 31) == 0) {
    if (vals[0] != 0.0) atomicAdd(I.sbar + 0, vals[0]);
    if (vals[1] != 0.0) atomicAdd(I.sbar + 1, vals[1]);
    if (vals[2] != 0.0) atomicAdd(I.thbar + 0, vals[2]);
    if (vals[3] != 0.0) atomicAdd(I.thbar + 1, vals[3]);
    if (vals[4] != 0.0) atomicAdd(I.thbar + 2, vals[4]);
  }
}

// cmax-bar to the cell that attains each maximum: Xb(cell) += sbar_d dcfast_d/dX
__global__ void adj_cmax2d(const KParams P, const double* X, const double* bg, const int* argmax,
                           const double* sbar, double* Xb) {
  const int d = threadIdx.x;
  if (d >= 2) return;
  const long nc = P.ncell;
  const long c = argmax[d];
  if (c < 0 || c >= nc || sbar[d] == 0.0) return;
  double x[6], g[4], xb[6] = {0, 0, 0, 0, 0, 0};
  for (int f = 0; f < 6; f++) x[f] = X[f * nc + c];
  for (int f = 0; f < 4; f++) g[f] = bg[f * nc + c];
  cfast_vjp(P.gamma, x, g, d, sbar[d], xb);
  for (int f = 0; f < 6; f++) atomicAdd(Xb + f * nc + c, xb[f]);
}

// per-dimension max of the fast speed over all cells and the first cell
// that attains it (two passes: the max, then the smallest index equal to it)
__global__ void cmax_value2d(const KParams P, const double* X, const double* bg, unsigned long long* mx) {
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nc = P.ncell;
  double v[2] = {0, 0};
  if (c < nc)
    for (int d = 0; d < 2; d++)
      v[d] = cfast2(P.gamma, X[c], X[nc + c], X[2 * nc + c], X[3 * nc + c], X[4 * nc + c], X[5 * nc + c],
                    bg[c], bg[nc + c], bg[2 * nc + c], bg[3 * nc + c], d);
  for (int d = 0; d < 2; d++) {
    double w = v[d] > 0 ? v[d] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w = dmax0(w, __shfl_xor_sync(0xffffffffu, w, o));
    if ((threadIdx.x & 31) == 0) atomicMax(mx + d, (unsigned long long)__double_as_longlong(w));
  }
}

// the same for the four stage inputs of a step in one pass each
struct X4 {
  const double* x[4];
};

__global__ void cmax4_value2d(const KParams P, const X4 X, const double* bg, unsigned long long* mx) {
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nc = P.ncell;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (c < nc) {
    const double g0 = bg[c], g1 = bg[nc + c], g2 = bg[2 * nc + c], g3 = bg[3 * nc + c];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double* x = X.x[s];
#pragma unroll
      for (int d = 0; d < 2; d++)
        v[2 * s + d] = cfast2(P.gamma, x[c], x[nc + c], x[2 * nc + c], x[3 * nc + c], x[4 * nc + c],
                              x[5 * nc + c], g0, g1, g2, g3, d);
    }
  }
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double w = v[k] > 0 ? v[k] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w = dmax0(w, __shfl_xor_sync(0xffffffffu, w, o));
    if ((threadIdx.x & 31) == 0) atomicMax(mx + k, (unsigned long long)__double_as_longlong(w));
  }
}

__global__ void cmax4_argmax2d(const KParams P, const X4 X, const double* bg,
                               const unsigned long long* mx, int* arg) {
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nc = P.ncell;
  if (c >= nc) return;
  const double g0 = bg[c], g1 = bg[nc + c], g2 = bg[2 * nc + c], g3 = bg[3 * nc + c];
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const double* x = X.x[s];
#pragma unroll
    for (int d = 0; d < 2; d++) {
      const double v = cfast2(P.gamma, x[c], x[nc + c], x[2 * nc + c], x[3 * nc + c], x[4 * nc + c],
                              x[5 * nc + c], g0, g1, g2, g3, d);
      if (v == __longlong_as_double((long long)mx[2 * s + d])) atomicMin(arg + 2 * s + d, (int)c);
    }
  }
}

}  // namespace

// ---- host side: one RK4 step and its adjoint on caller device buffers -------
namespace {
__global__ void ghost_fill_adj2d(const KParams P, double* u) {
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (c >= P.ncell) return;
  const int i = (int)(c % P.n0), j = (int)(c / P.n0);
  const int si = ghost_source(i, P.n0, P.bc[0]), sj = ghost_source(j, P.n1, P.bc[1]);
  if (si == i && sj == j) return;
  const long s = (long)sj * P.n0 + si;
  for (int f = 0; f < 6; f++) u[f * P.ncell + c] = u[f * P.ncell + s];
}

__global__ void set_dt_t(double* dtb, double* tb, double dt, double t) {
  dtb[0] = dt;
  dtb[1] = dt;
  tb[0] = t;
  tb[1] = t;
}

// G^T x at cell c: the value plus those of its ghost images (interior
// cells), 0 at ghost cells
__device__ __forceinline__ double fold_at(const KParams& P, const double* x, long c, int i, int j) {
  if (i < 2 || i > P.n0 - 3 || j < 2 || j > P.n1 - 3) return 0.0;
  int ix[3], iy[3];
  ix[0] = i;
  iy[0] = j;
  const int nx = 1 + ghost_images(i, P.n0, P.bc[0], ix + 1);
  const int ny = 1 + ghost_images(j, P.n1, P.bc[1], iy + 1);
  double s = x[c];
  if (nx == 1 && ny == 1) return s;
  double g = 0.0;
  for (int b = 0; b < ny; b++)
    for (int a = 0; a < nx; a++) {
      if (a == 0 && b == 0) continue;
      g += x[(long)iy[b] * P.n0 + ix[a]];
    }
  return s + g;
}

// start of the backward: W = G^T ubar_next, ubar = W, k-bar_4 = W / 6
__global__ void adj_head(const KParams P, const double* ubn, double* W, double* ubar, double* Kb, double w4) {
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nc = P.ncell;
  if (c >= nc) return;
  const int i = (int)(c % P.n0), j = (int)(c / P.n0);
  for (int f = 0; f < 6; f++) {
    const double w = fold_at(P, ubn + f * nc, c, i, j);
    W[f * nc + c] = w;
    ubar[f * nc + c] = w;
    Kb[f * nc + c] = w4 * w;
  }
}

// end of stage s of the backward: t_s = G^T X-bar, ubar += t_s and (s > 0)
// k-bar_{s-1} = wk W + half t_s
__global__ void adj_tail(const KParams P, const double* Xb, const double* W, double* ubar, double* Kb,
                         double wk, double half, int more) {
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nc = P.ncell;
  if (c >= nc) return;
  const int i = (int)(c % P.n0), j = (int)(c / P.n0);
  for (int f = 0; f < 6; f++) {
    const double x = fold_at(P, Xb + f * nc, c, i, j);
    ubar[f * nc + c] += x;
    if (more) Kb[f * nc + c] = fma(half, x, wk * W[f * nc + c]);
  }
}
}  // namespace

struct Adjoint {
  smaug_params_t P{};
  KParams K{};
  long nc = 0;
  double* X[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // X1..X4, U'
  double* acc = nullptr;
  double* bg = nullptr;
  double* delx[2] = {nullptr, nullptr};
  double* pos[2] = {nullptr, nullptr};
  int* pad[2] = {nullptr, nullptr};
  unsigned long long* ring = nullptr;  // 3 slots x 3
  double* dtb = nullptr;               // [2]
  double* tb = nullptr;                // [2]
  int* flags = nullptr;
  double* W = nullptr;                 // folded adjoint of U'
  double* Kb = nullptr;                // k-bar of the current stage
  double* Xb = nullptr;                // X-bar of the current stage
  double* sbar = nullptr;              // [2]
  unsigned long long* mx = nullptr;    // [4][2] stage CFL maxima
  int* arg = nullptr;                  // [4][2] their cells
  double* tape = nullptr;              // [nslots][4][6][nc] stage inputs of taped steps
  int nslots = 0;
  double* ubar2 = nullptr;             // [6][nc] second adjoint buffer of the range backward
};

static void free_adj(Adjoint* a) {
  if (!a) return;
  for (auto* p : a->X) cudaFree(p);
  cudaFree(a->acc);
  cudaFree(a->bg);
  for (int d = 0; d < 2; d++) {
    cudaFree(a->delx[d]);
    cudaFree(a->pos[d]);
    cudaFree(a->pad[d]);
  }
  cudaFree(a->ring);
  cudaFree(a->dtb);
  cudaFree(a->tb);
  cudaFree(a->flags);
  cudaFree(a->W);
  cudaFree(a->Kb);
  cudaFree(a->Xb);
  cudaFree(a->sbar);
  cudaFree(a->mx);
  cudaFree(a->arg);
  cudaFree(a->tape);
  cudaFree(a->ubar2);
  delete a;
}

static size_t adj_smem() {
  return sizeof(double) * ((size_t)17 * RC + 6 * ANT + 2 * (RX + RY) + 3 * RC + 3 * ARSZ) +
         sizeof(int) * ARSZ;
}

static int adj_create(const smaug_params_t* p, const double* w, const double* pos, Adjoint** out) {
  if (!p || !w || !pos || !out) return set_error(SMAUG_E_INVALID, "null argument");
  if (p->version != SMAUG_PARAMS_VERSION) return set_error(SMAUG_E_INVALID, "parameter block version");
  if (p->ndim != 2) return set_error(SMAUG_E_UNSUPPORTED, "the adjoint is 2D");
  if (p->integrator != SMAUG_INT_RK4) return set_error(SMAUG_E_UNSUPPORTED, "the adjoint differentiates RK4 steps");
  if (p->precision != SMAUG_PREC_FP64) return set_error(SMAUG_E_UNSUPPORTED, "the adjoint is FP64");
  if (p->moddton != 0) return set_error(SMAUG_E_UNSUPPORTED, "the adjoint holds dt fixed: set moddton = 0");
  if (p->stencil_order == 6) return set_error(SMAUG_E_UNSUPPORTED, "the adjoint is of the 4th-order stencil");
  if (p->driver == SMAUG_DRIVER_GAUSS_STEP)
    return set_error(SMAUG_E_UNSUPPORTED, "the adjoint's driver acts in every step");
  if (p->n[0] < 8 || p->n[1] < 8) return set_error(SMAUG_E_INVALID, "grid too small");
  for (int d = 0; d < 2; d++) {
    const int b = p->boundtype[d][0];
    if (b != p->boundtype[d][1] ||
        (b != SMAUG_BC_PERIODIC && b != SMAUG_BC_CONTCD4 && b != SMAUG_BC_CONT && b != SMAUG_BC_SYMM))
      return set_error(SMAUG_E_UNSUPPORTED, "dim %d: boundary type %d not supported", d, b);
  }
  Adjoint* a = new Adjoint();
  auto fail = [&](int code) { free_adj(a); return code; };
  a->P = *p;
  const int n0 = p->n[0], n1 = p->n[1];
  const long nc = (long)n0 * n1;
  a->nc = nc;
  // metric (initgrid) as 1D arrays, positions along each axis
  std::vector<double> ps(pos, pos + 2 * nc), dl(2 * nc);
  int rc = grid_metric(2, p->n, ps.data(), dl.data());
  if (rc) return fail(rc);
  std::vector<double> dl1[2], ps1[2];
  for (int d = 0; d < 2; d++) {
    const int n = p->n[d];
    dl1[d].resize(n);
    ps1[d].resize(n);
    for (int k = 0; k < n; k++) {
      const long c = d == 0 ? (long)2 * n0 + k : (long)k * n0 + 2;
      dl1[d][k] = dl[(size_t)d * nc + c];
      ps1[d][k] = ps[(size_t)d * nc + c];
    }
  }
  // stray-pad sources (the same rule as the engine's)
  std::vector<int> pads[2];
  {
    const long m0 = n0 + 2, off = n0 + 1;
    pads[0].assign(n1, -1);
    pads[1].assign(n0, -1);
    for (long r = 0; r < n1; r++) {
      const long t = (r + 1) * m0 + (n0 + 1) - off;
      if (p->pad_model == SMAUG_PAD_STRAY && t >= 0 && t < nc) pads[0][r] = (int)t;
    }
    for (long r = 0; r < n0; r++) {
      const long t = (long)(n1 + 1) * m0 + (r + 1) - off;
      if (p->pad_model == SMAUG_PAD_STRAY && t >= 0 && t < nc) pads[1][r] = (int)t;
    }
  }
  KParams& K = a->K;
  K.n0 = n0;
  K.n1 = n1;
  K.n2 = 1;
  K.ncell = nc;
  set_boundaries(K, p, 2);
  for (int d = 0; d < 3; d++) {
    K.dx[d] = p->dx[d];
    K.g[d] = p->g[d];
    K.drv_x0[d] = p->drv_x0[d];
    K.drv_sigma[d] = p->drv_sigma[d];
  }
  K.gamma = p->gamma;
  K.courant = p->courant;
  K.dtmax = p->dtmax;
  for (int f = 0; f < SMAUG_MAXVAR; f++) K.chyp[f] = p->chyp[f];
  K.moddton = 0;
  K.hyperdif = p->hyperdifmom;
  K.has_grav = (p->g[0] != 0.0 || p->g[1] != 0.0);
  K.has_bg = 0;
  for (long c = 6 * nc; c < 10 * nc; c++)
    if (w[c] != 0.0) { K.has_bg = 1; break; }
  K.driver = p->driver;
  K.drv_amp = p->drv_amp;
  K.drv_period = p->drv_period;
#define A_TRY(call)                                                                             \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      return fail(set_error(_e == cudaErrorMemoryAllocation ? SMAUG_E_NOMEM : SMAUG_E_CUDA,    \
                            "%s: %s", #call, cudaGetErrorString(_e)));                         \
  } while (0)
  const size_t eb = sizeof(double) * 6 * nc;
  for (int k = 0; k < 5; k++) A_TRY(cudaMalloc(&a->X[k], eb));
  A_TRY(cudaMalloc(&a->acc, eb));
  A_TRY(cudaMalloc(&a->W, eb));
  A_TRY(cudaMalloc(&a->Kb, eb));
  A_TRY(cudaMalloc(&a->Xb, eb));
  A_TRY(cudaMemset(a->Xb, 0, eb));
  A_TRY(cudaMalloc(&a->bg, sizeof(double) * 4 * nc));
  A_TRY(cudaMemcpy(a->bg, w + 6 * nc, sizeof(double) * 4 * nc, cudaMemcpyHostToDevice));
  for (int d = 0; d < 2; d++) {
    A_TRY(cudaMalloc(&a->delx[d], sizeof(double) * p->n[d]));
    A_TRY(cudaMalloc(&a->pos[d], sizeof(double) * p->n[d]));
    A_TRY(cudaMalloc(&a->pad[d], sizeof(int) * pads[d].size()));
    A_TRY(cudaMemcpy(a->delx[d], dl1[d].data(), sizeof(double) * p->n[d], cudaMemcpyHostToDevice));
    A_TRY(cudaMemcpy(a->pos[d], ps1[d].data(), sizeof(double) * p->n[d], cudaMemcpyHostToDevice));
    A_TRY(cudaMemcpy(a->pad[d], pads[d].data(), sizeof(int) * pads[d].size(), cudaMemcpyHostToDevice));
  }
  A_TRY(cudaMalloc(&a->ring, sizeof(unsigned long long) * 9));
  A_TRY(cudaMalloc(&a->dtb, sizeof(double) * 2));
  A_TRY(cudaMalloc(&a->tb, sizeof(double) * 2));
  A_TRY(cudaMalloc(&a->flags, sizeof(int)));
  A_TRY(cudaMalloc(&a->sbar, sizeof(double) * 2));
  A_TRY(cudaMalloc(&a->mx, sizeof(unsigned long long) * 8));
  A_TRY(cudaMalloc(&a->arg, sizeof(int) * 8));
  A_TRY(cudaMemset(a->flags, 0, sizeof(int)));
  A_TRY(stage2d_set_attributes());
  A_TRY(cudaFuncSetAttribute(adj_stage2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adj_smem()));
#undef A_TRY
  *out = a;
  return SMAUG_OK;
}

#define G_LAUNCH(n) (unsigned)(((n) + 255) / 256), 256, 0, st

// forward RK4 step: X[0] = G(u) ... X[3] = stage 4 input, X[4] = U'
// One RK4 step from u; the stage inputs go to Xs[0..3] (the handle's own
// buffers or a tape slot), the result to X[4].
static int adj_fwd(Adjoint* a, const double* u, double t, cudaStream_t st, double* const* Xs) {
  const long nc = a->nc;
  const size_t eb = sizeof(double) * 6 * nc;
  CUDA_TRY(cudaMemcpyAsync(Xs[0], u, eb, cudaMemcpyDeviceToDevice, st));
  ghost_fill_adj2d<<<G_LAUNCH(nc)>>>(a->K, Xs[0]);
  CUDA_TRY(cudaMemsetAsync(a->ring, 0, sizeof(unsigned long long) * 9, st));
  cmax_value2d<<<G_LAUNCH(nc)>>>(a->K, Xs[0], a->bg, a->ring);
  set_dt_t<<<1, 1, 0, st>>>(a->dtb, a->tb, a->P.dt, t);
  CUDA_TRY(cudaGetLastError());
  for (int s = 0; s < 4; s++) {
    KBufs B{};
    B.uin = Xs[s];
    B.un = Xs[0];
    B.uout = s < 3 ? Xs[s + 1] : a->X[4];
    B.acc = a->acc;
    B.bg = a->bg;
    for (int d = 0; d < 2; d++) {
      B.delx[d] = a->delx[d];
      B.pos[d] = a->pos[d];
      B.padsrc[d] = a->pad[d];
    }
    B.cmax_in = reinterpret_cast<const double*>(a->ring + 3 * (s % 3));
    B.cmax_out = a->ring + 3 * ((s + 1) % 3);
    B.cmax_clear = a->ring + 3 * ((s + 2) % 3);
    B.dt_prev = a->dtb;
    B.dt_new = a->dtb + 1;
    B.t_prev = a->tb;
    B.t_new = a->tb + 1;
    B.flags = a->flags;
    B.mode = SMAUG_INT_RK4;
    B.stage = s;
    CUDA_TRY(launch_stage2d_any(SMAUG_INT_RK4, false, a->K, B, st));
  }
  return SMAUG_OK;
}

// The adjoint of one step from u.  Xs: the step's stage inputs from a tape
// slot, or null to recompute them from u.
static int adj_bwd(Adjoint* a, const double* u, const double* ubar_next, double* ubar, double* thbar,
                   double t, cudaStream_t st, double* const* Xs, bool thbar_accumulate = false) {
  if (!Xs) {
    int rc = adj_fwd(a, u, t, st, a->X);
    if (rc) return rc;
    Xs = a->X;
  }
  const long nc = a->nc;
  // CFL maxima of the four stage inputs and the cells that attain them
  CUDA_TRY(cudaMemsetAsync(a->mx, 0, sizeof(unsigned long long) * 8, st));
  CUDA_TRY(cudaMemsetAsync(a->arg, 0x7f, sizeof(int) * 8, st));
  const X4 x4{{Xs[0], Xs[1], Xs[2], Xs[3]}};
  cmax4_value2d<<<G_LAUNCH(nc)>>>(a->K, x4, a->bg, a->mx);
  cmax4_argmax2d<<<G_LAUNCH(nc)>>>(a->K, x4, a->bg, a->mx, a->arg);
  const double wk[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};  // k-bar = wk W + ...
  const double half[4] = {0.0, 0.5, 0.5, 1.0};   // X_s = U + half[s] k_{s-1}
  // W = G^T ubar_next; ubar = W; k-bar of stage 4 = W / 6
  adj_head<<<G_LAUNCH(nc)>>>(a->K, ubar_next, a->W, ubar, a->Kb, wk[3]);
  if (!thbar_accumulate) CUDA_TRY(cudaMemsetAsync(thbar, 0, sizeof(double) * 3, st));
  const double dt = a->P.dt;
  const double ts[4] = {t, t + 0.5 * dt, t + 0.5 * dt, t + dt};
  const size_t eb = sizeof(double) * 6 * nc;
  for (int s = 3; s >= 0; s--) {
    CUDA_TRY(cudaMemsetAsync(a->Xb, 0, eb, st));
    CUDA_TRY(cudaMemsetAsync(a->sbar, 0, sizeof(double) * 2, st));
    AdjIn I{};
    I.X = Xs[s];
    I.bg = a->bg;
    I.lam = a->Kb;
    I.Xb = a->Xb;
    I.sbar = a->sbar;
    I.thbar = thbar;
    I.cmax = reinterpret_cast<const double*>(a->mx + 2 * s);
    for (int d = 0; d < 2; d++) {
      I.delx[d] = a->delx[d];
      I.pos[d] = a->pos[d];
      I.padsrc[d] = a->pad[d];
    }
    I.dt = dt;
    I.tstage = ts[s];
    dim3 grid((a->K.n0 - 4 + TX - 1) / TX, (a->K.n1 - 4 + TY - 1) / TY);
    adj_stage2d<<<grid, dim3(TX, TY), adj_smem(), st>>>(a->K, I);
    adj_cmax2d<<<1, 32, 0, st>>>(a->K, Xs[s], a->bg, a->arg + 2 * s, a->sbar, a->Xb);
    // t_s = G^T X-bar; ubar += t_s; k-bar of the previous stage = wk W + half[s] t_s
    adj_tail<<<G_LAUNCH(nc)>>>(a->K, a->Xb, a->W, ubar, a->Kb, s > 0 ? wk[s - 1] : 0.0, half[s], s > 0);
    CUDA_TRY(cudaGetLastError());
  }
  return SMAUG_OK;
}

// y += x over n doubles
__global__ void add_inplace(double* y, const double* x, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

// stage-input pointers of tape slot `slot`
static int tape_slot(Adjoint* a, int slot, double** Xs) {
  if (slot < 0 || slot >= a->nslots)
    return set_error(SMAUG_E_INVALID, "tape slot %d outside [0, %d)", slot, a->nslots);
  for (int s = 0; s < 4; s++) Xs[s] = a->tape + ((size_t)slot * 4 + s) * 6 * a->nc;
  return SMAUG_OK;
}

}  // namespace smaug

using smaug::Adjoint;
static Adjoint* HA(smaug_adj_t h) { return reinterpret_cast<Adjoint*>(h); }

extern "C" int smaug_adj_create(const smaug_params_t* p, const double* w, const double* pos, smaug_adj_t* out) {
  smaug::clear_error();
  if (!out) return smaug::set_error(SMAUG_E_INVALID, "null handle pointer");
  *out = nullptr;
  Adjoint* a = nullptr;
  int rc = smaug::adj_create(p, w, pos, &a);
  if (rc) return rc;
  *out = reinterpret_cast<smaug_adj_t>(a);
  return SMAUG_OK;
}

extern "C" int smaug_adj_set_driver(smaug_adj_t h, double amp, double period, double x0) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Adjoint* a = HA(h);
  a->K.drv_amp = amp;
  a->K.drv_period = period;
  a->K.drv_x0[1] = x0;
  return SMAUG_OK;
}

extern "C" int smaug_adj_forward(smaug_adj_t h, const double* u, double* u_next, double t, void* stream) {
  smaug::clear_error();
  if (!h || !u || !u_next) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Adjoint* a = HA(h);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = smaug::adj_fwd(a, u, t, st, a->X);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(u_next, a->X[4], sizeof(double) * 6 * a->nc, cudaMemcpyDeviceToDevice, st));
  return SMAUG_OK;
}

extern "C" int smaug_adj_tape_reserve(smaug_adj_t h, int32_t nslots) {
  smaug::clear_error();
  if (!h || nslots < 0) return smaug::set_error(SMAUG_E_INVALID, "bad argument");
  Adjoint* a = HA(h);
  if (nslots <= a->nslots) return SMAUG_OK;
  CUDA_TRY(cudaDeviceSynchronize());
  cudaFree(a->tape);
  a->tape = nullptr;
  a->nslots = 0;
  const size_t bytes = sizeof(double) * (size_t)nslots * 4 * 6 * a->nc;
  if (cudaMalloc(&a->tape, bytes) != cudaSuccess) {
    cudaGetLastError();
    a->tape = nullptr;
    return smaug::set_error(SMAUG_E_NOMEM, "tape of %d steps (%zu bytes)", nslots, bytes);
  }
  a->nslots = nslots;
  return SMAUG_OK;
}

extern "C" int smaug_adj_forward_tape(smaug_adj_t h, const double* u, double* u_next, double t,
                                      int32_t slot, void* stream) {
  smaug::clear_error();
  if (!h || !u || !u_next) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Adjoint* a = HA(h);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* Xs[4];
  int rc = smaug::tape_slot(a, slot, Xs);
  if (!rc) rc = smaug::adj_fwd(a, u, t, st, Xs);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(u_next, a->X[4], sizeof(double) * 6 * a->nc, cudaMemcpyDeviceToDevice, st));
  return SMAUG_OK;
}

extern "C" int smaug_adj_backward_tape(smaug_adj_t h, int32_t slot, const double* ubar_next, double* ubar,
                                       double* thbar, double t, void* stream) {
  smaug::clear_error();
  if (!h || !ubar_next || !ubar || !thbar) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Adjoint* a = HA(h);
  double* Xs[4];
  int rc = smaug::tape_slot(a, slot, Xs);
  if (rc) return rc;
  return smaug::adj_bwd(a, nullptr, ubar_next, ubar, thbar, t, static_cast<cudaStream_t>(stream), Xs);
}

extern "C" int smaug_adj_backward_tape_range(smaug_adj_t h, int32_t slot_lo, int32_t nsteps,
                                             const double* gsteps, double* ubar, double* thbar,
                                             double t0, int32_t n_lo, void* stream) {
  smaug::clear_error();
  if (!h || !ubar || !thbar || nsteps < 0) return smaug::set_error(SMAUG_E_INVALID, "bad argument");
  Adjoint* a = HA(h);
  if (slot_lo < 0 || slot_lo + nsteps > a->nslots)
    return smaug::set_error(SMAUG_E_INVALID, "tape slots [%d, %d) outside [0, %d)", slot_lo, slot_lo + nsteps,
                            a->nslots);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long n6 = 6 * a->nc;
  if (!a->ubar2) CUDA_TRY(cudaMalloc(&a->ubar2, sizeof(double) * n6));
  double* cur = ubar;
  for (int k = nsteps - 1; k >= 0; k--) {
    if (gsteps) smaug::add_inplace<<<(unsigned)((n6 + 255) / 256), 256, 0, st>>>(cur, gsteps + k * n6, n6);
    double* Xs[4];
    int rc = smaug::tape_slot(a, slot_lo + k, Xs);
    if (rc) return rc;
    double* next = (cur == ubar) ? a->ubar2 : ubar;
    // the time of absolute step n_lo + k, formed as the caller forms it
    const double t = t0 + (double)(n_lo + k) * a->P.dt;
    rc = smaug::adj_bwd(a, nullptr, cur, next, thbar, t, st, Xs, true);
    if (rc) return rc;
    cur = next;
  }
  if (cur != ubar) CUDA_TRY(cudaMemcpyAsync(ubar, cur, sizeof(double) * n6, cudaMemcpyDeviceToDevice, st));
  return SMAUG_OK;
}

extern "C" int smaug_adj_backward(smaug_adj_t h, const double* u, const double* ubar_next, double* ubar,
                                  double* thbar, double t, void* stream) {
  smaug::clear_error();
  if (!h || !u || !ubar_next || !ubar || !thbar) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  return smaug::adj_bwd(HA(h), u, ubar_next, ubar, thbar, t, static_cast<cudaStream_t>(stream), nullptr);
}

extern "C" int smaug_adj_destroy(smaug_adj_t h) {
  smaug::clear_error();
  if (h) smaug::free_adj(HA(h));
  return SMAUG_OK;
}
