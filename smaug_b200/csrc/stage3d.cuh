// stage3d.cuh -- fused 3D stage kernel, included by stage3d.cu.
//
// One launch evaluates the reference's whole spatial operator (the 3D build,
// -DUSE_SAC_3D, of src/iosmaug.c:631-835) for an 8x8x4 tile of interior
// cells and writes the stage result, its ghost images and the per-dimension
// fast-speed maxima.  The terms and their arithmetic are those of the 2D
// kernel (stage2d.cuh) with three momentum and field components:
//   fluxes along each dimension and their 4th-order divergence
//     (src/centdiff1.cu:51-197, src/centdiff2.cu:203-323, grad3dn)
//   background energy coupling e -= dt p_tb dv_d/dx_d,
//     e += dt Bb_i Bb_d dv_d/dx_i (src/centdiff2.cu:80-115); the second sum
//     is evaluated in the pass of the derivative's direction i
//   gravity (src/centdiff2.cu:118-154)
//   hyperdiffusion of rho, e, m_c, B_c along every dimension
//     (src/hyperdifvisc1{r,l}.cu, src/hyperdif*source*.cu); the passes of
//     one field share one staging of q
//   user driver, stage combine, ghost images, CFL maxima.
// Sums per cell are reordered against the reference (per field instead of
// per dimension); agreement stays at rounding level.  The mixed precision
// form (template MIX) is the one of stage2d.cuh: float perturbation storage
// and hyperdiffusion arithmetic, double everywhere else.
//
// The state is read from global memory (L1/L2 resident across the passes of
// a block); shared memory holds 1/rho_t and q on the tile's 3-cell box,
// the per-axis metric, and one union of phase scratch:
//   flux phase:  7 flux arrays + 3 velocity arrays on the tile +-2 along the
//                direction
//   hyperdiffusion phase: q of one field on the box (shared by the passes
//                of all directions), the nu ratio on the tile +-1 across the
//                direction extended by one cell along it, two cross-term
//                arrays on the tile +-1 across the direction.
#pragma once

// (included inside namespace smaug)
namespace s3 {
#ifndef SMAUG_T3X
#define SMAUG_T3X 8
#endif
#ifndef SMAUG_T3Y
#define SMAUG_T3Y 8
#endif
#ifndef SMAUG_T3Z
#define SMAUG_T3Z 4
#endif
#ifndef SMAUG_MINB3D
#define SMAUG_MINB3D 3  // resident blocks per SM the 3D stage is compiled for
#endif
constexpr int T0 = SMAUG_T3X, T1 = SMAUG_T3Y, T2 = SMAUG_T3Z;  // tile (x fastest)
constexpr int NT = T0 * T1 * T2;       // threads per block, one cell each
constexpr int H = 3;                   // box halo
constexpr int BX = T0 + 2 * H, BY = T1 + 2 * H, BZ = T2 + 2 * H;
constexpr int BC = BX * BY * BZ;
constexpr int BS1 = BX, BS2 = BX * BY;  // box strides
__host__ __device__ constexpr int max3(int a, int b, int c) {
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}
// flux arrays: the tile +-2 (+-3 for the 6th-order derivative) along the direction
template <bool O6>
__host__ __device__ constexpr int fa() {
  return max3((T0 + (O6 ? 6 : 4)) * T1 * T2, T0 * (T1 + (O6 ? 6 : 4)) * T2, T0 * T1 * (T2 + (O6 ? 6 : 4)));
}
constexpr int NA = max3(T0 * (T1 + 2) * (T2 + 2), (T0 + 2) * T1 * (T2 + 2), (T0 + 2) * (T1 + 2) * T2);
// ratio area: the nu area extended by one cell below along the direction
constexpr int RA = max3((T0 + 1) * (T1 + 2) * (T2 + 2), (T0 + 2) * (T1 + 1) * (T2 + 2),
                        (T0 + 2) * (T1 + 2) * (T2 + 1));
constexpr int HYP_SCR = BC + RA + 2 * NA;
constexpr int NMET = 2 * (BX + BY + BZ);
template <bool MIX, bool O6 = false>
__host__ __device__ constexpr size_t union_bytes() {
  return 10 * fa<O6>() * sizeof(double) > HYP_SCR * sizeof(typename Form<MIX>::H)
             ? 10 * fa<O6>() * sizeof(double)
             : HYP_SCR * sizeof(typename Form<MIX>::H);
}
template <bool MIX, bool O6 = false>
__host__ __device__ constexpr size_t smem_bytes() {
  return sizeof(double) * (BC + NMET) + union_bytes<MIX, O6>() + sizeof(int) * BC;
}
__host__ __device__ constexpr int tdim(int d) { return d == 0 ? T0 : (d == 1 ? T1 : T2); }
__host__ __device__ constexpr int bstride(int d) { return d == 0 ? 1 : (d == 1 ? BS1 : BS2); }
}  // namespace s3

struct Box3 {
  double* R;       // [BC] 1/rho_t on the box
  double* dl[3];   // cell widths over the box extent of each axis
  double* rd[3];   // reciprocals
  void* U;         // union scratch
  int* C;          // [BC] q source code per box cell (box_code)
  int o[3];        // global coordinate of box index 0 per axis
  bool inner;      // the box lies inside the grid and off its pads
};

// q of a hyperdiffusion field from global memory (src/hyperdifvisc1r.cu:1225-1253)
template <typename ST, int KIND, int COMP>
__device__ __forceinline__ double hq3_global(const ST* u, const KBufs& B, long nc, long c) {
  const double rho = __ldg(u + c);
  if (KIND == 0) return rho;
  if (KIND == 3) return __ldg(u + (B3 + COMP) * nc + c);
  const double r = 1.0 / (rho + __ldg(B.bg + GRB * nc + c));
  if (KIND == 2) return (double)__ldg(u + (M3 + COMP) * nc + c) * r;
  double m2 = 0, b2 = 0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double m = __ldg(u + (M3 + a) * nc + c), b = __ldg(u + (B3 + a) * nc + c);
    m2 += m * m;
    b2 += b * b;
  }
  return (double)__ldg(u + E3 * nc + c) - 0.5 * (b2 + m2 * r);
}

// distance of box index l outside the tile range [H, H+T)
__device__ __forceinline__ int outside(int l, int T) {
  return l < s3::H ? s3::H - l : (l >= s3::H + T ? l - (s3::H + T - 1) : 0);
}

// (A) q of one field on the box: every cell within 1 of the tile on all
// axes but one, and within 3 on that one.  Pads: index -1 along an axis is
// the copy of index 5 (bc_hyperdifl), index n the stray tmp6 store of
// hyperdifvisc1r_parallel (source table B.padsrc).
template <bool MIX, int KIND, int COMP>
__device__ __forceinline__ void stage_q(const Box3& X, const KParams& P, const KBufs& B, int tid) {
  using HT = typename Form<MIX>::H;
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  HT* Q = static_cast<HT*>(X.U);
  const long nc = P.ncell;
  for (int r = tid; r < s3::BC; r += s3::NT) {
    const int code = X.C[r];
    double q = 0.0;
    if (code >= 0) {
      const long c = code;
      if (KIND == 0) {
        q = __ldg(u + c);
      } else if (KIND == 3) {
        q = __ldg(u + (B3 + COMP) * nc + c);
      } else if (KIND == 2) {
        q = (double)__ldg(u + (M3 + COMP) * nc + c) * X.R[r];
      } else {
        double m2 = 0, b2 = 0;
#pragma unroll
        for (int a = 0; a < 3; a++) {
          const double m = __ldg(u + (M3 + a) * nc + c), b = __ldg(u + (B3 + a) * nc + c);
          m2 += m * m;
          b2 += b * b;
        }
        q = (double)__ldg(u + E3 * nc + c) - 0.5 * (b2 + m2 * X.R[r]);
      }
    } else if (code <= -2) {
      q = hq3_global<ST, KIND, COMP>(u, B, nc, (long)(-2 - code));
    }
    Q[r] = (HT)q;
  }
  __syncthreads();
}

// Source code of box cell r for the q stagings (computed once per block):
// the cell index when the cell is in the grid and read by some pass, -2 - src
// for a pad (index -1 along an axis: the cell with that coordinate 5,
// bc_hyperdifl; index n: the stray tmp6 store of hyperdifvisc1r_parallel,
// source table B.padsrc), -1 for a zero.  The passes read the cells within 1
// of the tile on all axes but one and within 3 on that one.
__device__ __forceinline__ int box_code(const Box3& X, const KParams& P, const KBufs& B, int lx, int ly,
                                        int lz) {
  const int ox = outside(lx, s3::T0), oy = outside(ly, s3::T1), oz = outside(lz, s3::T2);
  if ((ox > 1) + (oy > 1) + (oz > 1) > 1) return -1;
  const int n0 = P.n0, n1 = P.n1, n2 = P.n2;
  const int g0 = X.o[0] + lx, g1 = X.o[1] + ly, g2 = X.o[2] + lz;
  const bool i0 = g0 >= 0 && g0 < n0, i1 = g1 >= 0 && g1 < n1, i2 = g2 >= 0 && g2 < n2;
  if (i0 && i1 && i2) return (int)(((long)g2 * n1 + g1) * n0 + g0);
  int src = -1;
  if (!i0 && i1 && i2) {
    if (g0 == -1) src = (int)(((long)g2 * n1 + g1) * n0 + 5);
    else if (g0 == n0) src = B.padsrc[0][(long)g2 * n1 + g1];
  } else if (i0 && !i1 && i2) {
    if (g1 == -1) src = (int)(((long)g2 * n1 + 5) * n0 + g0);
    else if (g1 == n1) src = B.padsrc[1][(long)g2 * n0 + g0];
  } else if (i0 && i1 && !i2) {
    if (g2 == -1) src = (int)(((long)5 * n1 + g1) * n0 + g0);
    else if (g2 == n2) src = B.padsrc[2][(long)g1 * n0 + g0];
  }
  return src >= 0 ? -2 - src : -1;
}

// One hyperdiffusion pass on staged q: field kind (0 rho, 1 energy,
// 2 momentum, 3 B), component COMP, direction DIM.
template <bool MIX, int KIND, int COMP, int DIM>
__device__ __forceinline__ void hyper_pass3(const Box3& X, const KParams& P, const KBufs& B, int tid,
                                            bool active, const int* lt, const int* gt, double dt,
                                            double* out) {
  constexpr bool CROSS = (KIND == 2 && COMP != DIM) || (KIND == 3);
  constexpr int QFIELD = (KIND == 0) ? R3 : (KIND == 1) ? E3 : (KIND == 2) ? M3 + COMP : B3 + COMP;
  constexpr int SD = s3::bstride(DIM);
  // nu area: the tile along DIM, +-1 across when cross terms need it
  constexpr int E0 = s3::T0 + ((CROSS && DIM != 0) ? 2 : 0);
  constexpr int E1 = s3::T1 + ((CROSS && DIM != 1) ? 2 : 0);
  constexpr int E2 = s3::T2 + ((CROSS && DIM != 2) ? 2 : 0);
  constexpr int G0 = s3::H - ((CROSS && DIM != 0) ? 1 : 0);
  constexpr int G1 = s3::H - ((CROSS && DIM != 1) ? 1 : 0);
  constexpr int G2 = s3::H - ((CROSS && DIM != 2) ? 1 : 0);
  constexpr int NAREA = E0 * E1 * E2;
  // ratio area: the nu area extended by one cell below along DIM
  constexpr int RE0 = E0 + (DIM == 0), RE1 = E1 + (DIM == 1), RE2 = E2 + (DIM == 2);
  constexpr int RG0 = G0 - (DIM == 0), RG1 = G1 - (DIM == 1), RG2 = G2 - (DIM == 2);
  constexpr int RAREA = RE0 * RE1 * RE2;
  constexpr int RS = DIM == 0 ? 1 : (DIM == 1 ? RE0 : RE0 * RE1);  // stride along DIM in R
  using HT = typename Form<MIX>::H;
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  const int n[3] = {P.n0, P.n1, P.n2};
  const long nc = P.ncell;
  const HT* Q = static_cast<const HT*>(X.U);
  HT* RR = static_cast<HT*>(X.U) + s3::BC;
  HT* C3 = RR + s3::RA;
  HT* C4 = C3 + s3::NA;
  auto aidx = [&](int lx, int ly, int lz) { return ((lz - G2) * E1 + (ly - G1)) * E0 + (lx - G0); };
  auto ridx = [&](int lx, int ly, int lz) { return ((lz - RG2) * RE1 + (ly - RG1)) * RE0 + (lx - RG0); };

  // (B) nu_r(i) = c(i) R(i), nu_l(i) = c(i) R(i-1) with
  // R(i) = max D3(i-1..i+1) / max D1(i-2..i+2) (hyperdifvisc2-4; the windows
  // of nu_l(i) are those of nu_r(i-1)); 0 where the denominator is 0
  const HT coef = (HT)(B.cmax_in[DIM] * P.chyp[QFIELD]);
  for (int r = tid; r < RAREA; r += s3::NT) {
    const int lx = RG0 + r % RE0, ly = RG1 + (r / RE0) % RE1, lz = RG2 + r / (RE0 * RE1);
    const int q0 = (lz * s3::BY + ly) * s3::BX + lx;
    HT q[6];
#pragma unroll
    for (int s = 0; s < 6; s++) q[s] = Q[q0 + (s - 2) * SD];
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
    for (int r = tid; r < NAREA; r += s3::NT) {
      const int lx = G0 + r % E0, ly = G1 + (r / E0) % E1, lz = G2 + r / (E0 * E1);
      const int g[3] = {X.o[0] + lx, X.o[1] + ly, X.o[2] + lz};
      HT c3 = 0, c4 = 0;
      if (X.inner ||
          (g[0] > 0 && g[0] < n[0] - 1 && g[1] > 0 && g[1] < n[1] - 1 && g[2] > 0 && g[2] < n[2] - 1)) {
        const int q0 = (lz * s3::BY + ly) * s3::BX + lx;
        const int la = DIM == 0 ? lx : (DIM == 1 ? ly : lz);
        // grad13n along DIM of q
        HT gq = ((Q[q0 + SD] - Q[q0 - SD]) * (HT)X.rd[DIM][la]) * (HT)0.5;
        if ((P.bt[DIM] != 0) && zero1n(g[DIM], n[DIM])) gq = 0;
        HT nsum = 0;
        if (X.inner || (g[0] >= 2 && g[0] <= n[0] - 3 && g[1] >= 2 && g[1] <= n[1] - 3 && g[2] >= 2 &&
                        g[2] <= n[2] - 3)) {
          const int rr = ridx(lx, ly, lz);
          const HT cc = (HT)X.dl[DIM][la] * coef;
          nsum = cc * RR[rr] + cc * RR[rr - RS];
        }
        const long c = ((long)g[2] * n[1] + g[1]) * n[0] + g[0];
        if (KIND == 2) {
          const HT tau = (gq * nsum) * (HT)0.25;
          c3 = (HT)((double)__ldg(u + c) + __ldg(B.bg + GRB * nc + c)) * tau;
          c4 = tau * (HT)__ldg(u + (M3 + DIM) * nc + c);
        } else {
          const HT t3 = (gq * nsum) * (HT)0.5;
          c3 = t3;
          c4 = t3 * (HT)__ldg(u + (B3 + DIM) * nc + c);
        }
      }
      C3[r] = c3;
      C4[r] = c4;
    }
    __syncthreads();
  }
  // (D) sources at the tile cells
  if (active) {
    const int la = lt[DIM];
    const int q0 = (lt[2] * s3::BY + lt[1]) * s3::BX + lt[0];
    const int nidx = aidx(lt[0], lt[1], lt[2]);
    const int rr = ridx(lt[0], lt[1], lt[2]);
    const HT cc = (HT)X.dl[DIM][la] * coef;
    const HT nur = cc * RR[rr], nul = cc * RR[rr - RS];
    const HT rdl = (HT)X.rd[DIM][la];
    const HT qc = Q[q0], qp = Q[q0 + SD], qm = Q[q0 - SD];
    HT gr = (qp - qc) * rdl;  // grad1r3n
    HT gl = (qc - qm) * rdl;  // grad1l3n
    if ((P.bt[DIM] != 0) && zero1n(gt[DIM], n[DIM])) { gr = 0; gl = 0; }
    if (KIND == 0) {
      out[R3] = out[R3] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 1) {
      out[E3] = out[E3] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 2) {
      // hyperdifmomsource1-3a (src/hyperdifmomsource1.cu:17-511), ii0 = COMP
      const long c = ((long)gt[2] * n[1] + gt[1]) * n[0] + gt[0];
      const long sd = DIM == 0 ? 1 : (DIM == 1 ? (long)n[0] : (long)n[0] * n[1]);
      const ST* rho = u;
      const double* rb = B.bg + GRB * nc;
      const ST* mf = u + (M3 + COMP) * nc;
      const double r0 = (double)__ldg(rho + c) + __ldg(rb + c);
      const HT t2 = (HT)((r0 + (double)__ldg(rho + c - sd) + __ldg(rb + c - sd)) * 0.5);
      const HT t3 = (HT)((r0 + (double)__ldg(rho + c + sd) + __ldg(rb + c + sd)) * 0.5);
      const double m0 = __ldg(mf + c);
      const HT t5 = (HT)((m0 + (double)__ldg(mf + c - sd)) * 0.5);
      const HT t6 = (HT)((m0 + (double)__ldg(mf + c + sd)) * 0.5);
      const double dm = (double)(((t3 * nur * gr - t2 * nul * gl) * rdl) * (HT)0.5);
      const double de = (double)(((t6 * nur * gr - t5 * nul * gl) * rdl) * (HT)0.5);
      out[M3 + COMP] = out[M3 + COMP] + dt * dm;
      out[E3] = out[E3] + dt * de;
      if (COMP == DIM) {
        out[M3 + COMP] = out[M3 + COMP] + dt * dm;
        out[E3] = out[E3] + dt * de;
      } else {
        // hyperdifmomsourcene5-6a: d/dx_COMP of (rho_t tau) and (tau m_DIM)
        constexpr int FS = COMP == 0 ? 1 : (COMP == 1 ? E0 : E0 * E1);
        const HT rdf = (HT)X.rd[COMP][lt[COMP]];
        HT g7 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
        HT g8 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
        if ((P.bt[COMP] != 0) && zero1n(gt[COMP], n[COMP])) { g7 = 0; g8 = 0; }
        out[M3 + DIM] = out[M3 + DIM] + dt * (double)g7;
        out[E3] = out[E3] + dt * (double)g8;
      }
    } else {
      // B component COMP diffused along DIM: hyperdifbsourcene (sb=-1) then
      // hyperdifbsource (sb=+1)
      constexpr int FS = COMP == 0 ? 1 : (COMP == 1 ? E0 : E0 * E1);
      const HT rdf = (HT)X.rd[COMP][lt[COMP]];
      HT g4 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
      HT g6 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
      if ((P.bt[COMP] != 0) && zero1n(gt[COMP], n[COMP])) { g4 = 0; g6 = 0; }
      out[B3 + DIM] = out[B3 + DIM] - dt * (double)g4;
      out[E3] = out[E3] - dt * (double)g6;
      const HT t2 = (qc + qm) * (HT)0.5, t3 = (qc + qp) * (HT)0.5;
      const double dB = (double)((gr * nur - gl * nul) * rdl);
      const double de = (double)((t3 * gr * nur - t2 * gl * nul) * rdl);
      out[B3 + COMP] = out[B3 + COMP] + dt * dB;
      out[E3] = out[E3] + dt * de;
    }
  }
  __syncthreads();
}

// fluxes along D at one cell: rho, m0..2, e, and the two B components across
// D (in increasing order); velocities for the background energy terms
template <bool BG, int D>
__device__ __forceinline__ void flux3(const double* s, const double* g, double r, double gamma,
                                      double* F, double* v) {
  const double m[3] = {s[1], s[2], s[3]};
  const double b[3] = {s[5], s[6], s[7]};
  const double bb[3] = {BG ? g[2] : 0.0, BG ? g[3] : 0.0, BG ? g[4] : 0.0};
  const double e = s[4], eb = BG ? g[0] : 0.0;
  const double md = m[D], vd = md * r;
  // computept3 (src/dervfields.cu:107-153)
  const double pt = (gamma - 1.0) * (e - 0.5 * (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) * r) -
                    (gamma - 2.0) * ((b[0] * bb[0] + b[1] * bb[1] + b[2] * bb[2]) +
                                     0.5 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]));
  const double bd = b[D], bbd = bb[D];
  F[0] = md;
#pragma unroll
  for (int c = 0; c < 3; c++) F[1 + c] = vd * m[c] + (c == D ? pt : 0.0) - (b[c] * bbd + bb[c] * bd) - b[c] * bd;
  const double bbm = bb[0] * m[0] + bb[1] * m[1] + bb[2] * m[2];
  const double bm = b[0] * m[0] + b[1] * m[1] + b[2] * m[2];
  F[4] = vd * (e + pt + eb) - (bd * bbm + bbd * bm + bd * bm) * r;
  constexpr int c1 = D == 0 ? 1 : 0, c2 = D == 2 ? 1 : 2;
  F[5] = vd * (b[c1] + bb[c1]) - (m[c1] * r) * (bd + bbd);
  F[6] = vd * (b[c2] + bb[c2]) - (m[c2] * r) * (bd + bbd);
  v[0] = m[0] * r;
  v[1] = m[1] * r;
  v[2] = m[2] * r;
}

// flux phase along D: fluxes on the tile +-2 along D (+-3 for the 6th-order
// derivative), divergence and the background energy terms at the tile cells
template <bool BG, bool MIX, int D, bool O6>
__device__ __forceinline__ void flux_pass3(const Box3& X, const KParams& P, const KBufs& B, int tid,
                                           bool active, const int* lt, const int* gt, double dt,
                                           const double* gc, double* out) {
  constexpr int FH = O6 ? 3 : 2, FA = s3::fa<O6>();
  constexpr int E0 = s3::T0 + (D == 0 ? 2 * FH : 0), E1 = s3::T1 + (D == 1 ? 2 * FH : 0);
  constexpr int E2 = s3::T2 + (D == 2 ? 2 * FH : 0);
  constexpr int G0 = s3::H - (D == 0 ? FH : 0), G1 = s3::H - (D == 1 ? FH : 0), G2 = s3::H - (D == 2 ? FH : 0);
  constexpr int NAREA = E0 * E1 * E2;
  constexpr int FS = D == 0 ? 1 : (D == 1 ? E0 : E0 * E1);
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  const int n[3] = {P.n0, P.n1, P.n2};
  const long nc = P.ncell;
  double* F = static_cast<double*>(X.U);
  for (int r = tid; r < NAREA; r += s3::NT) {
    const int lx = G0 + r % E0, ly = G1 + (r / E0) % E1, lz = G2 + r / (E0 * E1);
    const int g0 = X.o[0] + lx, g1 = X.o[1] + ly, g2 = X.o[2] + lz;
    double f[7] = {0, 0, 0, 0, 0, 0, 0}, v[3] = {0, 0, 0};
    if (X.inner || (g0 >= 0 && g0 < n[0] && g1 >= 0 && g1 < n[1] && g2 >= 0 && g2 < n[2])) {
      const long c = ((long)g2 * n[1] + g1) * n[0] + g0;
      double s[8], g[5] = {0, 0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < 8; k++) s[k] = __ldg(u + k * nc + c);
      if (BG) {
#pragma unroll
        for (int k = 0; k < 5; k++) g[k] = __ldg(B.bg + k * nc + c);
      }
      flux3<BG, D>(s, g, X.R[(lz * s3::BY + ly) * s3::BX + lx], P.gamma, f, v);
    }
#pragma unroll
    for (int k = 0; k < 7; k++) F[k * FA + r] = f[k];
    if (BG) {
#pragma unroll
      for (int k = 0; k < 3; k++) F[(7 + k) * FA + r] = v[k];
    }
  }
  __syncthreads();
  if (active) {
    const bool z = ((P.bt[D] != 0) && zero3dn(gt[D], n[D])) || (O6 && edge6(gt[D], n[D]));
    const double rdl2 = 0.5 * X.rd[D][lt[D]];
    const int fo = ((lt[2] - G2) * E1 + (lt[1] - G1)) * E0 + (lt[0] - G0);
    constexpr int c1 = D == 0 ? 1 : 0, c2 = D == 2 ? 1 : 2;
    const int fld[7] = {R3, M3, M3 + 1, M3 + 2, E3, B3 + c1, B3 + c2};
#pragma unroll
    for (int k = 0; k < 7; k++) {
      double gk = dflux<O6>(F + k * FA, fo, FS, rdl2);
      if (z) gk = 0;
      out[fld[k]] = out[fld[k]] - dt * gk;
    }
    if (BG) {
      // addenergyterms_cd2 (src/centdiff2.cu:80-115): -p_tb dv_D/dx_D, and
      // the derivative-along-D part of sum_i Bb_i Bb_d dv_d/dx_i
      const double bb[3] = {gc[2], gc[3], gc[4]};
      const double ptb = (P.gamma - 1) * gc[0] - 0.5 * (P.gamma - 2) * (bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
      double gv = dflux<O6>(F + (7 + D) * FA, fo, FS, rdl2);
      if (z) gv = 0;
      out[E3] -= dt * ptb * gv;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double gk = dflux<O6>(F + (7 + k) * FA, fo, FS, rdl2);
        if (z) gk = 0;
        out[E3] += dt * bb[D] * bb[k] * gk;
      }
    }
  }
  __syncthreads();
}

template <int MODE, bool BG, bool MIX, bool O6>
__global__ void __launch_bounds__(s3::NT, SMAUG_MINB3D) stage3d_fast(const KParams P, const KBufs B) {
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  extern __shared__ double smem[];
  Box3 X;
  X.R = smem;
  X.dl[0] = smem + s3::BC;
  X.dl[1] = X.dl[0] + s3::BX;
  X.dl[2] = X.dl[1] + s3::BY;
  X.rd[0] = X.dl[2] + s3::BZ;
  X.rd[1] = X.rd[0] + s3::BX;
  X.rd[2] = X.rd[1] + s3::BY;
  X.U = X.rd[2] + s3::BZ;
  X.C = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(X.U) + s3::union_bytes<MIX, O6>());
  const int tid = threadIdx.x;
  const int tx = tid % s3::T0, ty = (tid / s3::T0) % s3::T1, tz = tid / (s3::T0 * s3::T1);
  const int n[3] = {P.n0, P.n1, P.n2};
  const long nc = P.ncell;
  X.o[0] = 2 + blockIdx.x * s3::T0 - s3::H;
  X.o[1] = 2 + blockIdx.y * s3::T1 - s3::H;
  X.o[2] = 2 + blockIdx.z * s3::T2 - s3::H;
  // box indices 0 .. B-1 of every axis inside [0, n-1]: no bounds or pad
  // checks in the staging, flux and cross-term loops
  X.inner = X.o[0] >= 0 && X.o[1] >= 0 && X.o[2] >= 0 && X.o[0] + s3::BX <= n[0] &&
            X.o[1] + s3::BY <= n[1] && X.o[2] + s3::BZ <= n[2];

  // ---- 1/rho_t on the box and the per-axis metric ----------------------
  for (int r = tid; r < s3::BC; r += s3::NT) {
    const int lx = r % s3::BX, ly = (r / s3::BX) % s3::BY, lz = r / s3::BS2;
    const int g0 = X.o[0] + lx, g1 = X.o[1] + ly, g2 = X.o[2] + lz;
    double rinv = 1.0;
    if (X.inner || (g0 >= 0 && g0 < n[0] && g1 >= 0 && g1 < n[1] && g2 >= 0 && g2 < n[2])) {
      const long c = ((long)g2 * n[1] + g1) * n[0] + g0;
      rinv = 1.0 / ((double)__ldg(u + c) + __ldg(B.bg + GRB * nc + c));
    }
    X.R[r] = rinv;
    X.C[r] = box_code(X, P, B, lx, ly, lz);
  }
  for (int r = tid; r < s3::BX + s3::BY + s3::BZ; r += s3::NT) {
    const int a = r < s3::BX ? 0 : (r < s3::BX + s3::BY ? 1 : 2);
    const int l = r - (a == 0 ? 0 : (a == 1 ? s3::BX : s3::BX + s3::BY));
    const int g = X.o[a] + l;
    const double d = (g >= 0 && g < n[a]) ? B.delx[a][g] : 1.0;
    X.dl[a][l] = d;
    X.rd[a][l] = 1.0 / d;
  }

  // ---- dt of this step and stage time ----------------------------------
  double dt, tstage;
  const bool first = blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && tid == 0;
  if (B.stage == 0) {
    dt = device_dt(P, B.cmax_in, *B.dt_prev, 3);
    if (first) {
      *B.dt_new = dt;
      *B.t_new = *B.t_prev + dt;
      B.cmax_clear[0] = B.cmax_clear[1] = B.cmax_clear[2] = 0ull;
    }
    tstage = *B.t_prev;
  } else {
    dt = *B.dt_new;
    tstage = *B.t_prev + (B.stage == 3 ? dt : 0.5 * dt);
    if (first) B.cmax_clear[0] = B.cmax_clear[1] = B.cmax_clear[2] = 0ull;
  }
  __syncthreads();

  const int lt[3] = {tx + s3::H, ty + s3::H, tz + s3::H};
  const int gt[3] = {X.o[0] + lt[0], X.o[1] + lt[1], X.o[2] + lt[2]};
  const bool active = gt[0] <= n[0] - 3 && gt[1] <= n[1] - 3 && gt[2] <= n[2] - 3;
  const long co = active ? ((long)gt[2] * n[1] + gt[1]) * n[0] + gt[0] : 0;

  double sc[8], gc[5] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int f = 0; f < 8; f++) sc[f] = active ? (double)__ldg(u + f * nc + co) : 0.0;
#pragma unroll
  for (int f = 0; f < 5; f++) gc[f] = active ? __ldg(B.bg + f * nc + co) : 0.0;
  double out[8];
#pragma unroll
  for (int f = 0; f < 8; f++) {
    if (MODE != SMAUG_INT_EULER)
      out[f] = 0.0;
    else if (MIX)
      out[f] = active ? base_value<MIX>(B, f * nc + co) : 0.0;
    else
      out[f] = sc[f];
  }

  // ---- fluxes and divergence, direction 0, 1, 2 ----------------------------
  flux_pass3<BG, MIX, 0, O6>(X, P, B, tid, active, lt, gt, dt, gc, out);
  flux_pass3<BG, MIX, 1, O6>(X, P, B, tid, active, lt, gt, dt, gc, out);
  flux_pass3<BG, MIX, 2, O6>(X, P, B, tid, active, lt, gt, dt, gc, out);

  // ---- gravity (addgrav_cd2, src/centdiff2.cu:118-154) --------------------
  if (P.has_grav && active) {
    const double rho = sc[R3];
    out[M3 + 0] += dt * P.g[0] * rho;
    out[M3 + 1] += dt * P.g[1] * rho;
    out[M3 + 2] += dt * P.g[2] * rho;
    const double rr = rho * X.R[(lt[2] * s3::BY + lt[1]) * s3::BX + lt[0]];
    out[E3] += (dt * P.g[0] * sc[M3 + 0]) * rr;
    out[E3] += (dt * P.g[1] * sc[M3 + 1]) * rr;
    out[E3] += (dt * P.g[2] * sc[M3 + 2]) * rr;
  }

  // ---- hyperdiffusion: one q staging per field, then every direction ----
  if (P.hyperdif == 1) {
#define HP(K, C, D) hyper_pass3<MIX, K, C, D>(X, P, B, tid, active, lt, gt, dt, out)
#define SQ(K, C) stage_q<MIX, K, C>(X, P, B, tid)
    SQ(0, 0);
    HP(0, 0, 0); HP(0, 0, 1); HP(0, 0, 2);
    SQ(1, 0);
    HP(1, 0, 0); HP(1, 0, 1); HP(1, 0, 2);
    SQ(2, 0);
    HP(2, 0, 0); HP(2, 0, 1); HP(2, 0, 2);
    SQ(2, 1);
    HP(2, 1, 0); HP(2, 1, 1); HP(2, 1, 2);
    SQ(2, 2);
    HP(2, 2, 0); HP(2, 2, 1); HP(2, 2, 2);
    SQ(3, 0);
    HP(3, 0, 1); HP(3, 0, 2);
    SQ(3, 1);
    HP(3, 1, 0); HP(3, 1, 2);
    SQ(3, 2);
    HP(3, 2, 0); HP(3, 2, 1);
#undef SQ
#undef HP
  }

  // ---- user driver (source_parallel + addsourceterms2) ---------------------
  if (P.driver == SMAUG_DRIVER_GAUSS && active) {
    double v = P.drv_amp;
    if (P.drv_period > 0) v *= sin(tstage * 2.0 * M_PI / P.drv_period);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (P.drv_sigma[a] > 0) {
        const double x = B.pos[a][gt[a]] - P.drv_x0[a];
        v *= exp(-x * x / (P.drv_sigma[a] * P.drv_sigma[a]));
      }
    }
    const double rr = (MODE == SMAUG_INT_EULER) ? out[R3] : sc[R3];
    out[M3] = out[M3] + dt * v * (rr + gc[GRB]);
  }

  // ---- combine, write, ghost images, CFL maxima -----------------------------
  double cm[3] = {P.cmax_floor[0], P.cmax_floor[1], P.cmax_floor[2]};
  if (active) {
    double res[8];
    const bool is_base = (MODE == SMAUG_INT_EULER) || B.stage == 3;
    if (MODE == SMAUG_INT_EULER) {
#pragma unroll
      for (int f = 0; f < 8; f++) res[f] = out[f];
    } else {
      const double wgt = (B.stage == 0 || B.stage == 3) ? 1.0 / 6.0 : 1.0 / 3.0;
      const double cst = (B.stage == 2) ? 1.0 : 0.5;
#pragma unroll
      for (int f = 0; f < 8; f++) {
        const double dl = out[f];
        if (B.stage == 0) {
          const double u0 = MIX ? base_value<MIX>(B, f * nc + co) : sc[f];
          B.acc[f * nc + co] = u0 + wgt * dl;
          res[f] = u0 + cst * dl;
        } else if (B.stage < 3) {
          B.acc[f * nc + co] = B.acc[f * nc + co] + wgt * dl;
          res[f] = base_value<MIX>(B, f * nc + co) + cst * dl;
        } else {
          res[f] = B.acc[f * nc + co] + wgt * dl;
        }
      }
    }
    bool bad = false;
#pragma unroll
    for (int f = 0; f < 8; f++) bad |= !isfinite(res[f]);
    if (bad) atomicOr(B.flags, 1);
    int ix[3], iy[3], iz[3];
    ix[0] = gt[0];
    iy[0] = gt[1];
    iz[0] = gt[2];
    const int nx = 1 + ghost_images(gt[0], n[0], P.bc[0], ix + 1);
    const int ny = 1 + ghost_images(gt[1], n[1], P.bc[1], iy + 1);
    const int nz = 1 + ghost_images(gt[2], n[2], P.bc[2], iz + 1);
    bool negated = false;  // res holds the negated values
    for (int cz = 0; cz < nz; cz++)
      for (int b = 0; b < ny; b++)
        for (int a2 = 0; a2 < nx; a2++) {
          const long cc = ((long)iz[cz] * n[1] + iy[b]) * n[0] + ix[a2];
          // antisymmetric images carry the opposite sign (negation is exact)
          const bool neg = (((a2 > 0) && P.gneg[0]) != ((b > 0) && P.gneg[1])) != ((cz > 0) && P.gneg[2]);
          if (neg != negated) {
#pragma unroll
            for (int f = 0; f < 8; f++) res[f] = -res[f];
            negated = neg;
          }
          const double* r = res;
#pragma unroll
          for (int f = 0; f < 8; f++) store_value<MIX>(B, f * nc + cc, r[f], is_base);
          double gg[5];
          if (a2 == 0 && b == 0 && cz == 0) {
#pragma unroll
            for (int f = 0; f < 5; f++) gg[f] = gc[f];
          } else {
#pragma unroll
            for (int f = 0; f < 5; f++) gg[f] = __ldg(B.bg + f * nc + cc);
          }
          double cv[3];
          cfast3_all(P.gamma, r, gg, cv);
#pragma unroll
          for (int d = 0; d < 3; d++) cm[d] = dmax0(cm[d], cv[d]);
        }
  }
  __shared__ double red[s3::NT / 32][3];
#pragma unroll
  for (int d = 0; d < 3; d++)
    for (int o = 16; o > 0; o >>= 1) cm[d] = dmax0(cm[d], __shfl_xor_sync(0xffffffffu, cm[d], o));
  if ((tid & 31) == 0) {
    red[tid >> 5][0] = cm[0];
    red[tid >> 5][1] = cm[1];
    red[tid >> 5][2] = cm[2];
  }
  __syncthreads();
  if (tid < 3) {
    double v = 0.0;
    for (int w = 0; w < s3::NT / 32; w++) v = dmax0(v, red[w][tid]);
    atomicMax(&B.cmax_out[tid], (unsigned long long)__double_as_longlong(v));
  }
}

template <int MODE, bool MIX, bool O6>
static cudaError_t launch_stage3d_o(const KParams& K, const KBufs& B, cudaStream_t st) {
  dim3 grid((K.n0 - 4 + s3::T0 - 1) / s3::T0, (K.n1 - 4 + s3::T1 - 1) / s3::T1,
            (K.n2 - 4 + s3::T2 - 1) / s3::T2);
  if (K.has_bg)
    stage3d_fast<MODE, true, MIX, O6><<<grid, s3::NT, s3::smem_bytes<MIX, O6>(), st>>>(K, B);
  else
    stage3d_fast<MODE, false, MIX, O6><<<grid, s3::NT, s3::smem_bytes<MIX, O6>(), st>>>(K, B);
  return cudaGetLastError();
}
template <int MODE, bool MIX>
static cudaError_t launch_stage3d(const KParams& K, const KBufs& B, cudaStream_t st) {
  return K.order6 ? launch_stage3d_o<MODE, MIX, true>(K, B, st) : launch_stage3d_o<MODE, MIX, false>(K, B, st);
}

template <int MODE, bool BG, bool MIX, bool O6>
static cudaError_t stage3d_attr() {
  return cudaFuncSetAttribute(stage3d_fast<MODE, BG, MIX, O6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)s3::smem_bytes<MIX, O6>());
}
