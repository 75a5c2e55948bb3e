// stage3d_zm.cuh -- z-marching 3D stage kernel, included by the
// stage3d_zm_*.cu translation units (one per integrator and precision form).
//
// The operator is the one of the reference's 3D build (-DUSE_SAC_3D,
// src/iosmaug.c:631-835): fluxes along the three dimensions with their
// 4th-order (or USE_DORDER3 6th-order) divergence (src/centdiff1.cu:51-197,
// src/centdiff2.cu:203-323, grad3dn), the background energy coupling
// (src/centdiff2.cu:80-115), gravity (src/centdiff2.cu:118-154), the 21
// hyperdiffusion passes of rho, e, m_c, B_c (src/hyperdifvisc1{r,l}.cu,
// src/hyperdif*source*.cu), the user driver, the stage combine, the ghost
// images and the CFL maxima.  Sums per cell are reordered against the
// reference (per direction and field); agreement stays at rounding level.
//
// Structure.  A block owns a 16 x 8 column of cells (x fastest) and marches
// along z through a chunk of planes, producing one output plane per
// iteration.  Everything along x and y is plane-local, as in the 2D kernel:
// the state of the plane on the tile + 3-cell halo sits in shared memory, and
// the fluxes along x and y, the hyperdiffusion ratios along x and y and their
// cross terms are computed there.  Everything along z comes from rings that
// every plane enters once:
//   - z-fluxes (7 fluxes and, with background fields, 3 velocities) of the
//     planes k-FH .. k+FH of every tile column, for the z-divergence;
//   - q of the seven fields diffused along z, planes k-2 .. k+3, on the tile
//     columns (rho, e, m_z) or on the tile + 1 columns (m_x, m_y, B_x, B_y,
//     whose z-passes have cross terms along x or y); the ratio
//     R = max D3 / max D1 of a cell is computed once per plane and kept for
//     the next plane's nu_l;
//   - the cross terms of m_z and B_z diffused along x and y (their derivative
//     is along z): computed one plane ahead, on the look-ahead plane k+1
//     whose state is already staged, and kept per thread for the planes
//     k-1 .. k+1; the same look-ahead adds the diagonal parts of those four
//     passes to the next plane's accumulators.
// Shared memory (FP64, background fields, 4th order) holds the state of
// planes k and k+1 on the region, the q ring, the ratio planes, the flux ring
// and one union of plane-local scratch -- about 200 KB, one block of 256
// threads per SM; threads 0-127 own a column each, all 256 share the
// plane-local loops and the ring updates.
#pragma once

// (included inside namespace smaug)
namespace zm {
constexpr int TX = 16, TY = 8;          // tile (x fastest)
constexpr int NCOL = TX * TY;           // columns, one owner thread each
constexpr int NT = 2 * NCOL;            // threads per block
constexpr int H = 3;                    // region halo
constexpr int RX = TX + 2 * H, RY = TY + 2 * H, RC = RX * RY;  // 22 x 14 region
constexpr int HX = TX + 2, HY = TY + 2, HC = HX * HY;          // tile + 1 columns
constexpr int NQP = 6;                  // q ring planes k-2 .. k+3
constexpr int NQT = 3, NQH = 4;         // z fields on tile columns / on tile + 1 columns
__host__ __device__ constexpr int cmax2(int a, int b) { return a > b ? a : b; }
constexpr int RSZ = cmax2((TX + 1) * (TY + 2), (TX + 2) * (TY + 1));  // ratio area
constexpr int NSZ = cmax2(TX * (TY + 2), (TX + 2) * TY);              // cross-term area
template <bool O6>
__host__ __device__ constexpr int fh() { return O6 ? 3 : 2; }
template <bool O6>
__host__ __device__ constexpr int nf() { return 2 * fh<O6>() + 1; }
template <bool BG>
__host__ __device__ constexpr int nfq() { return BG ? 10 : 7; }
template <bool O6>
__host__ __device__ constexpr int fsz() {
  return cmax2((TX + 2 * fh<O6>()) * TY, TX * (TY + 2 * fh<O6>()));
}
__host__ __device__ constexpr size_t al16(size_t b) { return (b + 15) / 16 * 16; }

// byte offsets of the shared-memory arrays
template <bool BG, bool MIX, bool O6>
struct Lay {
  using ST = typename Form<MIX>::S;
  using HT = typename Form<MIX>::H;
  static constexpr size_t S = 0;                                        // [2][8][RC] ST
  static constexpr size_t RB = al16(S + 2 * 8 * RC * sizeof(ST));       // [2][RC] rho_b
  static constexpr size_t RI = al16(RB + 2 * RC * sizeof(double));      // [2][RC] 1/rho_t
  static constexpr size_t GB = al16(RI + 2 * RC * sizeof(double));      // [2][4][RC] eb, bb
  static constexpr size_t QH = al16(GB + (BG ? 2 * 4 * RC : 0) * sizeof(double));  // [NQP][4][HC]
  static constexpr size_t QT = al16(QH + NQP * NQH * HC * sizeof(HT));  // [NQP][3][NCOL]
  // [2][4][HC] ratios of the tile + 1 fields, then [2][3][NCOL] of the tile fields
  static constexpr size_t RZ = al16(QT + NQP * NQT * NCOL * sizeof(HT));
  static constexpr size_t FR = al16(RZ + (2 * NQH * HC + 2 * NQT * NCOL) * sizeof(HT));  // [NF][NFQ][NCOL]
  static constexpr size_t U = al16(FR + nf<O6>() * nfq<BG>() * NCOL * sizeof(double));
  static constexpr size_t UB = cmax2((int)(nfq<BG>() * fsz<O6>() * sizeof(double)),
                                     (int)((RC + RSZ + 2 * NSZ) * sizeof(HT)));
  static constexpr size_t MET = al16(U + UB);                            // dl0 rd0 [RX], dl1 rd1 [RY]
  static constexpr size_t TOTAL = al16(MET + 2 * (RX + RY) * sizeof(double));
  static_assert(TOTAL + 256 <= 232448, "shared memory of the z-marching kernel exceeds 227 KB");
};
}  // namespace zm

template <bool BG, bool MIX>
struct ZS {
  using ST = typename Form<MIX>::S;
  using HT = typename Form<MIX>::H;
  ST* S;       // [2][8][RC] evolved fields of the staged planes (buffer = plane & 1)
  double* RB;  // [2][RC]
  double* RI;  // [2][RC]
  double* GB;  // [2][4][RC] (BG only)
  HT* QH;      // q ring, tile + 1 columns: m_x, m_y, B_x, B_y
  HT* QT;      // q ring, tile columns: rho, e, m_z
  HT* RZ;      // ratios along z: tile + 1 fields [2][4][HC], tile fields [2][3][NCOL]
  double* FR;  // flux ring
  void* U;     // plane-local scratch
  double *dl0, *rd0, *dl1, *rd1;
  int x0, y0;  // grid coordinates of the first tile cell
  bool inner;  // the region lies inside the grid and off its pads
  __device__ __forceinline__ double v(int buf, int f, int l) const {  // evolved field f in double
    return (double)S[(buf * 8 + f) * zm::RC + l];
  }
};

__device__ __forceinline__ int zm_slot(int j) { return (j + zm::NQP) % zm::NQP; }

// q of a hyperdiffusion field from global memory (a stray pad's source cell;
// src/hyperdifvisc1r.cu:1225-1253)
template <typename ST, int KIND, int COMP>
__device__ __forceinline__ double zm_hq_global(const ST* u, const KBufs& B, long nc, long c) {
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

// ---- staging of one plane of the region -----------------------------------
template <bool BG, bool MIX>
__device__ __forceinline__ void zm_load_region(const ZS<BG, MIX>& Z, const KParams& P, const KBufs& B,
                                               int plane, int tid) {
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  const long nc = P.ncell;
  const long pofs = (long)plane * P.n1 * P.n0;
  const int buf = plane & 1;
  ST* S = Z.S + buf * 8 * zm::RC;
  for (int r = tid; r < zm::RC; r += zm::NT) {
    const int lx = r % zm::RX, ly = r / zm::RX;
    const int gi = Z.x0 - zm::H + lx, gj = Z.y0 - zm::H + ly;
    const bool in = Z.inner || (gi >= 0 && gi < P.n0 && gj >= 0 && gj < P.n1);
    const long c = pofs + (long)gj * P.n0 + gi;
    double rho = 0.0;
#pragma unroll
    for (int f = 0; f < 8; f++) {
      const ST v = in ? __ldg(u + f * nc + c) : (ST)0;
      S[f * zm::RC + r] = v;
      if (f == 0) rho = (double)v;
    }
    const double rhob = in ? __ldg(B.bg + GRB * nc + c) : 1.0;
    Z.RB[buf * zm::RC + r] = rhob;
    Z.RI[buf * zm::RC + r] = 1.0 / (rho + rhob);
    if (BG) {
      const int gf[4] = {GEB, GBB, GBB + 1, GBB + 2};
#pragma unroll
      for (int a = 0; a < 4; a++) Z.GB[(buf * 4 + a) * zm::RC + r] = in ? __ldg(B.bg + gf[a] * nc + c) : 0.0;
    }
  }
}

// q of a hyperdiffusion field at region cell l of buffer buf
template <bool BG, bool MIX, int KIND, int COMP>
__device__ __forceinline__ double zm_hq(const ZS<BG, MIX>& Z, int buf, int l) {
  if (KIND == 0) return Z.v(buf, R3, l);
  if (KIND == 3) return Z.v(buf, B3 + COMP, l);
  const double ri = Z.RI[buf * zm::RC + l];
  if (KIND == 2) return Z.v(buf, M3 + COMP, l) * ri;
  double m2 = 0, b2 = 0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double m = Z.v(buf, M3 + a, l), b = Z.v(buf, B3 + a, l);
    m2 += m * m;
    b2 += b * b;
  }
  return Z.v(buf, E3, l) - 0.5 * (b2 + m2 * ri);
}

// q of one field on the region of plane `plane` (buffer plane & 1), with the
// reference's pads along x and y: index -1 holds the copy of index 5
// (bc_hyperdifl), index n the stray tmp6 store (source table B.padsrc)
template <bool BG, bool MIX, int KIND, int COMP>
__device__ __forceinline__ void zm_stage_q(const ZS<BG, MIX>& Z, const KParams& P, const KBufs& B,
                                           int plane, int tid) {
  using HT = typename Form<MIX>::H;
  using ST = typename Form<MIX>::S;
  HT* Q = static_cast<HT*>(Z.U);
  const int buf = plane & 1;
  if (Z.inner) {
    for (int r = tid; r < zm::RC; r += zm::NT) Q[r] = (HT)zm_hq<BG, MIX, KIND, COMP>(Z, buf, r);
    __syncthreads();
    return;
  }
  const int n0 = P.n0, n1 = P.n1;
  const long nc = P.ncell;
  for (int r = tid; r < zm::RC; r += zm::NT) {
    const int lx = r % zm::RX, ly = r / zm::RX;
    const int ci = Z.x0 - zm::H + lx, cj = Z.y0 - zm::H + ly;
    const bool inx = ci >= 0 && ci < n0, iny = cj >= 0 && cj < n1;
    double q = 0.0;
    if (inx && iny) {
      q = zm_hq<BG, MIX, KIND, COMP>(Z, buf, r);
    } else if (iny) {
      if (ci == -1) {
        q = zm_hq<BG, MIX, KIND, COMP>(Z, buf, r + 6);
      } else if (ci == n0) {
        const int src = B.padsrc[0][(long)plane * n1 + cj];
        if (src >= 0) q = zm_hq_global<ST, KIND, COMP>(static_cast<const ST*>(B.uin), B, nc, src);
      }
    } else if (inx) {
      if (cj == -1) {
        q = zm_hq<BG, MIX, KIND, COMP>(Z, buf, r + 6 * zm::RX);
      } else if (cj == n1) {
        const int src = B.padsrc[1][(long)plane * n0 + ci];
        if (src >= 0) q = zm_hq_global<ST, KIND, COMP>(static_cast<const ST*>(B.uin), B, nc, src);
      }
    }
    Q[r] = (HT)q;
  }
  __syncthreads();
}

// ---- rings -------------------------------------------------------------------
// q of the seven z-diffused fields at plane j on the tile + 1 columns (the
// tile columns only for rho, e, m_z); plane -1 is the copy of plane 5
// (bc_hyperdifl), plane n2 the stray tmp6 store (B.padsrc[2])
template <bool BG, bool MIX>
__device__ __forceinline__ void zm_ring_q(const ZS<BG, MIX>& Z, const KParams& P, const KBufs& B, int j,
                                          int i0, int stride) {
  using ST = typename Form<MIX>::S;
  using HT = typename Form<MIX>::H;
  const ST* u = static_cast<const ST*>(B.uin);
  const long nc = P.ncell;
  const int n0 = P.n0, n1 = P.n1, n2 = P.n2;
  const int s = zm_slot(j);
  for (int i = i0; i < zm::HC; i += stride) {
    const int hx = i % zm::HX, hy = i / zm::HX;
    const int ci = Z.x0 - 1 + hx, cj = Z.y0 - 1 + hy;
    long c = -1;
    if (ci < n0 && cj < n1) {  // ci, cj >= 1 always
      if (j == -1)
        c = ((long)5 * n1 + cj) * n0 + ci;
      else if (j == n2)
        c = B.padsrc[2][(long)cj * n0 + ci];
      else
        c = ((long)j * n1 + cj) * n0 + ci;
    }
    double qr = 0, qe = 0, qm[3] = {0, 0, 0}, qb[3] = {0, 0, 0};
    if (c >= 0) {
      const double rho = (double)__ldg(u + c);
      const double r = 1.0 / (rho + __ldg(B.bg + GRB * nc + c));
      double m2 = 0, b2 = 0;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const double m = __ldg(u + (M3 + a) * nc + c), b = __ldg(u + (B3 + a) * nc + c);
        m2 += m * m;
        b2 += b * b;
        qm[a] = m * r;
        qb[a] = b;
      }
      qr = rho;
      qe = (double)__ldg(u + E3 * nc + c) - 0.5 * (b2 + m2 * r);
    }
    HT* qh = Z.QH + s * zm::NQH * zm::HC;
    qh[0 * zm::HC + i] = (HT)qm[0];
    qh[1 * zm::HC + i] = (HT)qm[1];
    qh[2 * zm::HC + i] = (HT)qb[0];
    qh[3 * zm::HC + i] = (HT)qb[1];
    if (hx >= 1 && hx <= zm::TX && hy >= 1 && hy <= zm::TY) {
      const int col = (hy - 1) * zm::TX + (hx - 1);
      HT* qt = Z.QT + s * zm::NQT * zm::NCOL;
      qt[0 * zm::NCOL + col] = (HT)qr;
      qt[1 * zm::NCOL + col] = (HT)qe;
      qt[2 * zm::NCOL + col] = (HT)qm[2];
    }
  }
}

// fluxes along D at one cell: rho, m0..2, e, and the two B components across
// D (in increasing order); velocities for the background energy terms
template <bool BG, int D>
__device__ __forceinline__ void zm_flux(const double* s, const double* g, double r, double gamma,
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

// z-fluxes of plane j at the column of grid cell (gi, gj) into the flux ring
template <bool BG, bool MIX, bool O6>
__device__ __forceinline__ void zm_ring_flux(const ZS<BG, MIX>& Z, const KParams& P, const KBufs& B, int j,
                                             int col, int gi, int gj) {
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  const long nc = P.ncell;
  double F[7] = {0, 0, 0, 0, 0, 0, 0}, v[3] = {0, 0, 0};
  if (j >= 0 && j < P.n2) {
    const long c = ((long)j * P.n1 + gj) * P.n0 + gi;
    double s[8], g[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 8; k++) s[k] = (double)__ldg(u + k * nc + c);
    const double rhob = __ldg(B.bg + GRB * nc + c);
    if (BG) {
#pragma unroll
      for (int k = 0; k < 5; k++) g[k] = __ldg(B.bg + k * nc + c);
    }
    zm_flux<BG, 2>(s, g, 1.0 / (s[0] + rhob), P.gamma, F, v);
  }
  double* fr = Z.FR + ((j + zm::nf<O6>()) % zm::nf<O6>()) * zm::nfq<BG>() * zm::NCOL;
#pragma unroll
  for (int q = 0; q < 7; q++) fr[q * zm::NCOL + col] = F[q];
  if (BG) {
#pragma unroll
    for (int q = 0; q < 3; q++) fr[(7 + q) * zm::NCOL + col] = v[q];
  }
}

// ratio R = max D3 / max D1 along z at plane k from the q ring (q(k-2..k+3))
template <typename HT>
__device__ __forceinline__ HT zm_ratio(const HT* ring, int k, int stride_slot, int idx) {
  HT q[6];
#pragma unroll
  for (int s = 0; s < 6; s++) q[s] = ring[zm_slot(k - 2 + s) * stride_slot + idx];
  HT t4 = 0, t5 = 0;
#pragma unroll
  for (int a = 0; a < 3; a++) t4 = hmax0(t4, (HT)fabs((HT)3 * (q[a + 2] - q[a + 1]) - (q[a + 3] - q[a])));
#pragma unroll
  for (int a = 0; a < 5; a++) t5 = hmax0(t5, (HT)fabs(q[a + 1] - q[a]));
  return (t5 > 0) ? hdiv(t4, t5) : (HT)0;
}

// ---- hyperdiffusion along x or y on a staged plane ----------------------------
// One pass of field kind KIND (0 rho, 1 e, 2 m, 3 B), component COMP, along
// DIM in {0, 1} on plane `plane` (q staged by zm_stage_q).  Cross terms whose
// derivative is along x or y (COMP in {0, 1}) are completed here; for COMP = 2
// the cross quantities of the thread's own cell are returned in z3, z4 (their
// z-derivative is taken by the planes above and below).  Contributions go to
// acc (the plane's accumulators).
template <bool BG, bool MIX, int KIND, int COMP, int DIM>
__device__ __forceinline__ void zm_xy_pass(const ZS<BG, MIX>& Z, const KParams& P, const KBufs& B, int tid,
                                           int plane, bool own, int lxo, int lyo, int gi, int gj, double dt,
                                           double* acc, typename Form<MIX>::H& z3,
                                           typename Form<MIX>::H& z4) {
  using HT = typename Form<MIX>::H;
  constexpr bool XCROSS = (KIND == 2 && COMP != DIM) || (KIND == 3);
  constexpr bool CROSS = XCROSS && COMP != 2;   // plane-local cross term
  constexpr int QFIELD = (KIND == 0) ? R3 : (KIND == 1) ? E3 : (KIND == 2) ? M3 + COMP : B3 + COMP;
  constexpr int SQ = DIM == 0 ? 1 : zm::RX;      // stride along DIM in the region
  const int buf = plane & 1;
  const int n0 = P.n0, n1 = P.n1, nd = DIM == 0 ? n0 : n1;
  const HT* Q = static_cast<const HT*>(Z.U);
  HT* RR = static_cast<HT*>(Z.U) + zm::RC;
  HT* C3 = RR + zm::RSZ;
  HT* C4 = C3 + zm::NSZ;
  constexpr int TX = zm::TX, TY = zm::TY, HL = zm::H;
  constexpr int exR = DIM == 0 ? TX + 1 : (CROSS ? TX + 2 : TX);
  constexpr int eyR = DIM == 0 ? (CROSS ? TY + 2 : TY) : TY + 1;
  constexpr int oxR = DIM == 0 ? HL - 1 : (CROSS ? HL - 1 : HL);
  constexpr int oyR = DIM == 0 ? (CROSS ? HL - 1 : HL) : HL - 1;
  constexpr int SR = DIM == 0 ? 1 : exR;
  constexpr int exN = (DIM == 0) ? TX : TX + 2, eyN = (DIM == 0) ? TY + 2 : TY;
  constexpr int oxN = (DIM == 0) ? HL : HL - 1, oyN = (DIM == 0) ? HL - 1 : HL;
  auto ri = [&](int lx, int ly) { return (ly - oyR) * exR + (lx - oxR); };
  auto ni = [&](int lx, int ly) { return (ly - oyN) * exN + (lx - oxN); };
  const HT coef = (HT)(B.cmax_in[DIM] * P.chyp[QFIELD]);
  const double* dlv = DIM == 0 ? Z.dl0 : Z.dl1;
  const double* rdv = DIM == 0 ? Z.rd0 : Z.rd1;

  // ratio R(i) = max D3(i-1..i+1) / max D1(i-2..i+2) from q(i-2..i+3)
  for (int r = tid; r < exR * eyR; r += zm::NT) {
    const int lx = oxR + r % exR, ly = oyR + r / exR;
    const int l = ly * zm::RX + lx;
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
  // cross-term arrays on the tile +-1 across (hyperdifmomsourcene2-4 /
  // hyperdifbsourcene1b-4)
  if (CROSS) {
    for (int r = tid; r < exN * eyN; r += zm::NT) {
      const int lx = oxN + r % exN, ly = oyN + r / exN;
      const int ci = Z.x0 - HL + lx, cj = Z.y0 - HL + ly;
      HT c3 = 0, c4 = 0;
      if (Z.inner || (ci > 0 && ci < n0 - 1 && cj > 0 && cj < n1 - 1)) {
        const int a = DIM == 0 ? ci : cj;
        const int l = ly * zm::RX + lx;
        HT g = ((Q[l + SQ] - Q[l - SQ]) * (HT)(DIM == 0 ? Z.rd0[lx] : Z.rd1[ly])) * (HT)0.5;
        if ((P.bt[DIM] != 0) && zero1n(a, nd)) g = 0;
        HT nsum = 0;
        if (Z.inner || (ci >= 2 && ci <= n0 - 3 && cj >= 2 && cj <= n1 - 3)) {
          const int rr = ri(lx, ly);
          const HT c = (HT)(DIM == 0 ? Z.dl0[lx] : Z.dl1[ly]) * coef;
          nsum = c * RR[rr] + c * RR[rr - SR];
        }
        if (KIND == 2) {
          const HT tau = (g * nsum) * (HT)0.25;
          c3 = (HT)(Z.v(buf, R3, l) + Z.RB[buf * zm::RC + l]) * tau;
          c4 = tau * (HT)Z.v(buf, M3 + DIM, l);
        } else {
          const HT t3 = (g * nsum) * (HT)0.5;
          c3 = t3;
          c4 = t3 * (HT)Z.v(buf, B3 + DIM, l);
        }
      }
      C3[r] = c3;
      C4[r] = c4;
    }
    __syncthreads();
  }
  if (own) {
    const int a = DIM == 0 ? gi : gj;
    const int la = DIM == 0 ? lxo : lyo;
    const int l = lyo * zm::RX + lxo;
    const int rr = ri(lxo, lyo);
    const HT c = (HT)dlv[la] * coef;
    const HT nur = c * RR[rr], nul = c * RR[rr - SR];
    const HT rdl = (HT)rdv[la];
    const HT qc = Q[l], qp = Q[l + SQ], qm = Q[l - SQ];
    HT gr = (qp - qc) * rdl;  // grad1r3n
    HT gl = (qc - qm) * rdl;  // grad1l3n
    if ((P.bt[DIM] != 0) && zero1n(a, nd)) { gr = 0; gl = 0; }
    if (KIND == 0) {
      acc[R3] = acc[R3] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 1) {
      acc[E3] = acc[E3] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 2) {
      // hyperdifmomsource1-3a (src/hyperdifmomsource1.cu:17-511), ii0 = COMP
      const double rb0 = Z.RB[buf * zm::RC + l], rbm = Z.RB[buf * zm::RC + l - SQ],
                   rbp = Z.RB[buf * zm::RC + l + SQ];
      const double r0 = Z.v(buf, R3, l) + rb0;
      const HT t2 = (HT)((r0 + Z.v(buf, R3, l - SQ) + rbm) * 0.5);
      const HT t3 = (HT)((r0 + Z.v(buf, R3, l + SQ) + rbp) * 0.5);
      const double mf = Z.v(buf, M3 + COMP, l);
      const HT t5 = (HT)((mf + Z.v(buf, M3 + COMP, l - SQ)) * 0.5);
      const HT t6 = (HT)((mf + Z.v(buf, M3 + COMP, l + SQ)) * 0.5);
      const double dm = (double)(((t3 * nur * gr - t2 * nul * gl) * rdl) * (HT)0.5);
      const double de = (double)(((t6 * nur * gr - t5 * nul * gl) * rdl) * (HT)0.5);
      acc[M3 + COMP] = acc[M3 + COMP] + dt * dm;
      acc[E3] = acc[E3] + dt * de;
      if (COMP == DIM) {
        acc[M3 + COMP] = acc[M3 + COMP] + dt * dm;
        acc[E3] = acc[E3] + dt * de;
      } else if (CROSS) {
        // hyperdifmomsourcene5-6a: d/dx_COMP of (rho_t tau) and (tau m_DIM)
        constexpr int FS = (COMP == 0) ? 1 : exN;
        const int af = COMP == 0 ? gi : gj;
        const HT rdf = (HT)(COMP == 0 ? Z.rd0[lxo] : Z.rd1[lyo]);
        const int nidx = ni(lxo, lyo);
        HT g7 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
        HT g8 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
        if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) { g7 = 0; g8 = 0; }
        acc[M3 + DIM] = acc[M3 + DIM] + dt * (double)g7;
        acc[E3] = acc[E3] + dt * (double)g8;
      }
    } else {
      // B component COMP diffused along DIM: hyperdifbsourcene (sb=-1) then
      // hyperdifbsource (sb=+1)
      if (CROSS) {
        constexpr int FS = (COMP == 0) ? 1 : exN;
        const int af = COMP == 0 ? gi : gj;
        const HT rdf = (HT)(COMP == 0 ? Z.rd0[lxo] : Z.rd1[lyo]);
        const int nidx = ni(lxo, lyo);
        HT g4 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
        HT g6 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
        if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) { g4 = 0; g6 = 0; }
        acc[B3 + DIM] = acc[B3 + DIM] - dt * (double)g4;
        acc[E3] = acc[E3] - dt * (double)g6;
      }
      const HT t2 = (qc + qm) * (HT)0.5, t3 = (qc + qp) * (HT)0.5;
      const double dB = (double)((gr * nur - gl * nul) * rdl);
      const double de = (double)((t3 * gr * nur - t2 * gl * nul) * rdl);
      acc[B3 + COMP] = acc[B3 + COMP] + dt * dB;
      acc[E3] = acc[E3] + dt * de;
    }
    if (XCROSS && COMP == 2) {
      // cross quantities of the own cell, differentiated along z later
      HT g = ((qp - qm) * rdl) * (HT)0.5;
      if ((P.bt[DIM] != 0) && zero1n(a, nd)) g = 0;
      const HT nsum = c * RR[rr] + c * RR[rr - SR];
      if (KIND == 2) {
        const HT tau = (g * nsum) * (HT)0.25;
        z3 = (HT)(Z.v(buf, R3, l) + Z.RB[buf * zm::RC + l]) * tau;
        z4 = tau * (HT)Z.v(buf, M3 + DIM, l);
      } else {
        const HT t3 = (g * nsum) * (HT)0.5;
        z3 = t3;
        z4 = t3 * (HT)Z.v(buf, B3 + DIM, l);
      }
    }
  }
  __syncthreads();
}

// ---- hyperdiffusion along z at plane k ----------------------------------------
// Field kind KIND / component COMP; q and the ratios come from the rings (tile
// fields rho, e, m_z; tile + 1 fields m_x, m_y, B_x, B_y), the state of the
// planes k and k+1 from the staged region, that of plane k-1 from the
// thread's carried values prev_rt (rho, rho_b) and prev_m.
template <bool BG, bool MIX, int KIND, int COMP>
__device__ __forceinline__ void zm_z_pass(const ZS<BG, MIX>& Z, const KParams& P, const KBufs& B, int tid,
                                          int k, bool own, int lxo, int lyo, int gi, int gj, double dt,
                                          double dlz, double rdz, const double* prev_rt, const double* prev_m,
                                          double* acc) {
  using HT = typename Form<MIX>::H;
  constexpr bool CROSS = (KIND == 2 && COMP != 2) || (KIND == 3);
  constexpr int QFIELD = (KIND == 0) ? R3 : (KIND == 1) ? E3 : (KIND == 2) ? M3 + COMP : B3 + COMP;
  constexpr int FT = (KIND == 0) ? 0 : (KIND == 1) ? 1 : 2;  // tile-field ring index
  constexpr int FHI = (KIND == 2) ? COMP : 2 + COMP;          // tile + 1 field ring index
  constexpr int TX = zm::TX, TY = zm::TY, HL = zm::H;
  const int n0 = P.n0, n1 = P.n1, n2 = P.n2;
  const int bk = k & 1, bp = (k + 1) & 1;  // region buffers of planes k and k+1
  const HT coef = (HT)(B.cmax_in[2] * P.chyp[QFIELD]);
  const HT c = (HT)dlz * coef;
  const bool zk = (P.bt[2] != 0) && zero1n(k, n2);
  HT* C3 = static_cast<HT*>(Z.U) + zm::RC + zm::RSZ;
  HT* C4 = C3 + zm::NSZ;
  constexpr int exN = (COMP == 0) ? TX + 2 : TX, eyN = (COMP == 0) ? TY : TY + 2;
  constexpr int oxN = (COMP == 0) ? HL - 1 : HL, oyN = (COMP == 0) ? HL : HL - 1;
  const HT* rzh_c = Z.RZ + (bk * zm::NQH + FHI) * zm::HC;
  const HT* rzh_p = Z.RZ + ((1 - bk) * zm::NQH + FHI) * zm::HC;
  if (CROSS) {
    // cross-term arrays on the tile +-1 along COMP (hyperdifmomsourcene2-4 /
    // hyperdifbsourcene1b-4 with the derivative of q along z)
    const HT* qp = Z.QH + (zm_slot(k + 1) * zm::NQH + FHI) * zm::HC;
    const HT* qm = Z.QH + (zm_slot(k - 1) * zm::NQH + FHI) * zm::HC;
    for (int r = tid; r < exN * eyN; r += zm::NT) {
      const int lx = oxN + r % exN, ly = oyN + r / exN;
      const int ci = Z.x0 - HL + lx, cj = Z.y0 - HL + ly;
      const int hc = (ly - HL + 1) * zm::HX + (lx - HL + 1);
      HT c3 = 0, c4 = 0;
      if (ci > 0 && ci < n0 - 1 && cj > 0 && cj < n1 - 1) {
        const int l = ly * zm::RX + lx;
        HT g = ((qp[hc] - qm[hc]) * (HT)rdz) * (HT)0.5;
        if (zk) g = 0;
        HT nsum = 0;
        if (ci >= 2 && ci <= n0 - 3 && cj >= 2 && cj <= n1 - 3) nsum = c * rzh_c[hc] + c * rzh_p[hc];
        if (KIND == 2) {
          const HT tau = (g * nsum) * (HT)0.25;
          c3 = (HT)(Z.v(bk, R3, l) + Z.RB[bk * zm::RC + l]) * tau;
          c4 = tau * (HT)Z.v(bk, M3 + 2, l);
        } else {
          const HT t3 = (g * nsum) * (HT)0.5;
          c3 = t3;
          c4 = t3 * (HT)Z.v(bk, B3 + 2, l);
        }
      }
      C3[r] = c3;
      C4[r] = c4;
    }
    __syncthreads();
  }
  if (own) {
    const int col = (lyo - HL) * TX + (lxo - HL);
    const int hc = (lyo - HL + 1) * zm::HX + (lxo - HL + 1);
    HT qc, qp, qm, rcur, rprev;
    if (CROSS) {
      qc = Z.QH[(zm_slot(k) * zm::NQH + FHI) * zm::HC + hc];
      qp = Z.QH[(zm_slot(k + 1) * zm::NQH + FHI) * zm::HC + hc];
      qm = Z.QH[(zm_slot(k - 1) * zm::NQH + FHI) * zm::HC + hc];
      rcur = rzh_c[hc];
      rprev = rzh_p[hc];
    } else {
      const HT* rzt = Z.RZ + 2 * zm::NQH * zm::HC;
      qc = Z.QT[(zm_slot(k) * zm::NQT + FT) * zm::NCOL + col];
      qp = Z.QT[(zm_slot(k + 1) * zm::NQT + FT) * zm::NCOL + col];
      qm = Z.QT[(zm_slot(k - 1) * zm::NQT + FT) * zm::NCOL + col];
      rcur = rzt[(bk * zm::NQT + FT) * zm::NCOL + col];
      rprev = rzt[((1 - bk) * zm::NQT + FT) * zm::NCOL + col];
    }
    const HT nur = c * rcur, nul = c * rprev;
    const HT rdl = (HT)rdz;
    HT gr = (qp - qc) * rdl;
    HT gl = (qc - qm) * rdl;
    if (zk) { gr = 0; gl = 0; }
    const int l = lyo * zm::RX + lxo;
    if (KIND == 0) {
      acc[R3] = acc[R3] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 1) {
      acc[E3] = acc[E3] + dt * (double)((nur * gr - nul * gl) * rdl);
    } else if (KIND == 2) {
      const double r0 = Z.v(bk, R3, l) + Z.RB[bk * zm::RC + l];
      const HT t2 = (HT)((r0 + prev_rt[0] + prev_rt[1]) * 0.5);
      const HT t3 = (HT)((r0 + Z.v(bp, R3, l) + Z.RB[bp * zm::RC + l]) * 0.5);
      const double mf = Z.v(bk, M3 + COMP, l);
      const HT t5 = (HT)((mf + prev_m[COMP]) * 0.5);
      const HT t6 = (HT)((mf + Z.v(bp, M3 + COMP, l)) * 0.5);
      const double dm = (double)(((t3 * nur * gr - t2 * nul * gl) * rdl) * (HT)0.5);
      const double de = (double)(((t6 * nur * gr - t5 * nul * gl) * rdl) * (HT)0.5);
      acc[M3 + COMP] = acc[M3 + COMP] + dt * dm;
      acc[E3] = acc[E3] + dt * de;
      if (COMP == 2) {
        acc[M3 + COMP] = acc[M3 + COMP] + dt * dm;
        acc[E3] = acc[E3] + dt * de;
      } else {
        constexpr int FS = (COMP == 0) ? 1 : exN;
        const int nidx = (lyo - oyN) * exN + (lxo - oxN);
        const int af = COMP == 0 ? gi : gj;
        const HT rdf = (HT)(COMP == 0 ? Z.rd0[lxo] : Z.rd1[lyo]);
        HT g7 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
        HT g8 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
        if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) { g7 = 0; g8 = 0; }
        acc[M3 + 2] = acc[M3 + 2] + dt * (double)g7;
        acc[E3] = acc[E3] + dt * (double)g8;
      }
    } else {
      constexpr int FS = (COMP == 0) ? 1 : exN;
      const int nidx = (lyo - oyN) * exN + (lxo - oxN);
      const int af = COMP == 0 ? gi : gj;
      const HT rdf = (HT)(COMP == 0 ? Z.rd0[lxo] : Z.rd1[lyo]);
      HT g4 = ((C3[nidx + FS] - C3[nidx - FS]) * rdf) * (HT)0.5;
      HT g6 = ((C4[nidx + FS] - C4[nidx - FS]) * rdf) * (HT)0.5;
      if ((P.bt[COMP] != 0) && zero1n(af, COMP == 0 ? n0 : n1)) { g4 = 0; g6 = 0; }
      acc[B3 + 2] = acc[B3 + 2] - dt * (double)g4;
      acc[E3] = acc[E3] - dt * (double)g6;
      const HT t2 = (qc + qm) * (HT)0.5, t3 = (qc + qp) * (HT)0.5;
      const double dB = (double)((gr * nur - gl * nul) * rdl);
      const double de = (double)((t3 * gr * nur - t2 * gl * nul) * rdl);
      acc[B3 + COMP] = acc[B3 + COMP] + dt * dB;
      acc[E3] = acc[E3] + dt * de;
    }
  }
  if (CROSS) __syncthreads();
}

// ---- fluxes along x or y on plane k and their divergence ----------------------
template <bool BG, bool MIX, int D, bool O6>
__device__ __forceinline__ void zm_flux_xy(const ZS<BG, MIX>& Z, const KParams& P, int tid, int k, bool own,
                                           int lxo, int lyo, int gi, int gj, double dt, const double* gc,
                                           double* acc) {
  constexpr int FHh = zm::fh<O6>(), FA = zm::fsz<O6>();
  constexpr int TX = zm::TX, TY = zm::TY, HL = zm::H;
  constexpr int E0 = TX + (D == 0 ? 2 * FHh : 0), E1 = TY + (D == 1 ? 2 * FHh : 0);
  constexpr int G0 = HL - (D == 0 ? FHh : 0), G1 = HL - (D == 1 ? FHh : 0);
  constexpr int FS = D == 0 ? 1 : E0;
  const int buf = k & 1;
  const int n[2] = {P.n0, P.n1};
  double* F = static_cast<double*>(Z.U);
  for (int r = tid; r < E0 * E1; r += zm::NT) {
    const int lx = G0 + r % E0, ly = G1 + r / E0;
    const int g0 = Z.x0 - HL + lx, g1 = Z.y0 - HL + ly;
    double f[7] = {0, 0, 0, 0, 0, 0, 0}, v[3] = {0, 0, 0};
    if (Z.inner || (g0 >= 0 && g0 < n[0] && g1 >= 0 && g1 < n[1])) {
      const int l = ly * zm::RX + lx;
      double s[8], g[5] = {0, 0, 0, 0, 0};
#pragma unroll
      for (int q = 0; q < 8; q++) s[q] = Z.v(buf, q, l);
      if (BG) {
        g[GEB] = Z.GB[(buf * 4 + 0) * zm::RC + l];
        g[GRB] = Z.RB[buf * zm::RC + l];
#pragma unroll
        for (int a = 0; a < 3; a++) g[GBB + a] = Z.GB[(buf * 4 + 1 + a) * zm::RC + l];
      }
      zm_flux<BG, D>(s, g, Z.RI[buf * zm::RC + l], P.gamma, f, v);
    }
#pragma unroll
    for (int q = 0; q < 7; q++) F[q * FA + r] = f[q];
    if (BG) {
#pragma unroll
      for (int q = 0; q < 3; q++) F[(7 + q) * FA + r] = v[q];
    }
  }
  __syncthreads();
  if (own) {
    const int a = D == 0 ? gi : gj;
    const bool z = ((P.bt[D] != 0) && zero3dn(a, n[D])) || (O6 && edge6(a, n[D]));
    const double rdl2 = 0.5 * (D == 0 ? Z.rd0[lxo] : Z.rd1[lyo]);
    const int fo = (lyo - G1) * E0 + (lxo - G0);
    constexpr int c1 = D == 0 ? 1 : 0, c2 = D == 2 ? 1 : 2;
    const int fld[7] = {R3, M3, M3 + 1, M3 + 2, E3, B3 + c1, B3 + c2};
#pragma unroll
    for (int q = 0; q < 7; q++) {
      double gk = dflux<O6>(F + q * FA, fo, FS, rdl2);
      if (z) gk = 0;
      acc[fld[q]] = acc[fld[q]] - dt * gk;
    }
    if (BG) {
      // addenergyterms_cd2 (src/centdiff2.cu:80-115): -p_tb dv_D/dx_D and the
      // derivative-along-D part of sum_i Bb_i Bb_d dv_d/dx_i
      const double bb[3] = {gc[2], gc[3], gc[4]};
      const double ptb = (P.gamma - 1) * gc[0] - 0.5 * (P.gamma - 2) * (bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
      double gv = dflux<O6>(F + (7 + D) * FA, fo, FS, rdl2);
      if (z) gv = 0;
      acc[E3] -= dt * ptb * gv;
#pragma unroll
      for (int q = 0; q < 3; q++) {
        double gk = dflux<O6>(F + (7 + q) * FA, fo, FS, rdl2);
        if (z) gk = 0;
        acc[E3] += dt * bb[D] * bb[q] * gk;
      }
    }
  }
  __syncthreads();
}

// z-divergence of the flux ring at plane k (own column)
template <bool BG, bool O6>
__device__ __forceinline__ void zm_flux_z(const double* FR, const KParams& P, int k, int col, double dt,
                                          double rdz, const double* gc, double* acc) {
  constexpr int FHh = zm::fh<O6>(), NFr = zm::nf<O6>(), NQ = zm::nfq<BG>();
  const bool z = ((P.bt[2] != 0) && zero3dn(k, P.n2)) || (O6 && edge6(k, P.n2));
  const double rdl2 = 0.5 * rdz;
  auto at = [&](int q, double* w) {
#pragma unroll
    for (int s = 0; s < 2 * FHh + 1; s++) w[s] = FR[(((k - FHh + s + NFr) % NFr) * NQ + q) * zm::NCOL + col];
  };
  const int fld[7] = {R3, M3, M3 + 1, M3 + 2, E3, B3, B3 + 1};
#pragma unroll
  for (int q = 0; q < 7; q++) {
    double w[2 * FHh + 1];
    at(q, w);
    double gk = dflux<O6>(w, FHh, 1, rdl2);
    if (z) gk = 0;
    acc[fld[q]] = acc[fld[q]] - dt * gk;
  }
  if (BG) {
    const double bb[3] = {gc[2], gc[3], gc[4]};
    const double ptb = (P.gamma - 1) * gc[0] - 0.5 * (P.gamma - 2) * (bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
    double w[2 * FHh + 1];
    at(7 + 2, w);
    double gv = dflux<O6>(w, FHh, 1, rdl2);
    if (z) gv = 0;
    acc[E3] -= dt * ptb * gv;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      at(7 + q, w);
      double gk = dflux<O6>(w, FHh, 1, rdl2);
      if (z) gk = 0;
      acc[E3] += dt * bb[2] * bb[q] * gk;
    }
  }
}

template <int MODE, bool BG, bool MIX, bool O6>
__global__ void __launch_bounds__(zm::NT, 1) stage3d_zm(const KParams P, const KBufs B, int zchunk) {
  using ST = typename Form<MIX>::S;
  using HT = typename Form<MIX>::H;
  using L = zm::Lay<BG, MIX, O6>;
  extern __shared__ __align__(16) unsigned char zsm[];
  ZS<BG, MIX> Z;
  Z.S = reinterpret_cast<ST*>(zsm + L::S);
  Z.RB = reinterpret_cast<double*>(zsm + L::RB);
  Z.RI = reinterpret_cast<double*>(zsm + L::RI);
  Z.GB = reinterpret_cast<double*>(zsm + L::GB);
  Z.QH = reinterpret_cast<HT*>(zsm + L::QH);
  Z.QT = reinterpret_cast<HT*>(zsm + L::QT);
  Z.RZ = reinterpret_cast<HT*>(zsm + L::RZ);
  Z.FR = reinterpret_cast<double*>(zsm + L::FR);
  Z.U = zsm + L::U;
  Z.dl0 = reinterpret_cast<double*>(zsm + L::MET);
  Z.rd0 = Z.dl0 + zm::RX;
  Z.dl1 = Z.rd0 + zm::RX;
  Z.rd1 = Z.dl1 + zm::RY;
  const int tid = threadIdx.x;
  const int n0 = P.n0, n1 = P.n1, n2 = P.n2;
  const long nc = P.ncell;
  Z.x0 = 2 + blockIdx.x * zm::TX;
  Z.y0 = 2 + blockIdx.y * zm::TY;
  Z.inner = blockIdx.x >= 1 && blockIdx.y >= 1 && Z.x0 + zm::TX + zm::H <= n0 && Z.y0 + zm::TY + zm::H <= n1;
  const int k0 = 2 + blockIdx.z * zchunk;
  const int k1 = min(k0 + zchunk, n2 - 2);

  // owner of a column: threads 0..NCOL-1
  const bool owner = tid < zm::NCOL;
  const int tx = tid % zm::TX, ty = (tid / zm::TX) % zm::TY;
  const int lxo = tx + zm::H, lyo = ty + zm::H;
  const int gi = Z.x0 + tx, gj = Z.y0 + ty;
  const bool own = owner && gi <= n0 - 3 && gj <= n1 - 3;  // owner of an interior column
  const int col = ty * zm::TX + tx;

  // per-axis metric of the region
  for (int r = tid; r < zm::RX + zm::RY; r += zm::NT) {
    if (r < zm::RX) {
      const int g = Z.x0 - zm::H + r;
      const double d = (g >= 0 && g < n0) ? B.delx[0][g] : 1.0;
      Z.dl0[r] = d;
      Z.rd0[r] = 1.0 / d;
    } else {
      const int g = Z.y0 - zm::H + (r - zm::RX);
      const double d = (g >= 0 && g < n1) ? B.delx[1][g] : 1.0;
      Z.dl1[r - zm::RX] = d;
      Z.rd1[r - zm::RX] = 1.0 / d;
    }
  }

  // dt of this step and stage time
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

  // ---- prologue: q ring planes k0-3 .. k0, flux ring planes k0-FH .. k0+FH-3
  for (int j = k0 - 3; j <= k0; j++) zm_ring_q(Z, P, B, j, tid, zm::NT);
  if (owner && gi < n0 && gj < n1)
    for (int j = k0 - zm::fh<O6>(); j <= k0 + zm::fh<O6>() - 3; j++) zm_ring_flux<BG, MIX, O6>(Z, P, B, j, col, gi, gj);

  // per-thread state carried along z
  HT zp[4][2], zc[4][2], zn[4][2];  // z-cross quantities of planes k-1, k, k+1
#pragma unroll
  for (int a = 0; a < 4; a++) zp[a][0] = zp[a][1] = zc[a][0] = zc[a][1] = zn[a][0] = zn[a][1] = (HT)0;
  double onext[8], ocur[8];         // look-ahead accumulators (m_z, B_z, e used)
#pragma unroll
  for (int f = 0; f < 8; f++) onext[f] = ocur[f] = 0.0;
  double prev_rt[2] = {0, 0}, prev_m[3] = {0, 0, 0};  // rho, rho_b and m at plane k-1
  double cm[3] = {P.cmax_floor[0], P.cmax_floor[1], P.cmax_floor[2]};

  for (int k = k0 - 2; k < k1; k++) {
    // ---- stage plane k+1 (plane k was staged by the previous iteration)
    __syncthreads();
    zm_load_region(Z, P, B, k + 1, tid);
    // ---- rings: fluxes of plane k+FH (owners), q of plane k+3 (the others)
    if (owner) {
      if (gi < n0 && gj < n1) zm_ring_flux<BG, MIX, O6>(Z, P, B, k + zm::fh<O6>(), col, gi, gj);
    } else {
      zm_ring_q(Z, P, B, k + 3, tid - zm::NCOL, zm::NCOL);
    }
    __syncthreads();
    // ---- ratios along z of plane k (the next plane's nu_l needs them too)
    if (k >= k0 - 1) {
      HT* rzh = Z.RZ + (k & 1) * zm::NQH * zm::HC;
      for (int i = tid; i < zm::NQH * zm::HC; i += zm::NT) {
        const int f = i / zm::HC, hc = i % zm::HC;
        rzh[f * zm::HC + hc] = zm_ratio(Z.QH + f * zm::HC, k, zm::NQH * zm::HC, hc);
      }
      HT* rzt = Z.RZ + 2 * zm::NQH * zm::HC + (k & 1) * zm::NQT * zm::NCOL;
      for (int i = tid; i < zm::NQT * zm::NCOL; i += zm::NT) {
        const int f = i / zm::NCOL, c = i % zm::NCOL;
        rzt[f * zm::NCOL + c] = zm_ratio(Z.QT + f * zm::NCOL, k, zm::NQT * zm::NCOL, c);
      }
    }
    // ---- look-ahead plane k+1: m_z and B_z diffused along x and y
    const int kn = k + 1;
#pragma unroll
    for (int f = 0; f < 8; f++) onext[f] = 0.0;
    if (P.hyperdif == 1 && kn >= 2 && kn <= n2 - 3) {
      zm_stage_q<BG, MIX, 2, 2>(Z, P, B, kn, tid);
      zm_xy_pass<BG, MIX, 2, 2, 0>(Z, P, B, tid, kn, own, lxo, lyo, gi, gj, dt, onext, zn[0][0], zn[0][1]);
      zm_xy_pass<BG, MIX, 2, 2, 1>(Z, P, B, tid, kn, own, lxo, lyo, gi, gj, dt, onext, zn[1][0], zn[1][1]);
      zm_stage_q<BG, MIX, 3, 2>(Z, P, B, kn, tid);
      zm_xy_pass<BG, MIX, 3, 2, 0>(Z, P, B, tid, kn, own, lxo, lyo, gi, gj, dt, onext, zn[2][0], zn[2][1]);
      zm_xy_pass<BG, MIX, 3, 2, 1>(Z, P, B, tid, kn, own, lxo, lyo, gi, gj, dt, onext, zn[3][0], zn[3][1]);
    } else {
#pragma unroll
      for (int a = 0; a < 4; a++) zn[a][0] = zn[a][1] = (HT)0;
    }

    if (k >= k0) {
      // ---- plane k
      const int bk = k & 1;
      const int lo = lyo * zm::RX + lxo;
      const long co = own ? ((long)k * n1 + gj) * n0 + gi : 0;
      const double dlz = B.delx[2][k], rdz = 1.0 / dlz;
      double sc[8], gc[5] = {0, 0, 0, 0, 0};
#pragma unroll
      for (int f = 0; f < 8; f++) sc[f] = Z.v(bk, f, lo);
      gc[GRB] = Z.RB[bk * zm::RC + lo];
      if (BG) {
        gc[GEB] = Z.GB[(bk * 4 + 0) * zm::RC + lo];
#pragma unroll
        for (int a = 0; a < 3; a++) gc[GBB + a] = Z.GB[(bk * 4 + 1 + a) * zm::RC + lo];
      }
      double out[8];
#pragma unroll
      for (int f = 0; f < 8; f++) {
        if (MODE != SMAUG_INT_EULER)
          out[f] = 0.0;
        else if (MIX)
          out[f] = own ? base_value<MIX>(B, f * nc + co) : 0.0;
        else
          out[f] = sc[f];
      }
      // fluxes and divergence along x, y (plane-local) and z (flux ring)
      zm_flux_xy<BG, MIX, 0, O6>(Z, P, tid, k, own, lxo, lyo, gi, gj, dt, gc, out);
      zm_flux_xy<BG, MIX, 1, O6>(Z, P, tid, k, own, lxo, lyo, gi, gj, dt, gc, out);
      if (own) zm_flux_z<BG, O6>(Z.FR, P, k, col, dt, rdz, gc, out);
      // gravity (addgrav_cd2, src/centdiff2.cu:118-154)
      if (P.has_grav && own) {
        const double rho = sc[R3];
        out[M3 + 0] += dt * P.g[0] * rho;
        out[M3 + 1] += dt * P.g[1] * rho;
        out[M3 + 2] += dt * P.g[2] * rho;
        const double rr = rho * Z.RI[bk * zm::RC + lo];
        out[E3] += (dt * P.g[0] * sc[M3 + 0]) * rr;
        out[E3] += (dt * P.g[1] * sc[M3 + 1]) * rr;
        out[E3] += (dt * P.g[2] * sc[M3 + 2]) * rr;
      }
      if (P.hyperdif == 1) {
        HT dz3 = 0, dz4 = 0;
#define XYP(K, C, D) zm_xy_pass<BG, MIX, K, C, D>(Z, P, B, tid, k, own, lxo, lyo, gi, gj, dt, out, dz3, dz4)
#define ZP(K, C) \
  zm_z_pass<BG, MIX, K, C>(Z, P, B, tid, k, own, lxo, lyo, gi, gj, dt, dlz, rdz, prev_rt, prev_m, out)
        zm_stage_q<BG, MIX, 0, 0>(Z, P, B, k, tid);
        XYP(0, 0, 0); XYP(0, 0, 1); ZP(0, 0);
        zm_stage_q<BG, MIX, 1, 0>(Z, P, B, k, tid);
        XYP(1, 0, 0); XYP(1, 0, 1); ZP(1, 0);
        zm_stage_q<BG, MIX, 2, 0>(Z, P, B, k, tid);
        XYP(2, 0, 0); XYP(2, 0, 1); ZP(2, 0);
        zm_stage_q<BG, MIX, 2, 1>(Z, P, B, k, tid);
        XYP(2, 1, 0); XYP(2, 1, 1); ZP(2, 1);
        ZP(2, 2);
        zm_stage_q<BG, MIX, 3, 0>(Z, P, B, k, tid);
        XYP(3, 0, 1); ZP(3, 0);
        zm_stage_q<BG, MIX, 3, 1>(Z, P, B, k, tid);
        XYP(3, 1, 0); ZP(3, 1);
#undef XYP
#undef ZP
        if (own) {
          // m_z and B_z diffused along x and y: their diagonal parts (from the
          // previous plane's look-ahead) and their cross terms, differentiated
          // along z from the planes below and above
          out[M3 + 2] += ocur[M3 + 2];
          out[B3 + 2] += ocur[B3 + 2];
          out[E3] += ocur[E3];
          const bool zz = (P.bt[2] != 0) && zero1n(k, n2);
#pragma unroll
          for (int a = 0; a < 4; a++) {
            HT g3 = ((zn[a][0] - zp[a][0]) * (HT)rdz) * (HT)0.5;
            HT g4 = ((zn[a][1] - zp[a][1]) * (HT)rdz) * (HT)0.5;
            if (zz) { g3 = 0; g4 = 0; }
            if (a < 2) {  // momentum: d/dz (rho_t tau) -> m_DIM, d/dz (tau m_DIM) -> e
              out[M3 + a] = out[M3 + a] + dt * (double)g3;
              out[E3] = out[E3] + dt * (double)g4;
            } else {      // field: -d/dz (...) -> B_DIM, e
              out[B3 + a - 2] = out[B3 + a - 2] - dt * (double)g3;
              out[E3] = out[E3] - dt * (double)g4;
            }
          }
        }
      }
      // user driver (source_parallel + addsourceterms2)
      if (P.driver == SMAUG_DRIVER_GAUSS && own) {
        double v = P.drv_amp;
        if (P.drv_period > 0) v *= sin(tstage * 2.0 * M_PI / P.drv_period);
        const int gt[3] = {gi, gj, k};
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
      // combine, write, ghost images, CFL maxima
      if (own) {
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
        ix[0] = gi;
        iy[0] = gj;
        iz[0] = k;
        const int nx = 1 + ghost_images(gi, n0, P.bc[0], ix + 1);
        const int ny = 1 + ghost_images(gj, n1, P.bc[1], iy + 1);
        const int nz = 1 + ghost_images(k, n2, P.bc[2], iz + 1);
        bool negated = false;  // res holds the negated values
        for (int cz = 0; cz < nz; cz++)
          for (int b = 0; b < ny; b++)
            for (int a2 = 0; a2 < nx; a2++) {
              const long cc = ((long)iz[cz] * n1 + iy[b]) * n0 + ix[a2];
              // antisymmetric images carry the opposite sign (negation is exact)
              const bool neg = (((a2 > 0) && P.gneg[0]) != ((b > 0) && P.gneg[1])) != ((cz > 0) && P.gneg[2]);
              if (neg != negated) {
#pragma unroll
                for (int f = 0; f < 8; f++) res[f] = -res[f];
                negated = neg;
              }
#pragma unroll
              for (int f = 0; f < 8; f++) store_value<MIX>(B, f * nc + cc, res[f], is_base);
              double gg[5];
              if (BG && a2 == 0 && b == 0 && cz == 0) {
#pragma unroll
                for (int f = 0; f < 5; f++) gg[f] = gc[f];
              } else {
#pragma unroll
                for (int f = 0; f < 5; f++) gg[f] = __ldg(B.bg + f * nc + cc);
              }
              double cv[3];
              cfast3_all(P.gamma, res, gg, cv);
#pragma unroll
              for (int d = 0; d < 3; d++) cm[d] = dmax0(cm[d], cv[d]);
            }
      }
    }
    // ---- carry along z
    if (own) {
      const int bk = k & 1;
      const int lo = lyo * zm::RX + lxo;
      prev_rt[0] = Z.v(bk, R3, lo);
      prev_rt[1] = Z.RB[bk * zm::RC + lo];
#pragma unroll
      for (int a = 0; a < 3; a++) prev_m[a] = Z.v(bk, M3 + a, lo);
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
      zp[a][0] = zc[a][0];
      zp[a][1] = zc[a][1];
      zc[a][0] = zn[a][0];
      zc[a][1] = zn[a][1];
    }
#pragma unroll
    for (int f = 0; f < 8; f++) ocur[f] = onext[f];
  }

  __shared__ double red[zm::NT / 32][3];
#pragma unroll
  for (int d = 0; d < 3; d++)
    for (int o = 16; o > 0; o >>= 1) cm[d] = dmax0(cm[d], __shfl_xor_sync(0xffffffffu, cm[d], o));
  __syncthreads();
  if ((tid & 31) == 0) {
    red[tid >> 5][0] = cm[0];
    red[tid >> 5][1] = cm[1];
    red[tid >> 5][2] = cm[2];
  }
  __syncthreads();
  if (tid < 3) {
    double v = 0.0;
    for (int w = 0; w < zm::NT / 32; w++) v = dmax0(v, red[w][tid]);
    atomicMax(&B.cmax_out[tid], (unsigned long long)__double_as_longlong(v));
  }
}

// planes per block along z: the largest chunk (64 at most) that still gives
// every SM several blocks
inline int zm_chunk(const KParams& K, int nsm) {
  const long cols = (long)((K.n0 - 4 + zm::TX - 1) / zm::TX) * ((K.n1 - 4 + zm::TY - 1) / zm::TY);
  const int nz = K.n2 - 4;
  int zc = 64;
  while (zc > 8 && cols * ((nz + zc - 1) / zc) < 8L * nsm) zc /= 2;
  return zc < nz ? zc : nz;
}

template <int MODE, bool MIX, bool O6>
static cudaError_t launch_stage3d_zm_o(const KParams& K, const KBufs& B, cudaStream_t st, int nsm) {
  const int zc = zm_chunk(K, nsm);
  dim3 grid((K.n0 - 4 + zm::TX - 1) / zm::TX, (K.n1 - 4 + zm::TY - 1) / zm::TY, (K.n2 - 4 + zc - 1) / zc);
  if (K.has_bg)
    stage3d_zm<MODE, true, MIX, O6><<<grid, zm::NT, zm::Lay<true, MIX, O6>::TOTAL, st>>>(K, B, zc);
  else
    stage3d_zm<MODE, false, MIX, O6><<<grid, zm::NT, zm::Lay<false, MIX, O6>::TOTAL, st>>>(K, B, zc);
  return cudaGetLastError();
}

template <int MODE, bool BG, bool MIX, bool O6>
static cudaError_t stage3d_zm_attr() {
  return cudaFuncSetAttribute(stage3d_zm<MODE, BG, MIX, O6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)zm::Lay<BG, MIX, O6>::TOTAL);
}

// one translation unit per (integrator, precision form): its launcher, with
// both stencil orders and both background specialisations, and the shared
// memory attributes of those four kernels
#define SMAUG_ZM_UNIT(MODE, MIX, NAME)                                                            \
  cudaError_t zm_launch_##NAME(const KParams& K, const KBufs& B, cudaStream_t st, int nsm) {      \
    return K.order6 ? launch_stage3d_zm_o<MODE, MIX, true>(K, B, st, nsm)                          \
                    : launch_stage3d_zm_o<MODE, MIX, false>(K, B, st, nsm);                        \
  }                                                                                               \
  cudaError_t zm_attr_##NAME() {                                                                  \
    cudaError_t e;                                                                                \
    if ((e = stage3d_zm_attr<MODE, true, MIX, false>())) return e;                                \
    if ((e = stage3d_zm_attr<MODE, true, MIX, true>())) return e;                                 \
    if ((e = stage3d_zm_attr<MODE, false, MIX, false>())) return e;                               \
    return stage3d_zm_attr<MODE, false, MIX, true>();                                             \
  }
