// dndsg_limiter.cuh -- the CWBAP limiter, VRFiniteVolume2D::ReconstructionWBAPLimitFacialV3
// (DNDS_FV_VR.hpp:2053-2329), and the 3WBAP limiter ReconstructionWBAPLimitFacialV2 (:1749-2047, at
// the end of this file), with the biway/multiway WBAP kernels of
// DNDS_FV_Limiters.hpp:341-449 and the characteristic matrices fML/fMR of
// DNDS_FV_EulerSolver.hpp:749-795.  Arithmetic in the storage precision: FP64 in FP64 contexts, FP32 in
// FP32-bulk contexts.
//
// Passes:
//   face:  smoothness-indicator integrals IJI, ISI of rho and E at the face's
//          first gauss point (the reference integrates with LINE_1 weight 2 but
//          reads the LINE_3 data of point 0), one thread per face;
//   cell:  indicator si = sqrt(max_k IJI_k / ISI_k) * P^2 (P = 2), one thread per
//          cell, which lists the cells to limit;
//   limit: four lanes per listed cell (one per conserved variable; the
//          characteristic projections exchange values by shuffles), order by
//          order (P2 rows 2..4, then P1 rows 0..1) biway WBAP against each
//          neighbour in characteristic space and a multiway WBAP of the results,
//          into a compact buffer that a last pass scatters back over the listed
//          cells' coefficients (the others keep theirs: nothing is copied).
#pragma once
#include "dndsg_bodies.cuh"

namespace dg {

// per-face data of the limiting pass, one row of kLimStride values per face (the cell-centric limiting
// pass reads a face's matrix rows together; the row is padded to 16-byte multiples), in the context's
// precision:
//   [0, 25)   msR2L (right-cell coefficients -> left basis), row-major
//   [25, 50)  msL2R
// (the indicator's data is the compact limG / limCell below)
constexpr int kLimE = 50;
constexpr int kLimStride = 52;
DG_HD int64_t lim_at(int64_t f, int e) { return f * kLimStride + e; }
constexpr int kMsR2L = 0, kMsL2R = 25;
// the indicator's compact data, in the context's precision: per face (AoSoA E = kLimG) the frame
// coordinates (xi, eta) of gauss point 0 in the left and the right cell and the 6 face weights; per
// cell ([N][kLimCell]) the frame's Pinv (row-major) and basis moments, padded to 12 so that a cell's
// row is read in 16-byte vectors.  D at the point follows from these (p2_diffs_at), a fifth of the bytes
// of storing it.
constexpr int kLimG = 10;
constexpr int kLimCell = 12;

struct LimView {
  int64_t N, F, Fi;
  int nfmax;
  const int32_t* cellFace;
  const int32_t* faceL;
  const int32_t* faceR;
  const double* faceNormal;
  const double* faceArea;
  const void* limFace;     // T [F][kLimStride] (T = the context's precision)
  const void* limG;        // T [F] AoSoA kLimG (T = the context's precision)
  const void* limCell;     // T [N][kLimCell]
  const double* u;
  void* faceInd;           // T [F][4]: IJI_rho, IJI_E, ISI_rho, ISI_E
  double* indicator;       // [N]
  double gamma;
  double tangWeight, tangModMin, tangModPower;
  int tangModLoc;
  const double* vol;
  double porder2;
  double scale;
  double nStd;
  int ifAll;
};

// setup: the limiter data of one interior face (face part of initBaseDiffCache,
// DNDS_FV_VR.cpp:536-712): D at gauss point 0 for both sides and the secondary
// reconstruction matrices from the derivative matrices at the face centre
template <class T>
DG_HD bool setup_limiter_face(int64_t f, const MeshView& m, const SetupParams& p, const CellSetup* cells,
                              const double* faceW, T* lim) {
  int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
  for (int e = 0; e < kLimStride; e++) lim[lim_at(f, e)] = T(0);
  if (R < 0) return true;
  FaceGeom g = face_geom(f, m);
  double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
  double DL[6][5], DR[6][5];
  p2_diffs(cells[L].fr, g.cx, g.cy, DL);
  p2_diffs(cells[R].fr, g.cx - sx, g.cy - sy, DR);
  // msR2L solves DL[1:] X = DR[1:]; msL2R solves DR[1:] X = DL[1:]
  double A[5][5], B[5][5];
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) { A[i][j] = DL[i + 1][j]; B[i][j] = DR[i + 1][j]; }
  bool ok = lu5_solve(A, B);
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) lim[lim_at(f, kMsR2L + i * 5 + j)] = (T)B[i][j];
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) { A[i][j] = DR[i + 1][j]; B[i][j] = DL[i + 1][j]; }
  ok = lu5_solve(A, B) && ok;
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) lim[lim_at(f, kMsL2R + i * 5 + j)] = (T)B[i][j];
  return ok;
}

// face pass of the smoothness indicator (DNDS_FV_VR.hpp:2075-2127)
// the setup of the compact data: face f's frame coordinates and weights, and (f < N) cell f's frame
template <class T>
DG_HD void setup_limiter_compact(int64_t f, const MeshView& m, const CellSetup* cells, const double* faceW, T* g,
                                 T* cellFr) {
  if (f < m.F) {
    const int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
    const FaceGeom fg = face_geom(f, m);
    const double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
    double xe[4] = {0, 0, 0, 0};
    p2_frame_coords(cells[L].fr, fg.gx[0], fg.gy[0], xe[0], xe[1]);
    if (R >= 0) p2_frame_coords(cells[R].fr, fg.gx[0] - sx, fg.gy[0] - sy, xe[2], xe[3]);
    for (int k = 0; k < 4; k++) g[aos(f, k, kLimG)] = (T)xe[k];
    for (int k = 0; k < 6; k++) g[aos(f, 4 + k, kLimG)] = (T)faceW[f * 6 + k];
  }
  if (f < m.N) {
    const CellFrame& fr = cells[f].fr;
    T* o = cellFr + f * kLimCell;
    o[0] = (T)fr.Pinv[0][0]; o[1] = (T)fr.Pinv[0][1]; o[2] = (T)fr.Pinv[1][0]; o[3] = (T)fr.Pinv[1][1];
    for (int k = 0; k < 5; k++) o[4 + k] = (T)fr.moment[k];
    for (int k = 9; k < kLimCell; k++) o[k] = T(0);
  }
}

// the indicator integrals of one face, in the storage precision T: FP64 in FP64 contexts, FP32 in
// FP32-bulk contexts (computed in T, scaled by the FP64 face area and stored in T for the cell pass)
template <class T>
DG_HD void limiter_face_indicator(int64_t f, const LimView& v, const T* urec) {
  using C = T;
  int32_t L = v.faceL[f], R = v.faceR[f];
  T* out = static_cast<T*>(v.faceInd) + f * 4;
  if (R < 0) {
    const T zero[4] = {T(0), T(0), T(0), T(0)};
    store_row(out, zero);
    return;
  }
  // per side: the rows of the cell's basis derivatives at gauss point 0 (from the cell's frame) times
  // its rho and E coefficients, the mean added to the value row; one side's derivatives live at a time
  const T* g = static_cast<const T*>(v.limG);
  const T* cf = static_cast<const T*>(v.limCell);
  const int var[2] = {0, 3};
  C sv[2][6][2];
  for (int side = 0; side < 2; side++) {
    const int64_t cell = side ? R : L;
    // the cell's frame row and its 5 x 4 coefficients (rho and E are used): in FP32 as 16-byte vectors
    // (a fourth of the load instructions of the issue-bound pass); in FP64, whose pass runs at two
    // blocks per SM with 128 registers, the nine frame values and ten coefficients one by one
    T c[kLimCell], rows[5][4];
    if constexpr (sizeof(T) == 4) {
      for (int k = 0; k < kLimCell; k += 4) load_row(cf + cell * kLimCell + k, &c[k]);
      for (int q = 0; q < 5; q++) load_row(urec + cell * 20 + 4 * q, rows[q]);
    } else {
      for (int k = 0; k < 9; k++) c[k] = cf[cell * kLimCell + k];
      for (int q = 0; q < 5; q++) {
        rows[q][0] = urec[cell * 20 + 4 * q];
        rows[q][3] = urec[cell * 20 + 4 * q + 3];
      }
    }
    const C Q[2][2] = {{c[0], c[1]}, {c[2], c[3]}};
    const C mo[5] = {c[4], c[5], c[6], c[7], c[8]};
    C D[6][5];
    p2_diffs_at<C>(Q, mo, g[aos(f, 2 * side, kLimG)], g[aos(f, 2 * side + 1, kLimG)], D);
    for (int k = 0; k < 2; k++) {
      C r[5];
      for (int q = 0; q < 5; q++) r[q] = rows[q][k == 0 ? 0 : 3];
      for (int d = 0; d < 6; d++) {
        C a = C(0);
        for (int q = 0; q < 5; q++) a += D[d][q] * r[q];
        if (d == 0) a += (C)v.u[cell * 4 + var[k]];
        sv[side][d][k] = a;
      }
    }
  }
  C val[6][2], jump[6][2];
  for (int c = 0; c < 2; c++)
    for (int d = 0; d < 6; d++) {
      val[d][c] = (sv[0][d][c] + sv[1][d][c]) * C(0.5);
      jump[d][c] = (sv[0][d][c] - sv[1][d][c]) * C(0.5);
    }
  C W[6];
  for (int k = 0; k < 6; k++) W[k] = g[aos(f, 4 + k, kLimG)];
  const double area = v.faceArea[f];
  C tm = C(1);  // the tangential-weight modifier; exactly 1 when tangWeightModMin is 1
  if (v.tangModMin != 1.0) {
    const double sL = sqrt(v.vol[L]) / area, sR = sqrt(v.vol[R]) / area;
    const double arMax = dmax(1.0, dmax(sL, sR));
    tm = (C)pow((1.0 / arMax) * (1 - v.tangModMin) + v.tangModMin, v.tangModPower);
  }
  const FaceFunctionalT<C> Fn = make_functional<C>(W, (C)v.faceNormal[2 * f], (C)v.faceNormal[2 * f + 1],
                                                   (C)v.tangWeight, tm, v.tangModLoc);
  C ij[2] = {C(0), C(0)}, is[2] = {C(0), C(0)};
  for (int a = 0; a < 6; a++)
    for (int c = 0; c < 2; c++) {
      C pj = C(0), ps = C(0);
      for (int r = 0; r < 6; r++) { pj += Fn.t[a][r] * jump[r][c]; ps += Fn.t[a][r] * val[r][c]; }
      ij[c] += pj * pj;
      is[c] += ps * ps;
    }
  // |n| of gauss point 0 is area/2, times the LINE_1 weight 2
  const T rec[4] = {(T)((double)ij[0] * area), (T)((double)ij[1] * area), (T)((double)is[0] * area),
                    (T)((double)is[1] * area)};
  store_row(out, rec);
}

// cell pass of the indicator: si = sqrt(max |IJI/ISI|) * P^2, the face integrals (precision T) summed
// in FP64
template <class T>
DG_HD double limiter_cell_indicator(int64_t i, const LimView& v) {
  double sj[2] = {0, 0}, ss[2] = {0, 0};
  for (int k = 0; k < v.nfmax; k++) {
    int32_t sf = v.cellFace[aos(i, k, v.nfmax)];
    if (sf == kEmptySlot) continue;
    int32_t f = sf >= 0 ? sf : ~sf;
    T d[4];
    load_row(static_cast<const T*>(v.faceInd) + (int64_t)f * 4, d);
    sj[0] += (double)d[0]; sj[1] += (double)d[1]; ss[0] += (double)d[2]; ss[1] += (double)d[3];
  }
  double s0 = sj[0] / (ss[0] + kVerySmall), s1 = sj[1] / (ss[1] + kVerySmall);
  return sqrt(dmax(fabs(s0), fabs(s1))) * v.porder2;
}

DG_HD double signE(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
DG_HD float signE(float x) { return x > 0 ? 1.0f : (x < 0 ? -1.0f : 0.0f); }

// Quotients and square roots of the limiting pass.  FP64 contexts keep exact operations; in FP32-bulk
// contexts the pass is bound by instruction issue, and the hardware approximations serve: __fdividef
// (2 ulp for divisors in [2^-126, 2^126], which every divisor it is given here lies in) and x rsqrt(x)
// (about 2 ulp), far below the FP32 tolerance of the limited coefficients
DG_HD double lim_div(double a, double b) { return a / b; }
DG_HD double lim_sqrt(double x) { return sqrt(x); }
DG_HD float lim_div(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdividef(a, b);
#else
  return a / b;
#endif
}
DG_HD float lim_sqrt(float x) {
#if defined(__CUDA_ARCH__)
  return x > 0.f ? x * rsqrtf(x) : 0.f;
#else
  return sqrtf(x);
#endif
}

// FWBAP_L2_Biway(u1, u2, out, n) (DNDS_FV_Limiters.hpp:410-449), p = 4
DG_HD double wbap_biway(double u1, double u2, double n) {
  double frac = u1 / (fabs(u2) + 1e-12) * signE(u2);
  double th1 = frac * frac * frac, th2 = (frac * frac) * (frac * frac);
  return u1 * (n + th1) / (n + th2);
}
// the same in FP32: |frac| is capped at 1e9 so that frac^4 stays finite (above the cap the
// FP64 result is below 1e-9 |u1|, under FP32 resolution of u1, and the capped one is as small)
DG_HD float wbap_biway(float u1, float u2, float n) {
  float frac = lim_div(u1, fabsf(u2) + 1e-12f) * signE(u2);  // divisor in [1e-12, FLT_MAX]
  frac = copysignf(fminf(fabsf(frac), 1e9f), frac);
  const float th1 = frac * frac * frac, th2 = (frac * frac) * (frac * frac);
  return u1 * lim_div(n + th1, n + th2);  // divisor in [n, n + 1e36], n >= 1
}
// one term of FWBAP_L2_Multiway (DNDS_FV_Limiters.hpp:341-405): theta = u0 / (|s| + verySmall^(1/4))
// * sign(s), accumulated as theta^4 (down) and theta^3 (up); in FP32 capped at 1e9 as above
DG_HD void wbap_multi_term(double u0, double s, double& up, double& down) {
  const double ti = u0 / (fabs(s) + 1e-50) * signE(s);
  down += (ti * ti) * (ti * ti);
  up += ti * ti * ti;
}
DG_HD void wbap_multi_term(float u0, float s, float& up, float& down) {
  float ti = s != 0.f ? u0 / fabsf(s) * signE(s) : 0.f;
  ti = copysignf(fminf(fabsf(ti), 1e9f), ti);
  down += (ti * ti) * (ti * ti);
  up += ti * ti * ti;
}

// Row `a` of the left and right characteristic matrices fML / fMR at the face mean state
// (DNDS_FV_EulerSolver.hpp:749-795, Gas::EulerGasLeft/RightEigenVector, DNDS_Gas.hpp:17-71):
// Lrow[q] = L[a][q] and Rrow[q] = R[a][q], in the arithmetic type C.
template <class C>
DG_HD void char_rows(int a, C gamma, const double* UL, const double* UR, C nx, C ny, C Lrow[4], C Rrow[4]) {
  C UC[4], r[4];
  for (int k = 0; k < 4; k++) UC[k] = (C)((UL[k] + UR[k]) * 0.5);
  to_normal_frame(UC, nx, ny, r);
  const C ir = lim_div(C(1), r[0]);
  const C vx = r[1] * ir, vy = r[2] * ir, vs = vx * vx + vy * vy;
  C p, a2, H, as, sc, asg, a2g, a4g;  // as / (gamma - 1), as^2 / (gamma - 1), 4 as^2 / (gamma - 1)
  const C gb = gamma - C(1);
  if constexpr (sizeof(C) == 4) {  // FP32: one reciprocal each of rho, a^2 and gamma - 1
    const C igb = lim_div(C(1), gb);
    p = gb * (r[3] - r[0] * C(0.5) * vs);
    a2 = gamma * p * ir;
    H = (r[3] + p) * ir;
    as = lim_sqrt(a2);
    sc = gb * lim_div(C(0.5), a2);
    asg = as * igb;
    a2g = a2 * igb;
    a4g = C(4) * a2g;
  } else {  // FP64: the operations in the order of the reference's expressions
    thermal(r[3], r[0], vs, gamma, p, a2, H);
    as = sqrt(a2);
    sc = gb / (C(2) * as * as);
    asg = as / gb;
    a2g = (as * as) / gb;
    a4g = C(4) / gb * (as * as);
  }
  C L0[4];
  if (a == 0) { L0[0] = H + asg * (vx - as); L0[1] = -vx - asg; L0[2] = -vy; L0[3] = C(1); }
  else if (a == 1) { L0[0] = -C(2) * H + a4g; L0[1] = vx * 2; L0[2] = vy * 2; L0[3] = -C(2); }
  else if (a == 2) { L0[0] = vy * (-C(2) * a2g); L0[1] = C(0); L0[2] = C(2) * a2g; L0[3] = C(0); }
  else { L0[0] = H - asg * (vx + as); L0[1] = -vx + asg; L0[2] = -vy; L0[3] = C(1); }
  // L = L0 * diag(1, base^T) in the momentum block: columns 1, 2 times [[nx, ny], [-ny, nx]]
  const C c1 = L0[1] * sc, c2 = L0[2] * sc;
  Lrow[0] = L0[0] * sc; Lrow[1] = c1 * nx - c2 * ny; Lrow[2] = c1 * ny + c2 * nx; Lrow[3] = L0[3] * sc;
  // R0 rows 1 and 2 mix under the rotation: R[1] = nx R0[1] - ny R0[2], R[2] = ny R0[1] + nx R0[2]
  const C R1[4] = {vx - as, vx, C(0), vx + as}, R2[4] = {vy, vy, C(1), vy};
  if (a == 0) { Rrow[0] = C(1); Rrow[1] = C(1); Rrow[2] = C(0); Rrow[3] = C(1); }
  else if (a == 3) { Rrow[0] = H - vx * as; Rrow[1] = C(0.5) * vs; Rrow[2] = vy; Rrow[3] = H + vx * as; }
  else if (a == 1) { for (int j = 0; j < 4; j++) Rrow[j] = nx * R1[j] - ny * R2[j]; }
  else { for (int j = 0; j < 4; j++) Rrow[j] = ny * R1[j] + nx * R2[j]; }
}

// The limiting pass of one listed cell on four lanes of a warp (the group's lane c owns conservative
// variable c of every coefficient row and row c of the characteristic matrices), into o (the cell's 20
// limited coefficients; rows a pass does not limit are copied).  V3 = true: ReconstructionWBAPLimitFacialV3
// (CWBAP), both orders per cell (P2 rows 2..4, then P1 rows 0..1 against the neighbour's secondary
// reconstruction whose rows 2..4 come from this cell's P2 biway results), biway with n = 1, multiway
// with n = WBAP_nStd centred on the cell's own coefficients.  V3 = false: one pass of
// ReconstructionWBAPLimitFacialV2 (3WBAP) for rows [LS, LS + NR), biway with n = WBAP_nStd, multiway
// with n = 1 centred on the first neighbour's result (a cell without interior faces keeps its rows).
// Arithmetic in the storage precision T.  All 32 lanes of the warp call this together (valid = false
// for a group without a cell): the characteristic projections exchange values by width-4 shuffles.
template <class T, bool V3, int PASS, int NF>
__device__ __forceinline__ void limiter_cell4(bool valid, int64_t i, int c, const LimView& v, const T* urec, T* o) {
  using C = T;
  const T* ms = static_cast<const T*>(v.limFace);
  const C gamma = (C)v.gamma, nStd = (C)v.nStd;
  C ri[5];
  for (int q = 0; q < 5; q++) ri[q] = valid ? urec[i * 20 + q * 4 + c] : C(0);
  double ui[4] = {1.0, 0.0, 0.0, 2.5};
  if (valid) for (int k = 0; k < 4; k++) ui[k] = v.u[i * 4 + k];
  // multiway sums per coefficient row; V2 also keeps the first neighbour's result (its centre)
  C up[5], down[5], first[5];
  for (int q = 0; q < 5; q++) up[q] = down[q] = first[q] = C(0);
  int nO = 0;
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const int32_t sf = valid ? v.cellFace[aos(i, k, NF)] : kEmptySlot;
    const int32_t f0 = sf >= 0 ? sf : ~sf;
    const int side = sf >= 0 ? 0 : 1;
    int32_t j = -1;
    if (sf != kEmptySlot) j = side == 0 ? v.faceR[f0] : v.faceL[f0];
    // every lane runs every slot (the shuffles below need all 32 lanes); a slot without an interior
    // neighbour computes on this cell's own data and is not accumulated
    const bool has = j >= 0;
    const int64_t jj = has ? j : (valid ? i : 0);
    const int64_t f = has ? f0 : 0;
    const int eMs = side == 0 ? kMsR2L : kMsL2R, eMsO = side == 0 ? kMsL2R : kMsR2L;
    C uOO[5];
    for (int q = 0; q < 5; q++) uOO[q] = urec[jj * 20 + q * 4 + c];
    double uo[4];
    for (int q = 0; q < 4; q++) uo[q] = has ? v.u[jj * 4 + q] : ui[q];
    C Lrow[4], Rrow[4];  // the face's characteristic rows, shared by both orders
    char_rows<C>(c, gamma, side ? uo : ui, side ? ui : uo, (C)v.faceNormal[2 * f], (C)v.faceNormal[2 * f + 1],
                 Lrow, Rrow);
    // biway WBAP of coefficient row q against this neighbour, in characteristic space, back to
    // conservative variables (column c of the result)
    auto biway_row = [&](int q, const C* other) -> C {
      C oin = C(0);
      for (int t = 0; t < 5; t++) oin += (C)ms[lim_at(f, eMs + q * 5 + t)] * other[t];
      const C tin = ri[q];
      C co = C(0), ct = C(0);
      for (int a = 0; a < 4; a++) {
        co += Lrow[a] * __shfl_sync(0xffffffffu, oin, a, 4);
        ct += Lrow[a] * __shfl_sync(0xffffffffu, tin, a, 4);
      }
      const C limc = wbap_biway(ct, co, V3 ? C(1) : nStd);
      C sback = C(0);
      for (int a = 0; a < 4; a++) sback += Rrow[a] * __shfl_sync(0xffffffffu, limc, a, 4);
      return sback;
    };
    if (V3) {
      // P2 rows 2..4 against the neighbour's secondary reconstruction; then P1 rows 0..1 against it
      // with rows 2..4 from this face's P2 results (successive SR): the two orders' multiway sums are
      // independent, so one pass over the faces does both
      C uF[3];
      for (int r = 0; r < 3; r++) {
        uF[r] = biway_row(2 + r, uOO);
        if (has) wbap_multi_term(ri[2 + r], uF[r], up[2 + r], down[2 + r]);
      }
      C uO1[5] = {uOO[0], uOO[1], C(0), C(0), C(0)};
      for (int q = 2; q < 5; q++)
        for (int t = 2; t < 5; t++) uO1[q] += (C)ms[lim_at(f, eMsO + q * 5 + t)] * uF[t - 2];
      for (int r = 0; r < 2; r++) {
        const C sb = biway_row(r, uO1);
        if (has) wbap_multi_term(ri[r], sb, up[r], down[r]);
      }
    } else {
      constexpr int ls = PASS == 0 ? 2 : 0, nr = PASS == 0 ? 3 : 2;
      for (int r = 0; r < nr; r++) {
        const C sb = biway_row(ls + r, uOO);
        if (!has) continue;
        if (nO == 0) first[ls + r] = sb;
        else wbap_multi_term(first[ls + r], sb, up[ls + r], down[ls + r]);
      }
    }
    if (has) nO++;
  }
  C res[5];
  for (int q = 0; q < 5; q++) res[q] = ri[q];
  if (V3) {
    for (int q = 0; q < 5; q++) res[q] = ri[q] * lim_div(up[q] + nStd, down[q] + nStd);
  } else if (nO > 0) {
    constexpr int ls = PASS == 0 ? 2 : 0, nr = PASS == 0 ? 3 : 2;
    for (int r = 0; r < nr; r++) res[ls + r] = first[ls + r] * (up[ls + r] + C(1)) / (down[ls + r] + C(1));
  }
  if (valid)
    for (int q = 0; q < 5; q++) o[q * 4 + c] = (T)res[q];
}

}  // namespace dg
