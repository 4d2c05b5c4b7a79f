// dndsg_limiter.cuh -- the CWBAP limiter, VRFiniteVolume2D::ReconstructionWBAPLimitFacialV3
// (DNDS_FV_VR.hpp:2053-2329) with the biway/multiway WBAP kernels of
// DNDS_FV_Limiters.hpp:341-449 and the characteristic matrices fML/fMR of
// DNDS_FV_EulerSolver.hpp:749-795.  Arithmetic in FP64 for both storage precisions.
//
// Three passes:
//   face:  smoothness-indicator integrals IJI, ISI of rho and E at the face's
//          first gauss point (the reference integrates with LINE_1 weight 2 but
//          reads the LINE_3 data of point 0), one thread per face;
//   cell:  indicator si = sqrt(max_k IJI_k / ISI_k) * P^2 (P = 2), one thread per
//          cell, which lists the cells to limit;
//   limit: one thread per listed cell, order-by-order (P2 rows 2..4, then P1
//          rows 0..1) biway WBAP against each neighbour in characteristic space
//          and a multiway WBAP of the results, into a compact buffer that a last
//          pass scatters back over the listed cells' coefficients (the others
//          keep theirs: nothing is copied).
#pragma once
#include "dndsg_bodies.cuh"

namespace dg {

// per-face data of the limiting pass, tile-major AoSoA with E = kLimE (FP64):
//   [0, 25)   msR2L (right-cell coefficients -> left basis), row-major
//   [25, 50)  msL2R
// (the indicator's data is the compact limG / limCell below)
constexpr int kLimE = 50;
constexpr int kMsR2L = 0, kMsL2R = 25;
// the indicator's compact data, in the context's precision: per face (AoSoA E = kLimG) the frame
// coordinates (xi, eta) of gauss point 0 in the left and the right cell and the 6 face weights; per
// cell ([N][kLimCell]) the frame's Pinv (row-major) and basis moments.  D at the point follows from
// these (p2_diffs_at), a fifth of the bytes of storing it.
constexpr int kLimG = 10;
constexpr int kLimCell = 9;

struct LimView {
  int64_t N, F, Fi;
  int nfmax;
  const int32_t* cellFace;
  const int32_t* faceL;
  const int32_t* faceR;
  const double* faceNormal;
  const double* faceArea;
  const double* limFace;   // AoSoA kLimE
  const void* limG;        // T [F] AoSoA kLimG (T = the context's precision)
  const void* limCell;     // T [N][kLimCell]
  const double* u;
  double* faceInd;         // [F][4]: IJI_rho, IJI_E, ISI_rho, ISI_E
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
DG_HD bool setup_limiter_face(int64_t f, const MeshView& m, const SetupParams& p, const CellSetup* cells,
                              const double* faceW, double* lim) {
  int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
  for (int e = 0; e < kLimE; e++) lim[aos(f, e, kLimE)] = 0.0;
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
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) lim[aos(f, kMsR2L + i * 5 + j, kLimE)] = B[i][j];
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) { A[i][j] = DR[i + 1][j]; B[i][j] = DL[i + 1][j]; }
  ok = lu5_solve(A, B) && ok;
  for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) lim[aos(f, kMsL2R + i * 5 + j, kLimE)] = B[i][j];
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
  }
}

template <class T>
DG_HD void limiter_face_indicator(int64_t f, const LimView& v, const T* urec) {
  int32_t L = v.faceL[f], R = v.faceR[f];
  double* out = &v.faceInd[f * 4];
  if (R < 0) { out[0] = out[1] = out[2] = out[3] = 0; return; }
  // per side: the rows of the cell's basis derivatives at gauss point 0 (from the cell's frame) times
  // its rho and E coefficients, the mean added to the value row; one side's derivatives live at a time
  const T* g = static_cast<const T*>(v.limG);
  const T* cf = static_cast<const T*>(v.limCell);
  const int var[2] = {0, 3};
  double sv[2][6][2];
  for (int side = 0; side < 2; side++) {
    const int64_t cell = side ? R : L;
    const T* c = cf + cell * kLimCell;
    const double Q[2][2] = {{(double)c[0], (double)c[1]}, {(double)c[2], (double)c[3]}};
    const double mo[5] = {(double)c[4], (double)c[5], (double)c[6], (double)c[7], (double)c[8]};
    double D[6][5];
    p2_diffs_at(Q, mo, (double)g[aos(f, 2 * side, kLimG)], (double)g[aos(f, 2 * side + 1, kLimG)], D);
    for (int k = 0; k < 2; k++) {
      double r[5];
      for (int q = 0; q < 5; q++) r[q] = (double)urec[cell * 20 + q * 4 + var[k]];
      for (int d = 0; d < 6; d++) {
        double a = 0;
        for (int q = 0; q < 5; q++) a += D[d][q] * r[q];
        if (d == 0) a += v.u[cell * 4 + var[k]];
        sv[side][d][k] = a;
      }
    }
  }
  double val[6][2], jump[6][2];
  for (int c = 0; c < 2; c++)
    for (int d = 0; d < 6; d++) {
      val[d][c] = (sv[0][d][c] + sv[1][d][c]) * 0.5;
      jump[d][c] = (sv[0][d][c] - sv[1][d][c]) * 0.5;
    }
  double W[6];
  for (int k = 0; k < 6; k++) W[k] = (double)g[aos(f, 4 + k, kLimG)];
  const double area = v.faceArea[f];
  double sL = sqrt(v.vol[L]) / area, sR = sqrt(v.vol[R]) / area;
  double arMax = dmax(1.0, dmax(sL, sR));
  double tm = pow((1.0 / arMax) * (1 - v.tangModMin) + v.tangModMin, v.tangModPower);
  FaceFunctional Fn = make_functional(W, v.faceNormal[2 * f], v.faceNormal[2 * f + 1], v.tangWeight, tm, v.tangModLoc);
  double ij[2] = {0, 0}, is[2] = {0, 0};
  for (int a = 0; a < 6; a++)
    for (int c = 0; c < 2; c++) {
      double pj = 0, ps = 0;
      for (int r = 0; r < 6; r++) { pj += Fn.t[a][r] * jump[r][c]; ps += Fn.t[a][r] * val[r][c]; }
      ij[c] += pj * pj;
      is[c] += ps * ps;
    }
  // |n| of gauss point 0 is area/2, times the LINE_1 weight 2
  out[0] = ij[0] * area; out[1] = ij[1] * area; out[2] = is[0] * area; out[3] = is[1] * area;
}

// cell pass of the indicator: si = sqrt(max |IJI/ISI|) * P^2
DG_HD double limiter_cell_indicator(int64_t i, const LimView& v) {
  double sj[2] = {0, 0}, ss[2] = {0, 0};
  for (int k = 0; k < v.nfmax; k++) {
    int32_t sf = v.cellFace[aos(i, k, v.nfmax)];
    if (sf == kEmptySlot) continue;
    int32_t f = sf >= 0 ? sf : ~sf;
    const double* d = &v.faceInd[(int64_t)f * 4];
    sj[0] += d[0]; sj[1] += d[1]; ss[0] += d[2]; ss[1] += d[3];
  }
  double s0 = sj[0] / (ss[0] + kVerySmall), s1 = sj[1] / (ss[1] + kVerySmall);
  return sqrt(dmax(fabs(s0), fabs(s1))) * v.porder2;
}

// characteristic matrices at the face mean state (fML / fMR, DNDS_FV_EulerSolver.hpp:749-795)
DG_HD void char_matrices(double gamma, const double* UL, const double* UR, double nx, double ny, double Lm[4][4],
                         double Rm[4][4]) {
  double UC[4], r[4];
  for (int k = 0; k < 4; k++) UC[k] = (UL[k] + UR[k]) * 0.5;
  to_normal_frame(UC, nx, ny, r);
  double ir = 1.0 / r[0];
  double vx = r[1] * ir, vy = r[2] * ir, vs = vx * vx + vy * vy, p, a2, H;
  thermal(r[3], r[0], vs, gamma, p, a2, H);
  double a = sqrt(a2), gb = gamma - 1, sc = gb / (2 * a * a);
  double L0[4][4] = {{H + a / gb * (vx - a), -vx - a / gb, -vy, 1},
                     {-2 * H + 4 / gb * (a * a), vx * 2, vy * 2, -2},
                     {vy * (-2 * (a * a) / gb), 0, 2 * (a * a) / gb, 0},
                     {H - a / gb * (vx + a), -vx + a / gb, -vy, 1}};
  // L = L0 * diag(1, base^T) in the momentum block: columns 1,2 times [[nx, ny], [-ny, nx]]
  for (int i = 0; i < 4; i++) {
    double c1 = L0[i][1] * sc, c2 = L0[i][2] * sc;
    Lm[i][0] = L0[i][0] * sc;
    Lm[i][1] = c1 * nx - c2 * ny;
    Lm[i][2] = c1 * ny + c2 * nx;
    Lm[i][3] = L0[i][3] * sc;
  }
  double R0[4][4] = {{1, 1, 0, 1}, {vx - a, vx, 0, vx + a}, {vy, vy, 1, vy}, {H - vx * a, 0.5 * vs, vy, H + vx * a}};
  for (int j = 0; j < 4; j++) {
    Rm[0][j] = R0[0][j];
    Rm[1][j] = nx * R0[1][j] - ny * R0[2][j];
    Rm[2][j] = ny * R0[1][j] + nx * R0[2][j];
    Rm[3][j] = R0[3][j];
  }
}

DG_HD double signE(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

// FWBAP_L2_Biway(u1, u2, out, n) (DNDS_FV_Limiters.hpp:410-449), p = 4
DG_HD double wbap_biway(double u1, double u2, double n) {
  double frac = u1 / (fabs(u2) + 1e-12) * signE(u2);
  double th1 = frac * frac * frac, th2 = (frac * frac) * (frac * frac);
  return u1 * (n + th1) / (n + th2);
}

// limiting pass for one cell (one the indicator pass listed); writes its 20 limited coefficients to o
template <class T>
DG_HD void limiter_cell(int64_t i, const LimView& v, const T* urec, T* o) {
  const T* ri = &urec[i * 20];
  const double sm4 = 1e-50;  // verySmallReal^(1/4)
  double res[5][4];
  double uFaces[4][3][4];  // biway results of the P2 pass per face, this cell's basis
  const double* ui = &v.u[i * 4];
  for (int pass = 0; pass < 2; pass++) {
    const int ls = pass == 0 ? 2 : 0, nr = pass == 0 ? 3 : 2;
    double up[3][4], down[3][4];
    for (int r = 0; r < 3; r++) for (int c = 0; c < 4; c++) { up[r][c] = 0; down[r][c] = 0; }
    for (int k = 0; k < v.nfmax; k++) {
      int32_t sf = v.cellFace[aos(i, k, v.nfmax)];
      if (sf == kEmptySlot) continue;
      int32_t f = sf >= 0 ? sf : ~sf;
      int side = sf >= 0 ? 0 : 1;
      int32_t j = side == 0 ? v.faceR[f] : v.faceL[f];
      if (j < 0) continue;
      // ms: other -> this basis; msO: this -> other basis
      const int eMs = side == 0 ? kMsR2L : kMsL2R, eMsO = side == 0 ? kMsL2R : kMsR2L;
      double uOO[5][4];
      for (int q = 0; q < 5; q++) for (int c = 0; c < 4; c++) uOO[q][c] = (double)urec[(int64_t)j * 20 + q * 4 + c];
      if (pass == 1) {
        for (int q = 2; q < 5; q++)
          for (int c = 0; c < 4; c++) {
            double s = 0;
            for (int t = 2; t < 5; t++) s += v.limFace[aos(f, eMsO + q * 5 + t, kLimE)] * uFaces[k][t - 2][c];
            uOO[q][c] = s;
          }
      }
      double oin[3][4], tin[3][4];
      for (int r = 0; r < nr; r++)
        for (int c = 0; c < 4; c++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += v.limFace[aos(f, eMs + (ls + r) * 5 + q, kLimE)] * uOO[q][c];
          oin[r][c] = s;
          tin[r][c] = (double)ri[(ls + r) * 4 + c];
        }
      const double* uj = &v.u[(int64_t)j * 4];
      const double* uL = side ? uj : ui;
      const double* uR = side ? ui : uj;
      double Lm[4][4], Rm[4][4];
      char_matrices(v.gamma, uL, uR, v.faceNormal[2 * f], v.faceNormal[2 * f + 1], Lm, Rm);
      for (int r = 0; r < nr; r++) {
        double co[4], ct[4], lim[4];
        for (int a = 0; a < 4; a++) {
          double so = 0, st2 = 0;
          for (int q = 0; q < 4; q++) { so += Lm[a][q] * oin[r][q]; st2 += Lm[a][q] * tin[r][q]; }
          co[a] = so; ct[a] = st2;
        }
        for (int a = 0; a < 4; a++) lim[a] = wbap_biway(ct[a], co[a], 1.0);
        for (int a = 0; a < 4; a++) {
          double s = 0;
          for (int q = 0; q < 4; q++) s += Rm[a][q] * lim[q];
          if (pass == 0) uFaces[k][r][a] = s;
          // FWBAP_L2_Multiway accumulation against uOthers[0] = this cell's coefficients
          double u0 = (double)ri[(ls + r) * 4 + a];
          double ti = u0 / (fabs(s) + sm4) * signE(s);
          down[r][a] += (ti * ti) * (ti * ti);
          up[r][a] += ti * ti * ti;
        }
      }
    }
    for (int r = 0; r < nr; r++)
      for (int c = 0; c < 4; c++) {
        double u0 = (double)ri[(ls + r) * 4 + c];
        res[ls + r][c] = u0 * (up[r][c] + v.nStd) / (down[r][c] + v.nStd);
      }
  }
  for (int q = 0; q < 5; q++) for (int c = 0; c < 4; c++) o[q * 4 + c] = (T)res[q][c];
}

}  // namespace dg
