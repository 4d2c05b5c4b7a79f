/*
 * dnds_oracle.cpp -- FP64 CPU restatement of the DNDS residual-evaluation
 * path.  TEST INFRASTRUCTURE ONLY: the parity oracle and the timed CPU
 * baseline; never linked into the product.  See dnds_oracle.h for the list of
 * reference functions restated here and the deviations.
 */
#include "dnds_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr double kVerySmall = 1e-200;  // verySmallReal, DNDS_Defines.h:70
constexpr double kPi = 3.14159265358979323846;
constexpr int kNB = 5;   // P2 basis without the mean (NDOF-1)
constexpr int kND = 6;   // P2 diffs {1, x, y, xx, xy, yy}
constexpr int kMaxV = 6;

// diffOperatorOrderList2D (DNDS_Elements.hpp:469-480), P2 part
const int kDO[kND][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}};
// factorial / combination tables (DNDS_Elements.hpp:542-562)
const int kFact[5] = {1, 1, 2, 6, 24};
const int kNComb[kND] = {1, 1, 1, 1, 2, 1};
inline int dfact(int p, int d) {  // p!/(p-d)!, 0 when d > p
  if (d > p) return 0;
  int r = 1;
  for (int i = 0; i < d; i++) r *= (p - i);
  return r;
}
inline double sqr(double x) { return x * x; }
inline double ipow(double x, int n) {
  double r = 1;
  for (int i = 0; i < n; i++) r *= x;
  return r;
}
inline double signE(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }  // Eigen .sign()

enum BC { kInner = -1, kWall = 1, kFar = 2, kWallEuler = 3, kWallNoSlip = 4,
          kDMRFar = -2, kRTFar = -3, kIVFar = -4, kRiemannFar = -5 };
inline bool isFarType(int b) { return b == kFar || b == kDMRFar || b == kRTFar || b == kIVFar || b == kRiemannFar; }

// quadrature (DNDS_Elements.hpp:326-430): LINE_3, TRI_4, QUAD_9
struct Quad { int n; double p[9][2]; double w[9]; };
Quad line3() {
  Quad q{}; q.n = 3; double a = std::sqrt(0.6);
  q.p[0][0] = -a; q.p[1][0] = 0; q.p[2][0] = a;
  q.w[0] = 5. / 9.; q.w[1] = 8. / 9.; q.w[2] = 5. / 9.;
  return q;
}
Quad tri4() {
  Quad q{}; q.n = 4;
  double P[4][2] = {{1. / 3., 1. / 3.}, {0.6, 0.2}, {0.2, 0.6}, {0.2, 0.2}};
  double W[4] = {-27. / 96., 25. / 96., 25. / 96., 25. / 96.};
  for (int i = 0; i < 4; i++) { q.p[i][0] = P[i][0]; q.p[i][1] = P[i][1]; q.w[i] = W[i]; }
  return q;
}
Quad quad9() {
  Quad q{}; q.n = 9; Quad l = line3();
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) {
      q.p[j * 3 + i][0] = l.p[i][0]; q.p[j * 3 + i][1] = l.p[j][0];
      q.w[j * 3 + i] = l.w[i] * l.w[j];
    }
  return q;
}

// shape functions of Tri3 / Quad4 (DNDS_Elements.hpp:1020-1090): N and dN/dxi
void shape(int nn, double xi, double eta, double N[4], double dN[2][4]) {
  if (nn == 3) {
    N[0] = 1 - xi - eta; N[1] = xi; N[2] = eta;
    dN[0][0] = -1; dN[0][1] = 1; dN[0][2] = 0;
    dN[1][0] = -1; dN[1][1] = 0; dN[1][2] = 1;
  } else {
    N[0] = (1 - xi) * (1 - eta) * 0.25; N[1] = (1 + xi) * (1 - eta) * 0.25;
    N[2] = (1 + xi) * (1 + eta) * 0.25; N[3] = (1 - xi) * (1 + eta) * 0.25;
    dN[0][0] = -(1 - eta) * 0.25; dN[0][1] = (1 - eta) * 0.25; dN[0][2] = (1 + eta) * 0.25; dN[0][3] = -(1 + eta) * 0.25;
    dN[1][0] = -(1 - xi) * 0.25; dN[1][1] = -(1 + xi) * 0.25; dN[1][2] = (1 + xi) * 0.25; dN[1][3] = (1 - xi) * 0.25;
  }
}

void parallel_for(int nthreads, int64_t n, const std::function<void(int64_t, int64_t)>& f) {
  if (nthreads <= 1 || n < 1024) { f(0, n); return; }
  std::vector<std::thread> th;
  int64_t chunk = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; t++) {
    int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto& t : th) t.join();
}

struct CellGeo {
  int nn;
  double xy[4][2];
  double vol;
  double bary[2];
  double pcenter[2];   // cellCenters: image of the parametric centre
  double sscale[2];    // CoordMinMaxScale (half extents)
  double e[2][2];      // unit inertia eigenvectors, e[0] = largest eigenvalue
  double moment[kND];  // baseMoments
  int nface;
  int faces[4];
};

struct FaceGeo {
  int L, R, bc;
  double shift[2];
  double area;          // faceArea
  double center[2];     // faceCenters
  double ncenter[2];    // faceNormCenter (|n| = area/2)
  double gp[3][2];      // physical gauss points
  double n[3][2];       // faceNorms per gauss point
  double wq[3];         // LINE_3 weights
  double D[3][2][kND][kND];  // faceDiBjGauss[gp][side][diff][base]
  double Dc[2][kND][kND];    // faceDiBjCenter
  double weights[kND];       // faceWeights
  double msR2L[kNB][kNB], msL2R[kNB][kNB];  // matrixSecondary
};

}  // namespace

struct orc_ctx {
  orc_settings s{};
  int nv = 4;
  int64_t N = 0, F = 0;
  int nthreads = 1;
  std::vector<CellGeo> cg;
  std::vector<FaceGeo> fg;
  // VR operator blocks
  std::vector<double> Ainv;    // [N][5][5]
  std::vector<double> AinvB;   // [N][4][5][5]
  std::vector<double> Ainvb;   // [N][4][5]
  // state
  std::vector<double> u, urec, urecNew, urec1;
  std::vector<double> dtFace, lambdaFace, deltaLambdaFace, lambdaCell;
  std::vector<double> dtCell;
  std::vector<double> Dinv;      // LU-SGS diagonal inverse [N][nv] (diagonal per variable)
  std::vector<double> Dmat;      // the diagonal itself (jacobianCell, for LUSGSMatrixVec)
  std::vector<int32_t> lusgsPart;  // partition of every cell for the partitioned sweeps (empty: none)
  // dual time stepping: BDF history (prevStart / cnPrev as ImplicitBDFDualTimeStep) or SDIRK
  // stage right-hand sides
  std::vector<std::vector<double>> odeVec;
  int odeOrder = 0, odeCnPrev = 0, odePrevStart = 0;
  double odeDtPrev = 0;
  std::vector<double> dWall;     // SA: wall distance per cell (first-order, from the cell barycentre)
  std::vector<double> srcJac;    // SA: jacobianCellSourceDiag [N][nv] of the last RHS
  double lastInc = 0;
  std::string err;
};

namespace {

// ------------------------------------------------------------------ basis
// VRFiniteVolume2D::FDiffBaseValue (DNDS_FV_VR.hpp:300-1019) for P2 at a
// physical point (px,py); D[diff][base]; moment subtracted from row 0.
void diff_base_value(const orc_ctx& c, const CellGeo& g, double px, double py, const double* moment,
                     double D[kND][kND]) {
  const orc_settings& s = c.s;
  double cx = s.base_center_type == 0 ? g.bary[0] : g.pcenter[0];
  double cy = s.base_center_type == 0 ? g.bary[1] : g.pcenter[1];
  double dx = px - cx, dy = py - cy;
  if (!s.use_local_coord) {
    double sx = g.sscale[0], sy = g.sscale[1];
    if (!s.anisotropic_lengths) { double n = std::sqrt(sx * sx + sy * sy); sx = sy = n; }
    double xs = dx / sx, ys = dy / sy;
    for (int id = 0; id < kND; id++)
      for (int ib = 0; ib < kND; ib++) {
        int qx = kDO[ib][0], qy = kDO[ib][1], ndx = kDO[id][0], ndy = kDO[id][1];
        int cc = dfact(qx, ndx) * dfact(qy, ndy);
        D[id][ib] = cc ? cc * ipow(xs, qx - ndx) * ipow(ys, qy - ndy) / (ipow(sx, ndx) * ipow(sy, ndy)) : 0.0;
      }
  } else {
    // normalised inertia frame, scaled by the cell's half extents in that frame
    double P[2][2] = {{g.e[0][0], g.e[1][0]}, {g.e[0][1], g.e[1][1]}};  // columns e0, e1
    double det = P[0][0] * P[1][1] - P[0][1] * P[1][0];
    double iP[2][2] = {{P[1][1] / det, -P[0][1] / det}, {-P[1][0] / det, P[0][0] / det}};
    double mn[2] = {1e300, 1e300}, mx[2] = {-1e300, -1e300};
    for (int k = 0; k < g.nn; k++) {
      double rx = g.xy[k][0] - cx, ry = g.xy[k][1] - cy;
      for (int r = 0; r < 2; r++) {
        double v = iP[r][0] * rx + iP[r][1] * ry;
        mn[r] = std::min(mn[r], v); mx[r] = std::max(mx[r], v);
      }
    }
    double sL0 = (mx[0] - mn[0]) * 0.5, sL1 = (mx[1] - mn[1]) * 0.5;
    double su = std::sqrt(sL0 * sL0 + sL1 * sL1);
    double a0 = s.anisotropic_lengths ? sL0 : su, a1 = s.anisotropic_lengths ? sL1 : su;
    P[0][0] *= a0; P[1][0] *= a0; P[0][1] *= a1; P[1][1] *= a1;
    det = P[0][0] * P[1][1] - P[0][1] * P[1][0];
    iP[0][0] = P[1][1] / det; iP[0][1] = -P[0][1] / det; iP[1][0] = -P[1][0] / det; iP[1][1] = P[0][0] / det;
    double xi = iP[0][0] * dx + iP[0][1] * dy, eta = iP[1][0] * dx + iP[1][1] * dy;
    for (int id = 0; id < kND; id++)
      for (int ib = 0; ib < kND; ib++) {
        int qx = kDO[ib][0], qy = kDO[ib][1], ndx = kDO[id][0], ndy = kDO[id][1];
        int cc = dfact(qx, ndx) * dfact(qy, ndy);
        D[id][ib] = cc ? cc * ipow(xi, qx - ndx) * ipow(eta, qy - ndy) : 0.0;
      }
    // Convert2dDiffsLinMap(D, iP^T) (DNDS_Elements.hpp:1491-1528)
    double M[2][2] = {{iP[0][0], iP[1][0]}, {iP[0][1], iP[1][1]}};
    for (int ib = 0; ib < kND; ib++) {
      double h[2][2] = {{D[3][ib], D[4][ib]}, {D[4][ib], D[5][ib]}};
      double t[2][2], r[2][2];
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) t[i][j] = M[i][0] * h[0][j] + M[i][1] * h[1][j];
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) r[i][j] = t[i][0] * M[j][0] + t[i][1] * M[j][1];
      D[3][ib] = r[0][0]; D[4][ib] = r[0][1]; D[5][ib] = r[1][1];
      double g0 = D[1][ib], g1 = D[2][ib];
      D[1][ib] = M[0][0] * g0 + M[0][1] * g1;
      D[2][ib] = M[1][0] * g0 + M[1][1] * g1;
    }
  }
  if (moment)
    for (int ib = 0; ib < kND; ib++) D[0][ib] -= moment[ib];
}

// VRFiniteVolume2D::FFaceFunctional (DNDS_FV_VR.hpp:1021-1293), the 6-weight
// branch (P2) and the generic diagonal-weight branch.  DI is nd x ni, DJ nd x nj
// (row-major with leading dims ldI/ldJ); Conj is ni x nj.
void face_functional(const orc_ctx& c, const FaceGeo& f, int ig, const double* DI, int ni, int ldI,
                     const double* DJ, int nj, int ldJ, const double* W, int nw, double* Conj) {
  const orc_settings& s = c.s;
  const CellGeo& gL = c.cg[f.L];
  const CellGeo& gR = c.cg[f.R >= 0 ? f.R : f.L];
  double sigL = std::sqrt(gL.vol) / f.area, sigR = std::sqrt(gR.vol) / f.area;
  double arMax = std::max({1.0, sigL, sigR});
  double tangModifier = (1. / arMax) * (1 - s.tang_weight_mod_min) + s.tang_weight_mod_min;
  tangModifier = std::pow(tangModifier, s.tang_weight_mod_power);
  int loc = s.tang_weight_mod_loc;
  auto di = [&](int r, int i) { return DI[r * ldI + i]; };
  auto dj = [&](int r, int j) { return DJ[r * ldJ + j]; };
  if (nw == 6) {
    const double epsR = 1e-50;
    double w2r, length;
    if (std::fabs(W[1]) >= epsR || std::fabs(W[2]) >= epsR) {
      w2r = std::fabs(W[1]) >= std::fabs(W[2]) ? W[3] / (W[1] * W[1]) : W[5] / (W[2] * W[2]);
      length = std::sqrt(W[1] * W[1] + W[2] * W[2]);
    } else {
      w2r = 0.0; length = 0;
    }
    const double* nv = ig >= 0 ? f.n[ig] : f.ncenter;
    double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1]);
    double n0 = nv[0] / nn * length, n1 = nv[1] / nn * length;
    double tf = s.tang_weight * tangModifier * (loc == 1 ? tangModifier : 1);
    double t0 = -n1 * tf, t1 = n0 * tf;
    double tm2 = (loc == 0 ? sqr(tangModifier) : 1);
    for (int i = 0; i < ni; i++)
      for (int j = 0; j < nj; j++) {
        double v = di(0, i) * dj(0, j) * W[0] * W[0];
        double a, b;
        a = di(1, i) * n0 + di(2, i) * n1; b = dj(1, j) * n0 + dj(2, j) * n1; v += a * b;
        a = di(1, i) * t0 + di(2, i) * t1; b = dj(1, j) * t0 + dj(2, j) * t1; v += a * b * tm2;
        a = (di(3, i) * n0 * n0 + di(4, i) * n0 * n1 * 2 + di(5, i) * n1 * n1) * w2r;
        b = (dj(3, j) * n0 * n0 + dj(4, j) * n0 * n1 * 2 + dj(5, j) * n1 * n1) * w2r;
        v += a * b;
        // mixed term exactly as the reference writes it (n0*t1*2, DNDS_FV_VR.hpp:1254-1261)
        a = (di(3, i) * n0 * t0 + di(4, i) * n0 * t1 * 2 + di(5, i) * n1 * t1) * w2r;
        b = (dj(3, j) * n0 * t0 + dj(4, j) * n0 * t1 * 2 + dj(5, j) * n1 * t1) * w2r;
        v += a * b * 2 * tm2;
        a = (di(3, i) * t0 * t0 + di(4, i) * t0 * t1 * 2 + di(5, i) * t1 * t1) * w2r;
        b = (dj(3, j) * t0 * t0 + dj(4, j) * t0 * t1 * 2 + dj(5, j) * t1 * t1) * w2r;
        v += a * b * tm2;
        Conj[i * nj + j] = v;
      }
  } else {
    for (int i = 0; i < ni; i++)
      for (int j = 0; j < nj; j++) {
        double v = 0;
        for (int r = 0; r < nw; r++) v += di(r, i) * W[r] * W[r] * dj(r, j);
        Conj[i * nj + j] = v;
      }
  }
}

// pivoted Gauss-Jordan solve A X = B, A n x n, B n x m (in place -> X in B)
bool gj_solve(int n, double* A, int m, double* B) {
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (A[p * n + k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[k * n + j], A[p * n + j]);
      for (int j = 0; j < m; j++) std::swap(B[k * m + j], B[p * m + j]);
    }
    double inv = 1.0 / A[k * n + k];
    for (int j = 0; j < n; j++) A[k * n + j] *= inv;
    for (int j = 0; j < m; j++) B[k * m + j] *= inv;
    for (int i = 0; i < n; i++) {
      if (i == k) continue;
      double fct = A[i * n + k];
      if (fct == 0.0) continue;
      for (int j = 0; j < n; j++) A[i * n + j] -= fct * A[k * n + j];
      for (int j = 0; j < m; j++) B[i * m + j] -= fct * B[k * m + j];
    }
  }
  return true;
}

// ------------------------------------------------------------------ gas
// Gas::IdealGasThermal (DNDS_Gas.hpp:73-79)
inline void thermal(double E, double rho, double vsqr, double gamma, double& p, double& asqr, double& H) {
  p = (gamma - 1) * (E - rho * 0.5 * vsqr);
  asqr = gamma * p / rho;
  H = (E + p) / rho;
}
// Gas::GasInviscidFlux, x direction (DNDS_Gas.hpp:113-119)
inline void inviscid_flux(const double* U, double vx, double p, double* F) {
  for (int k = 0; k < 4; k++) F[k] = U[k] * vx;
  F[1] += p;
  F[3] += vx * p;
}

// Gas::RoeFlux_IdealGas_HartenYee<2,0> (DNDS_Gas.hpp:406-654)
void roe_flux(const double* UL, const double* UR, double gamma, double* F, double dLambda) {
  const double scaleHartenYee = 0.05;
  double vL[2] = {UL[1] / UL[0], UL[2] / UL[0]}, vR[2] = {UR[1] / UR[0], UR[2] / UR[0]};
  double aL2, aR2, pL, pR, HL, HR;
  double vsL = vL[0] * vL[0] + vL[1] * vL[1], vsR = vR[0] * vR[0] + vR[1] * vR[1];
  thermal(UL[3], UL[0], vsL, gamma, pL, aL2, HL);
  thermal(UR[3], UR[0], vsR, gamma, pR, aR2, HR);
  double sL = std::sqrt(UL[0]), sR = std::sqrt(UR[0]);
  double vRoe[2] = {(sL * vL[0] + sR * vR[0]) / (sL + sR), (sL * vL[1] + sR * vR[1]) / (sL + sR)};
  double vsRoe = vRoe[0] * vRoe[0] + vRoe[1] * vRoe[1];
  double HRoe = (sL * HL + sR * HR) / (sL + sR);
  double a2Roe = (gamma - 1) * (HRoe - 0.5 * vsRoe);
  double FL[4], FR[4];
  inviscid_flux(UL, vL[0], pL, FL);
  inviscid_flux(UR, vR[0], pR, FR);
  double aRoe = std::sqrt(a2Roe);
  double lam0 = std::fabs(vRoe[0] - aRoe), lam123 = std::fabs(vRoe[0]), lam4 = std::fabs(vRoe[0] + aRoe);
  double thr = std::max(scaleHartenYee * (std::sqrt(vsRoe) + aRoe), dLambda);
  double thrS = thr * thr;
  if (lam0 < thr) lam0 = (sqr(lam0) + thrS) / (2 * thr);
  if (lam4 < thr) lam4 = (sqr(lam4) + thrS) / (2 * thr);
  double lam[4] = {lam0, lam123, lam123, lam4};
  // right eigenvectors (DNDS_Gas.hpp:17-37), dim = 2
  double Rv[4][4] = {{1, 1, 0, 1},
                     {vRoe[0] - aRoe, vRoe[0], 0, vRoe[0] + aRoe},
                     {vRoe[1], vRoe[1], 1, vRoe[1]},
                     {HRoe - vRoe[0] * aRoe, 0.5 * vsRoe, vRoe[1], HRoe + vRoe[0] * aRoe}};
  double dU[4];
  for (int k = 0; k < 4; k++) dU[k] = UR[k] - UL[k];
  double alpha[4];
  alpha[2] = dU[2] - vRoe[1] * dU[0];
  double dU4b = dU[3] - alpha[2] * vRoe[1];
  alpha[1] = (gamma - 1) / a2Roe * (dU[0] * (HRoe - vRoe[0] * vRoe[0]) + vRoe[0] * dU[1] - dU4b);
  alpha[0] = (dU[0] * (vRoe[0] + aRoe) - dU[1] - aRoe * alpha[1]) / (2 * aRoe);
  alpha[3] = dU[0] - (alpha[0] + alpha[1]);
  for (int r = 0; r < 4; r++) {
    double inc = 0;
    for (int k = 0; k < 4; k++) inc += Rv[r][k] * (lam[k] * alpha[k]);
    F[r] = (FL[r] + FR[r]) * 0.5 - 0.5 * inc;
  }
}

// Gas::HLLCFlux_IdealGas_HartenYee<2> (DNDS_Gas.hpp:312-403)
void hllc_flux(const double* UL, const double* UR, double gamma, double* F) {
  double vL[2] = {UL[1] / UL[0], UL[2] / UL[0]}, vR[2] = {UR[1] / UR[0], UR[2] / UR[0]};
  double aL2, aR2, pL, pR, HL, HR;
  thermal(UL[3], UL[0], vL[0] * vL[0] + vL[1] * vL[1], gamma, pL, aL2, HL);
  thermal(UR[3], UR[0], vR[0] * vR[0] + vR[1] * vR[1], gamma, pR, aR2, HR);
  double sL = std::sqrt(UL[0]), sR = std::sqrt(UR[0]);
  double vRoe0 = (sL * vL[0] + sR * vR[0]) / (sL + sR);
  double eta2 = 0.5 * (sL * sR) / sqr(sL + sR);
  double dsqr = (aL2 * sL + aR2 * sR) / (sL + sR) + eta2 * sqr(vR[0] - vL[0]);
  double SL = vRoe0 - std::sqrt(dsqr), SR = vRoe0 + std::sqrt(dsqr);
  double FL[4], FR[4];
  inviscid_flux(UL, vL[0], pL, FL);
  inviscid_flux(UR, vR[0], pR, FR);
  if (0 <= SL) { for (int k = 0; k < 4; k++) F[k] = FL[k]; return; }
  if (SR <= 0) { for (int k = 0; k < 4; k++) F[k] = FR[k]; return; }
  double SS = 0;
  double div = (UL[0] * (SL - vL[0]) - UR[0] * (SR - vR[0]));
  if (std::fabs(div) > kVerySmall) SS = (pR - pL + UL[1] * (SL - vL[0]) - UR[1] * (SR - vR[0])) / div;
  double DS[4] = {0, 1, 0, SS};
  if (SS >= 0) {
    double d = SL - SS;
    if (std::fabs(d) < kVerySmall) { for (int k = 0; k < 4; k++) F[k] = FL[k]; }
    else {
      double sc = (pL + UL[0] * (SL - vL[0]) * (SS - vL[0])) * SL;
      for (int k = 0; k < 4; k++) F[k] = ((UL[k] * SL - FL[k]) * SS + DS[k] * sc) / d;
    }
  } else {
    double d = SR - SS;
    if (std::fabs(d) < kVerySmall) { for (int k = 0; k < 4; k++) F[k] = FR[k]; }
    else {
      double sc = (pR + UR[0] * (SR - vR[0]) * (SS - vR[0])) * SR;
      for (int k = 0; k < 4; k++) F[k] = ((UR[k] * SR - FR[k]) * SS + DS[k] * sc) / d;
    }
  }
}

// conservative <-> primitive (DNDS_Gas.hpp:81-111), dim = 2
inline void cons2prim(const double* U, double* W, double gamma) {
  double vs = sqr(U[1] / U[0]) + sqr(U[2] / U[0]);
  W[0] = U[0]; W[1] = U[1] / U[0]; W[2] = U[2] / U[0];
  W[3] = (gamma - 1) * (U[3] - U[0] * 0.5 * vs);
}
inline void prim2cons(const double* W, double* U, double gamma) {
  double vs = W[1] * W[1] + W[2] * W[2];
  U[0] = W[0]; U[1] = W[1] * W[0]; U[2] = W[2] * W[0];
  U[3] = W[3] / (gamma - 1) + W[0] * 0.5 * vs;
}

// isentropic vortex state (DNDS_FV_EulerSolver.hpp:536-582 and
// DNDS_FV_EulerEvaluator.hpp:1100-1125); taper=true adds the rm=8 taper
void vortex_state(double x, double y, double xc, double yc, double gamma, bool taper, double* U) {
  double chi = 5, rm = 8;
  double r = std::sqrt(sqr(x - xc) + sqr(y - yc));
  double tp = taper ? (1 - 1. / std::exp(std::max(sqr(rm) - sqr(r), 0.0))) : 1.0;
  double dT = -(gamma - 1) / (8 * gamma * sqr(kPi)) * sqr(chi) * std::exp(1 - sqr(r)) * tp;
  double dux = chi / 2 / kPi * std::exp((1 - sqr(r)) / 2) * -(y - yc) * tp;
  double duy = chi / 2 / kPi * std::exp((1 - sqr(r)) / 2) * +(x - xc) * tp;
  double T = dT + 1, ux = dux + 1, uy = duy + 1;
  double rho = std::pow(T, 1 / (gamma - 1));
  double p = T * rho;
  U[0] = rho; U[1] = rho * ux; U[2] = rho * uy;
  U[3] = 0.5 * (sqr(ux) + sqr(uy)) * rho + p / (gamma - 1);
}

// EulerEvaluator::generateBoundaryValue (DNDS_FV_EulerEvaluator.hpp:958-1275)
// for the 2-D Euler model and, with c.nv = 5, the SA variable (a passive scalar: its primitive is
// U5 / rho, DNDS_Gas.hpp:82-107); un = unit normal, pc = face centre.  fixUL: at a no-slip wall the
// SA variable of both states is set to zero, UL included (USE_FIX_ZERO_SA_NUT_AT_WALL)
void boundary_value(const orc_ctx& c, double* UL, const double* un, const double* pc, double t,
                    int bc, double* UR, bool fixUL = false) {
  const double gamma = c.s.gamma;
  const int nv = c.nv;
  for (int k = 4; k < nv; k++) UR[k] = UL[k];
  if (bc == kFar) {
    const double* far = c.s.far_field;
    double vn = (UL[1] * un[0] + UL[2] * un[1]) / UL[0];
    double vs = sqr(UL[1] / UL[0]) + sqr(UL[2] / UL[0]);
    double p, a2, H;
    thermal(UL[3], UL[0], vs, gamma, p, a2, H);
    double a = std::sqrt(a2);
    if (vn - a > 0) { for (int k = 0; k < nv; k++) UR[k] = UL[k]; }
    else if (vn > 0) {
      double fp[4], lp[4];
      cons2prim(far, fp, gamma); cons2prim(UL, lp, gamma);
      lp[3] = fp[3];
      prim2cons(lp, UR, gamma);
    } else if (vn + a > 0) {
      double fp[4], lp[4];
      cons2prim(far, fp, gamma); cons2prim(UL, lp, gamma);
      fp[3] = lp[3];
      prim2cons(fp, UR, gamma);
      for (int k = 4; k < nv; k++) UR[k] = far[k];  // far primitive U5/rho times the far density
    } else {
      for (int k = 0; k < nv; k++) UR[k] = far[k];
    }
  } else if (bc == kIVFar) {
    vortex_state(pc[0], pc[1], 5 + t, 5 + t, gamma, false, UR);
  } else if (bc == kRiemannFar) {
    const double phi1 = -0.663324958071080, phi2 = -0.422115882408869, loc = 0.8;
    double p1 = loc + phi1 * t, p2 = loc + phi2 * t;
    double lp[4];
    cons2prim(UL, lp, gamma);
    double W[4] = {lp[0], lp[1], lp[2], lp[3]};
    const double bTol = 1e-9;
    if (std::fabs(pc[0] - 0.0) < bTol) {
      if (pc[1] <= p2) { W[0] = 0.137992831541219; W[1] = 1.206045378311055; W[2] = 1.206045378311055; W[3] = 0.029032258064516; }
      else { W[0] = 0.532258064516129; W[1] = 1.206045378311055; W[2] = 0.0; W[3] = 0.3; }
    } else if (std::fabs(pc[0] - 1.0) < bTol) {
      W[0] = lp[0]; W[1] = -lp[1]; W[2] = lp[2]; W[3] = lp[3];
    } else if (std::fabs(pc[1] - 1.0) < bTol) {
      W[0] = lp[0]; W[1] = lp[1]; W[2] = -lp[2]; W[3] = lp[3];
    } else if (std::fabs(pc[1] - 0.0) < bTol) {
      if (pc[0] <= p2) { W[0] = 0.137992831541219; W[1] = 1.206045378311055; W[2] = 1.206045378311055; W[3] = 0.029032258064516; }
      else { W[0] = 0.532258064516129; W[1] = 0.0; W[2] = 1.206045378311055; W[3] = 0.3; }
    } else {
      W[0] = W[1] = W[2] = W[3] = std::nan("");
    }
    (void)p1;
    prim2cons(W, UR, gamma);
  } else if (bc == kWallEuler) {
    for (int k = 0; k < 4; k++) UR[k] = UL[k];
    double d = UR[1] * un[0] + UR[2] * un[1];
    UR[1] -= d * un[0]; UR[2] -= d * un[1];
  } else if (bc == kWallNoSlip) {
    UR[0] = UL[0]; UR[1] = -UL[1]; UR[2] = -UL[2]; UR[3] = UL[3];
    if (nv > 4) {
      UR[4] = -UL[4];
      if (fixUL) UL[4] = UR[4] = 0;
    }
  } else {
    for (int k = 0; k < 4; k++) UR[k] = std::nan("");
  }
}

// EulerEvaluator::CompressRecPart (DNDS_FV_EulerEvaluator.hpp:1277-1360)
inline void compress_rec_part(const double* umean, const double* inc, double* ret, bool& compressed, int nv = 4) {
  for (int k = 0; k < nv; k++) ret[k] = umean[k] + inc[k];
  if (ret[0] < 0) { for (int k = 0; k < nv; k++) ret[k] = umean[k]; compressed = true; }
  double eK = (ret[1] * ret[1] + ret[2] * ret[2]) * 0.5 / (kVerySmall + ret[0]);
  double e = ret[3] - eK;
  if (e < 0) { for (int k = 0; k < nv; k++) ret[k] = umean[k]; compressed = true; }
}

// ------------------------------------------------------------------ setup
// A cell's faces in element-local face order, the order of the reference's cell2face (vol2face is
// filled per local face iface, DNDS_Mesh.hpp:288-320): face k joins nodes k and k+1 (FaceNodeList of
// TRI3 / QUAD4, DNDS_Elements.hpp:248-253).  A face is matched by its node pair, or -- a periodic face
// seen from its translated side -- by its midpoint against the edge midpoint moved by the face shift.
// Sums over a cell's faces run in this order, and V2's multiway WBAP is centred on the first face.
void order_cell_faces(const orc_mesh& m, int64_t i, int* faces, int nf) {
  const int nn = m.cell_nodes[4 * i + 3] < 0 ? 3 : 4;
  if (nf != nn) return;
  int out[4] = {-1, -1, -1, -1};
  bool used[4] = {false, false, false, false};
  for (int pass = 0; pass < 2; pass++)
    for (int e = 0; e < nn; e++) {
      if (out[e] >= 0) continue;
      const int p = m.cell_nodes[4 * i + e], q = m.cell_nodes[4 * i + (e + 1) % nn];
      const double mx = 0.5 * (m.node_xy[2 * p] + m.node_xy[2 * q]), my = 0.5 * (m.node_xy[2 * p + 1] + m.node_xy[2 * q + 1]);
      const double len = std::hypot(m.node_xy[2 * q] - m.node_xy[2 * p], m.node_xy[2 * q + 1] - m.node_xy[2 * p + 1]);
      for (int k = 0; k < nf && out[e] < 0; k++) {
        if (used[k]) continue;
        const int f = faces[k], a = m.face_nodes[2 * f], b = m.face_nodes[2 * f + 1];
        bool hit = (a == p && b == q) || (a == q && b == p);
        if (!hit && pass == 1 && m.face_shift) {
          const double fx = 0.5 * (m.node_xy[2 * a] + m.node_xy[2 * b]), fy = 0.5 * (m.node_xy[2 * a + 1] + m.node_xy[2 * b + 1]);
          const double sx = m.face_shift[2 * f], sy = m.face_shift[2 * f + 1];
          for (int sg = -1; sg <= 1 && !hit; sg += 2)
            hit = std::fabs(mx + sg * sx - fx) + std::fabs(my + sg * sy - fy) < 1e-9 * len;
        }
        if (hit) { out[e] = f; used[k] = true; }
      }
    }
  for (int e = 0; e < nn; e++)
    if (out[e] < 0) return;  // unmatched: keep the given order
  for (int e = 0; e < nn; e++) faces[e] = out[e];
}

int setup(orc_ctx& c, const orc_mesh& m) {
  const orc_settings& s = c.s;
  c.N = m.n_cells; c.F = m.n_faces;
  c.cg.resize(c.N);
  c.fg.resize(c.F);
  Quad q3 = tri4(), q4 = quad9(), ql = line3();
  for (int64_t i = 0; i < c.N; i++) { c.cg[i].nface = 0; }
  for (int64_t f = 0; f < c.F; f++) {
    int L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
    if (L < 0 || L >= c.N || R >= c.N) { c.err = "bad face_cells"; return 1; }
    if (c.cg[L].nface >= 4) { c.err = "cell with >4 faces"; return 1; }
    c.cg[L].faces[c.cg[L].nface++] = (int)f;
    if (R >= 0) {
      if (c.cg[R].nface >= 4) { c.err = "cell with >4 faces"; return 1; }
      c.cg[R].faces[c.cg[R].nface++] = (int)f;
    }
  }
  for (int64_t i = 0; i < c.N; i++) order_cell_faces(m, i, c.cg[i].faces, c.cg[i].nface);
  // --- cells: ImplicitFiniteVolume2D volumes, initMoment (DNDS_FV_VR.cpp:82-181)
  int bad = 0;
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      CellGeo& g = c.cg[i];
      g.nn = m.cell_nodes[4 * i + 3] < 0 ? 3 : 4;
      for (int k = 0; k < g.nn; k++) {
        int nd = m.cell_nodes[4 * i + k];
        g.xy[k][0] = m.node_xy[2 * nd]; g.xy[k][1] = m.node_xy[2 * nd + 1];
      }
      if (g.nface != g.nn) bad = 1;
      const Quad& q = g.nn == 3 ? q3 : q4;
      double N[4], dN[2][4];
      // parametric centre
      shape(g.nn, g.nn == 3 ? 1. / 3. : 0., g.nn == 3 ? 1. / 3. : 0., N, dN);
      g.pcenter[0] = g.pcenter[1] = 0;
      for (int k = 0; k < g.nn; k++) { g.pcenter[0] += N[k] * g.xy[k][0]; g.pcenter[1] += N[k] * g.xy[k][1]; }
      double mnx = 1e300, mxx = -1e300, mny = 1e300, mxy = -1e300;
      for (int k = 0; k < g.nn; k++) {
        mnx = std::min(mnx, g.xy[k][0]); mxx = std::max(mxx, g.xy[k][0]);
        mny = std::min(mny, g.xy[k][1]); mxy = std::max(mxy, g.xy[k][1]);
      }
      g.sscale[0] = (mxx - mnx) * 0.5; g.sscale[1] = (mxy - mny) * 0.5;
      // gauss data
      double gx[9][2], gdet[9];
      for (int ig = 0; ig < q.n; ig++) {
        shape(g.nn, q.p[ig][0], q.p[ig][1], N, dN);
        double x = 0, y = 0, J[2][2] = {{0, 0}, {0, 0}};
        for (int k = 0; k < g.nn; k++) {
          x += N[k] * g.xy[k][0]; y += N[k] * g.xy[k][1];
          for (int d = 0; d < 2; d++) { J[d][0] += dN[d][k] * g.xy[k][0]; J[d][1] += dN[d][k] * g.xy[k][1]; }
        }
        gx[ig][0] = x; gx[ig][1] = y;
        gdet[ig] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        if (gdet[ig] <= 0) bad = 2;
      }
      g.vol = 0;
      for (int ig = 0; ig < q.n; ig++) g.vol += gdet[ig] * q.w[ig];
      g.bary[0] = g.bary[1] = 0;
      for (int ig = 0; ig < q.n; ig++) {
        g.bary[0] += gx[ig][0] * gdet[ig] * q.w[ig];
        g.bary[1] += gx[ig][1] * gdet[ig] * q.w[ig];
      }
      g.bary[0] /= g.vol; g.bary[1] /= g.vol;
      double I[2][2] = {{0, 0}, {0, 0}};
      for (int ig = 0; ig < q.n; ig++) {
        double rx = gx[ig][0] - g.bary[0], ry = gx[ig][1] - g.bary[1];
        double w = gdet[ig] * q.w[ig];
        I[0][0] += rx * rx * w; I[0][1] += rx * ry * w; I[1][1] += ry * ry * w;
      }
      I[0][0] /= g.vol; I[0][1] /= g.vol; I[1][1] /= g.vol; I[1][0] = I[0][1];
      // eigen frame of the inertia (HardEigen::Eigen3x3RealSymEigenDecomposition, largest first)
      double a = I[0][0], bb = I[0][1], cc = I[1][1];
      double hm = 0.5 * (a + cc), hd = 0.5 * (a - cc);
      double rr = std::sqrt(hd * hd + bb * bb);
      double lmax = hm + rr;
      if (rr <= 1e-14 * std::fabs(hm)) {
        g.e[0][0] = 1; g.e[0][1] = 0; g.e[1][0] = 0; g.e[1][1] = 1;
      } else {
        double vx, vy;
        if (a >= cc) { vx = lmax - cc; vy = bb; } else { vx = bb; vy = lmax - a; }
        double nrm = std::sqrt(vx * vx + vy * vy);
        vx /= nrm; vy /= nrm;
        g.e[0][0] = vx; g.e[0][1] = vy; g.e[1][0] = -vy; g.e[1][1] = vx;
      }
      // base moments
      double mom[kND] = {0, 0, 0, 0, 0, 0};
      for (int ig = 0; ig < q.n; ig++) {
        double D[kND][kND];
        diff_base_value(c, g, gx[ig][0], gx[ig][1], nullptr, D);
        for (int ib = 0; ib < kND; ib++) mom[ib] += D[0][ib] * gdet[ig] * q.w[ig];
      }
      for (int ib = 0; ib < kND; ib++) g.moment[ib] = mom[ib] / g.vol;
      g.moment[0] = 1.;
    }
  });
  if (bad == 1) { c.err = "cell face count does not match its node count"; return 1; }
  if (bad == 2) { c.err = "non-positive cell jacobian (cell not counter-clockwise?)"; return 1; }

  // --- faces: initBaseDiffCache face part (DNDS_FV_VR.cpp:367-890)
  parallel_for(c.nthreads, c.F, [&](int64_t b, int64_t e) {
    for (int64_t f = b; f < e; f++) {
      FaceGeo& fg = c.fg[f];
      fg.L = m.face_cells[2 * f]; fg.R = m.face_cells[2 * f + 1]; fg.bc = m.face_bc[f];
      fg.shift[0] = m.face_shift ? m.face_shift[2 * f] : 0.0;
      fg.shift[1] = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
      int n0 = m.face_nodes[2 * f], n1 = m.face_nodes[2 * f + 1];
      double x0 = m.node_xy[2 * n0], y0 = m.node_xy[2 * n0 + 1], x1 = m.node_xy[2 * n1], y1 = m.node_xy[2 * n1 + 1];
      // Line2 jacobian: d(x,y)/dxi = (p1-p0)/2; normal (J01, -J00) (DNDS_Elements.hpp:1453-1461)
      double jx = (x1 - x0) * 0.5, jy = (y1 - y0) * 0.5;
      fg.ncenter[0] = jy; fg.ncenter[1] = -jx;
      fg.area = 0;
      fg.center[0] = (x0 + x1) * 0.5; fg.center[1] = (y0 + y1) * 0.5;
      for (int ig = 0; ig < 3; ig++) {
        double xi = ql.p[ig][0];
        fg.gp[ig][0] = x0 * (1 - xi) * 0.5 + x1 * (1 + xi) * 0.5;
        fg.gp[ig][1] = y0 * (1 - xi) * 0.5 + y1 * (1 + xi) * 0.5;
        fg.n[ig][0] = jy; fg.n[ig][1] = -jx;
        fg.wq[ig] = ql.w[ig];
      }
      // face length (ImplicitFiniteVolume2D, LINE_5 of a constant integrand)
      fg.area = 2.0 * std::sqrt(jx * jx + jy * jy);
      const CellGeo& gL = c.cg[fg.L];
      for (int ig = 0; ig < 3; ig++) {
        diff_base_value(c, gL, fg.gp[ig][0], fg.gp[ig][1], gL.moment, fg.D[ig][0]);
        if (fg.R >= 0) {
          const CellGeo& gR = c.cg[fg.R];
          diff_base_value(c, gR, fg.gp[ig][0] - fg.shift[0], fg.gp[ig][1] - fg.shift[1], gR.moment, fg.D[ig][1]);
        } else {
          std::memset(fg.D[ig][1], 0, sizeof(fg.D[ig][1]));
        }
      }
      diff_base_value(c, gL, fg.center[0], fg.center[1], gL.moment, fg.Dc[0]);
      if (fg.R >= 0) {
        const CellGeo& gR = c.cg[fg.R];
        diff_base_value(c, gR, fg.center[0] - fg.shift[0], fg.center[1] - fg.shift[1], gR.moment, fg.Dc[1]);
        // matrixSecondary: least squares DL X = DR (square, full rank -> exact solve)
        double A[25], B[25];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) { A[i * 5 + j] = fg.Dc[0][i + 1][j + 1]; B[i * 5 + j] = fg.Dc[1][i + 1][j + 1]; }
        gj_solve(5, A, 5, B);
        for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) fg.msR2L[i][j] = B[i * 5 + j];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) { A[i * 5 + j] = fg.Dc[1][i + 1][j + 1]; B[i * 5 + j] = fg.Dc[0][i + 1][j + 1]; }
        gj_solve(5, A, 5, B);
        for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) fg.msL2R[i][j] = B[i * 5 + j];
      } else {
        std::memset(fg.Dc[1], 0, sizeof(fg.Dc[1]));
        std::memset(fg.msR2L, 0, sizeof(fg.msR2L));
        std::memset(fg.msL2R, 0, sizeof(fg.msL2R));
      }
      // weights (DNDS_FV_VR.cpp:716-888)
      double delta[2];
      for (int k = 0; k < kND; k++) fg.weights[k] = 1.0;
      if (fg.R >= 0) {
        const CellGeo& gR = c.cg[fg.R];
        delta[0] = gR.bary[0] + fg.shift[0] - gL.bary[0];
        delta[1] = gR.bary[1] + fg.shift[1] - gL.bary[1];
      } else {
        for (int k = 0; k < kND; k++) fg.weights[k] = 0.0;
        delta[0] = fg.center[0] - gL.bary[0];
        delta[1] = fg.center[1] - gL.bary[1];
        if (fg.bc == kWall || fg.bc == kWallEuler) fg.weights[0] = s.wall_weight;
        else if (isFarType(fg.bc)) fg.weights[0] = s.far_weight;
        else if (fg.bc == kWallNoSlip) {
          fg.weights[0] = s.wall_weight;
          // USE_FIRST_ORDER_VISCOUS_WALL_DELTA_IN_VR_WEIGHT
          double nn = std::sqrt(sqr(fg.ncenter[0]) + sqr(fg.ncenter[1]));
          double nx = fg.ncenter[0] / nn, ny = fg.ncenter[1] / nn;
          double d = nx * delta[0] + ny * delta[1];
          delta[0] = nx * d; delta[1] = ny * d;
        }
      }
      double D = std::sqrt(sqr(delta[0]) + sqr(delta[1]));
      double S = fg.area;
      double GW = 1;
      switch (s.weight_scheme_geom) {
        case 0: break;
        case 1: GW = std::pow(1. / D, 0.5); break;
        case 2: GW = std::pow(1. / S, 0.5); break;
        case 3: GW = std::pow(S / D, 0.5 / 2); break;
      }
      if (s.tang_weight_direction == 0) {
        double nn = std::sqrt(sqr(fg.ncenter[0]) + sqr(fg.ncenter[1]));
        delta[0] = fg.ncenter[0] / nn * D; delta[1] = fg.ncenter[1] / nn * D;
      }
      delta[0] *= s.weight_len_scale; delta[1] *= s.weight_len_scale;
      const double hqm2[3] = {1, 0.4643, 0.1559};
      for (int id = 0; id < kND; id++) {
        int ndx = kDO[id][0], ndy = kDO[id][1];
        if (s.weight_scheme_dir == 0)
          fg.weights[id] *= GW * std::pow(delta[0], ndx) * std::pow(delta[1], ndy) * double(kNComb[id]) /
                            double(kFact[ndx + ndy]);
        else
          fg.weights[id] *= GW * std::pow(delta[0], ndx) * std::pow(delta[1], ndy) * 1 * hqm2[ndx + ndy];
      }
    }
  });

  // --- per-cell matrices: initReconstructionMatVec (DNDS_FV_VR.cpp:892-1154)
  c.Ainv.assign(c.N * 25, 0.0);
  c.AinvB.assign(c.N * 100, 0.0);
  c.Ainvb.assign(c.N * 20, 0.0);
  int singular = 0;
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      const CellGeo& g = c.cg[i];
      double A[25] = {0};
      for (int k = 0; k < g.nface; k++) {
        const FaceGeo& f = c.fg[g.faces[k]];
        int side = f.L == i ? 0 : 1;
        for (int ig = 0; ig < 3; ig++) {
          double conj[36];
          face_functional(c, f, ig, &f.D[ig][side][0][0], 6, 6, &f.D[ig][side][0][0], 6, 6, f.weights, 6, conj);
          double nn = std::sqrt(sqr(f.n[ig][0]) + sqr(f.n[ig][1]));
          for (int r = 0; r < 5; r++)
            for (int q = 0; q < 5; q++) A[r * 5 + q] += conj[(r + 1) * 6 + q + 1] * nn * f.wq[ig];
        }
      }
      double Acp[25], Ai[25];
      for (int k = 0; k < 25; k++) Acp[k] = A[k];
      for (int r = 0; r < 5; r++) for (int q = 0; q < 5; q++) Ai[r * 5 + q] = r == q ? 1.0 : 0.0;
      if (!gj_solve(5, Acp, 5, Ai)) singular = 1;
      for (int k = 0; k < 25; k++) c.Ainv[i * 25 + k] = Ai[k];
      double brow[4][5];
      for (int k = 0; k < g.nface; k++) {
        const FaceGeo& f = c.fg[g.faces[k]];
        int side = f.L == i ? 0 : 1;
        double B[25] = {0};
        bool hasB = false;
        if (f.R >= 0) {
          hasB = true;
          for (int ig = 0; ig < 3; ig++) {
            double conj[36];
            face_functional(c, f, ig, &f.D[ig][side][0][0], 6, 6, &f.D[ig][1 - side][0][0], 6, 6, f.weights, 6, conj);
            double nn = std::sqrt(sqr(f.n[ig][0]) + sqr(f.n[ig][1]));
            for (int r = 0; r < 5; r++)
              for (int q = 0; q < 5; q++) B[r * 5 + q] += conj[(r + 1) * 6 + q + 1] * nn * f.wq[ig];
          }
        } else if (isFarType(f.bc)) {
          hasB = true;
          for (int ig = 0; ig < 3; ig++) {
            double conj[36];
            face_functional(c, f, ig, &f.D[ig][0][0][0], 6, 6, &f.D[ig][0][0][0], 6, 6, f.weights, 6, conj);
            double nn = std::sqrt(sqr(f.n[ig][0]) + sqr(f.n[ig][1]));
            for (int r = 0; r < 5; r++)
              for (int q = 0; q < 5; q++) B[r * 5 + q] += conj[(r + 1) * 6 + q + 1] * nn * f.wq[ig];
          }
        }
        double* out = &c.AinvB[(i * 4 + k) * 25];
        if (hasB)
          for (int r = 0; r < 5; r++)
            for (int q = 0; q < 5; q++) {
              double v = 0;
              for (int t = 0; t < 5; t++) v += Ai[r * 5 + t] * B[t * 5 + q];
              out[r * 5 + q] = v;
            }
        // b row: FFaceFunctional(Ones(1,1), rowDiffI, w0)
        for (int q = 0; q < 5; q++) brow[k][q] = 0;
        for (int ig = 0; ig < 3; ig++) {
          double one = 1.0, conj[6];
          face_functional(c, f, ig, &one, 1, 1, &f.D[ig][side][0][0], 6, 6, f.weights, 1, conj);
          double nn = std::sqrt(sqr(f.n[ig][0]) + sqr(f.n[ig][1]));
          for (int q = 0; q < 5; q++) brow[k][q] += conj[q + 1] * nn * f.wq[ig];
        }
      }
      // vectorBatch = b * Ainv^T
      for (int k = 0; k < g.nface; k++)
        for (int r = 0; r < 5; r++) {
          double v = 0;
          for (int t = 0; t < 5; t++) v += brow[k][t] * Ai[r * 5 + t];
          c.Ainvb[(i * 4 + k) * 5 + r] = v;
        }
    }
  });
  if (singular) { c.err = "singular VR matrix A_ii"; return 1; }
  c.u.assign(c.N * c.nv, 0.0);
  c.urec.assign(c.N * 5 * c.nv, 0.0);
  c.urecNew.assign(c.N * 5 * c.nv, 0.0);
  c.urec1.assign(c.N * 5 * c.nv, 0.0);
  c.lambdaFace.assign(c.F, 0.0);
  c.deltaLambdaFace.assign(c.F, 0.0);
  c.lambdaCell.assign(c.N, 0.0);
  c.dtCell.assign(c.N, 0.0);
  return 0;
}

// ------------------------------------------------------------------ VR sweep
// ReconstructionJacobiStep (DNDS_FV_VR.hpp:1474-1713): Jacobi into urecNew then
// copy back, or in-place Gauss-Seidel in natural order when sor_instead.
void cell_vr_update(orc_ctx& c, int64_t i, const double* src, double* dst) {
  const int nv = c.nv;
  const CellGeo& g = c.cg[i];
  const double relax = c.s.jacobi_relax;
  double acc[5][kMaxV];
  for (int r = 0; r < 5; r++)
    for (int v = 0; v < nv; v++) acc[r][v] = (1 - relax) * src[(i * 5 + r) * nv + v];
  const double* ui = &c.u[i * nv];
  for (int k = 0; k < g.nface; k++) {
    const FaceGeo& f = c.fg[g.faces[k]];
    int side = f.L == i ? 0 : 1;
    int j = side == 0 ? f.R : f.L;
    const double* M = &c.AinvB[(i * 4 + k) * 25];
    const double* bv = &c.Ainvb[(i * 4 + k) * 5];
    if (j >= 0) {
      const double* uj = &c.u[j * nv];
      for (int r = 0; r < 5; r++)
        for (int v = 0; v < nv; v++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += M[r * 5 + q] * src[(j * 5 + q) * nv + v];
          acc[r][v] += relax * (s + (uj[v] - ui[v]) * bv[r]);
        }
    } else if (f.bc == kWall) {
      for (int r = 0; r < 5; r++)
        for (int v = 0; v < nv; v++) acc[r][v] += relax * ((0.0 - ui[v]) * bv[r]);
    } else if (isFarType(f.bc)) {
      for (int r = 0; r < 5; r++)
        for (int v = 0; v < nv; v++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += M[r * 5 + q] * src[(i * 5 + q) * nv + v];
          acc[r][v] += relax * s;
        }
    } else if (f.bc == kWallEuler || f.bc == kWallNoSlip) {
      double corr[5][kMaxV];
      for (int r = 0; r < 5; r++) for (int v = 0; v < nv; v++) corr[r][v] = 0;
      for (int ig = 0; ig < 3; ig++) {
        const double(*D)[kND] = f.D[ig][0];
        double uBL[kMaxV], uBV[kMaxV];
        for (int v = 0; v < nv; v++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += D[0][q + 1] * src[(i * 5 + q) * nv + v];
          uBL[v] = s + ui[v];
        }
        double nn = std::sqrt(sqr(f.n[ig][0]) + sqr(f.n[ig][1]));
        double un[2] = {f.n[ig][0] / nn, f.n[ig][1] / nn};
        if (f.bc == kWallEuler) {
          for (int v = 0; v < nv; v++) uBV[v] = uBL[v];
          double d = un[0] * uBV[1] + un[1] * uBV[2];
          uBV[1] = uBL[1] - un[0] * d; uBV[2] = uBL[2] - un[1] * d;
        } else {
          boundary_value(c, uBL, un, f.gp[ig], 0.0, f.bc, uBV, true);
        }
        double w0 = f.weights[0];
        for (int r = 0; r < 5; r++)
          for (int v = 0; v < nv; v++) corr[r][v] += D[0][r + 1] * w0 * w0 * (uBV[v] - ui[v]) * nn * f.wq[ig];
      }
      const double* Ai = &c.Ainv[i * 25];
      for (int r = 0; r < 5; r++)
        for (int v = 0; v < nv; v++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += Ai[r * 5 + q] * corr[q][v];
          acc[r][v] += relax * s;
        }
    }
  }
  for (int r = 0; r < 5; r++)
    for (int v = 0; v < nv; v++) dst[(i * 5 + r) * nv + v] = acc[r][v];
}

void vr_sweep(orc_ctx& c) {
  const int nv = c.nv;
  if (c.s.sor_instead) {
    std::vector<double> old = c.urec;
    for (int64_t i = 0; i < c.N; i++) cell_vr_update(c, i, c.urec.data(), c.urec.data());
    double nall = 0;
    for (int64_t k = 0; k < c.N * 5 * nv; k++) nall += sqr(c.urec[k] - old[k]);
    c.lastInc = nall / double(c.N);
    return;
  }
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) cell_vr_update(c, i, c.urec.data(), c.urecNew.data());
  });
  double nall = 0;
  for (int64_t k = 0; k < c.N * 5 * nv; k++) nall += sqr(c.urec[k] - c.urecNew[k]);
  c.lastInc = nall / double(c.N);
  std::swap(c.urec, c.urecNew);
}

// ------------------------------------------------------------------ limiter
// characteristic matrices fML / fMR (DNDS_FV_EulerSolver.hpp:749-795)
void char_matrices(double gamma, const double* UL, const double* UR, const double* n, double Lm[4][4],
                   double Rm[4][4]) {
  double UC[4];
  for (int k = 0; k < 4; k++) UC[k] = (UL[k] + UR[k]) * 0.5;
  // NormBuildLocalBaseV: columns n, (-ny, nx)
  double nb[2][2] = {{n[0], -n[1]}, {n[1], n[0]}};
  double m0 = nb[0][0] * UC[1] + nb[1][0] * UC[2], m1 = nb[0][1] * UC[1] + nb[1][1] * UC[2];
  UC[1] = m0; UC[2] = m1;
  double vx = UC[1] / UC[0], vy = UC[2] / UC[0];
  double vs = vx * vx + vy * vy, p, a2, H;
  thermal(UC[3], UC[0], vs, gamma, p, a2, H);
  double a = std::sqrt(a2), gb = gamma - 1;
  double L[4][4] = {{H + a / gb * (vx - a), -vx - a / gb, -vy, 1},
                    {-2 * H + 4 / gb * (a * a), vx * 2, vy * 2, -2},
                    {vy * (-2 * (a * a) / gb), 0, 2 * (a * a) / gb, 0},
                    {H - a / gb * (vx + a), -vx + a / gb, -vy, 1}};
  double sc = gb / (2 * a * a);
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) L[i][j] *= sc;
  // M(:, 1:2) *= normBase^T
  for (int i = 0; i < 4; i++) {
    double c1 = L[i][1], c2 = L[i][2];
    L[i][1] = c1 * nb[0][0] + c2 * nb[0][1];
    L[i][2] = c1 * nb[1][0] + c2 * nb[1][1];
  }
  double R[4][4] = {{1, 1, 0, 1}, {vx - a, vx, 0, vx + a}, {vy, vy, 1, vy}, {H - vx * a, 0.5 * vs, vy, H + vx * a}};
  // M(1:2, :) = normBase * M(1:2, :)
  for (int j = 0; j < 4; j++) {
    double r1 = R[1][j], r2 = R[2][j];
    R[1][j] = nb[0][0] * r1 + nb[0][1] * r2;
    R[2][j] = nb[1][0] * r1 + nb[1][1] * r2;
  }
  std::memcpy(Lm, L, sizeof(L));
  std::memcpy(Rm, R, sizeof(R));
}

// the smoothness indicator of both WBAP limiters (DNDS_FV_VR.hpp:2075-2138 for V3, the same
// integrals at :1771-1836 for V2): si = sqrt(max over rho, E of sum_f IJI / ISI) * P^2
std::vector<double> limiter_indicator(orc_ctx& c) {
  const int nv = c.nv;
  const int I4 = 3;
  std::vector<double> ind(c.N);
  const double porder2 = double(c.s.rec_order * c.s.rec_order);
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      const CellGeo& g = c.cg[i];
      double sumJ[2] = {0, 0}, sumS[2] = {0, 0};
      for (int k = 0; k < g.nface; k++) {
        const FaceGeo& f = c.fg[g.faces[k]];
        int side = f.L == i ? 0 : 1;
        int j = side == 0 ? f.R : f.L;
        if (j < 0) continue;  // uRecVal / jump are zero on boundary faces
        // one point: gauss point 0 of the LINE_3 data with the LINE_1 weight 2
        const int ig = 0;
        double val[kND][2], jump[kND][2];
        int cols[2] = {0, I4};
        for (int d = 0; d < kND; d++)
          for (int cc = 0; cc < 2; cc++) {
            int v = cols[cc];
            double sL = 0, sR = 0;
            for (int q = 0; q < 5; q++) {
              sL += f.D[ig][0][d][q + 1] * c.urec[(f.L * 5 + q) * nv + v];
              sR += f.D[ig][1][d][q + 1] * c.urec[(f.R * 5 + q) * nv + v];
            }
            if (d == 0) { sL += c.u[f.L * nv + v]; sR += c.u[f.R * nv + v]; }
            val[d][cc] = (sL + sR) * 0.5;
            jump[d][cc] = (sL - sR) * 0.5;
          }
        double ISI[4], IJI[4];
        face_functional(c, f, ig, &val[0][0], 2, 2, &val[0][0], 2, 2, f.weights, 6, ISI);
        face_functional(c, f, ig, &jump[0][0], 2, 2, &jump[0][0], 2, 2, f.weights, 6, IJI);
        double nn = std::sqrt(sqr(f.n[ig][0]) + sqr(f.n[ig][1]));
        for (int cc = 0; cc < 2; cc++) {
          sumJ[cc] += IJI[cc * 2 + cc] * nn * 2.0;
          sumS[cc] += ISI[cc * 2 + cc] * nn * 2.0;
        }
      }
      double s0 = sumJ[0] / (sumS[0] + kVerySmall), s1 = sumJ[1] / (sumS[1] + kVerySmall);
      double smax = std::max(std::fabs(s0), std::fabs(s1));
      ind[i] = std::sqrt(smax) * porder2;
    }
  });
  return ind;
}

// ReconstructionWBAPLimitFacialV3 (DNDS_FV_VR.hpp:2053-2329), normWBAP=false
void limiter_wbap(orc_ctx& c, bool ifAll, double* indicator_out) {
  const int nv = c.nv;
  std::vector<double> ind = limiter_indicator(c);
  if (indicator_out) std::memcpy(indicator_out, ind.data(), sizeof(double) * c.N);
  const double scale = c.s.wbap_smooth_indicator_scale;
  const double nStd = c.s.wbap_n_std;
  const double sm4 = std::pow(kVerySmall, 1.0 / 4);
  std::vector<double>& src = c.urec;   // uRecNewBuf == uRec (unlimited)
  std::vector<double>& out = c.urec1;  // uRecNewBuf1
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      if (ind[i] < scale && !ifAll) continue;
      const CellGeo& g = c.cg[i];
      double uFaces[4][5][kMaxV];
      for (int pass = 0; pass < 2; pass++) {
        int ls = pass == 0 ? 2 : 0, le = pass == 0 ? 4 : 1;
        int nr = le - ls + 1;
        double uOthers[5][3][kMaxV];
        int nO = 0;
        for (int r = 0; r < nr; r++) for (int v = 0; v < nv; v++) uOthers[0][r][v] = src[(i * 5 + ls + r) * nv + v];
        nO = 1;
        for (int k = 0; k < g.nface; k++) {
          const FaceGeo& f = c.fg[g.faces[k]];
          int side = f.L == i ? 0 : 1;
          int j = side == 0 ? f.R : f.L;
          if (j < 0) continue;
          double nn = std::sqrt(sqr(f.ncenter[0]) + sqr(f.ncenter[1]));
          double un[2] = {f.ncenter[0] / nn, f.ncenter[1] / nn};
          const double(*ms)[5] = side ? f.msL2R : f.msR2L;       // other -> this
          const double(*msO)[5] = side ? f.msR2L : f.msL2R;      // this -> other
          double uOO[5][kMaxV];
          for (int r = 0; r < 5; r++) for (int v = 0; v < nv; v++) uOO[r][v] = src[(j * 5 + r) * nv + v];
          if (le < 4) {
            for (int r = le + 1; r < 5; r++)
              for (int v = 0; v < nv; v++) {
                double s = 0;
                for (int q = le + 1; q < 5; q++) s += msO[r][q] * uFaces[k][q][v];
                uOO[r][v] = s;
              }
          }
          double uOtherIn[3][kMaxV], uThisIn[3][kMaxV];
          for (int r = 0; r < nr; r++)
            for (int v = 0; v < nv; v++) {
              double s = 0;
              for (int q = 0; q < 5; q++) s += ms[ls + r][q] * uOO[q][v];
              uOtherIn[r][v] = s;
              uThisIn[r][v] = uOthers[0][r][v];
            }
          const double* uR = side ? &c.u[i * nv] : &c.u[j * nv];
          const double* uL = side ? &c.u[j * nv] : &c.u[i * nv];
          double Lm[4][4], Rm[4][4];
          char_matrices(c.s.gamma, uL, uR, un, Lm, Rm);
          double cO[3][kMaxV], cT[3][kMaxV], lim[3][kMaxV];
          for (int r = 0; r < nr; r++)
            for (int a = 0; a < nv; a++) {
              double so = 0, st = 0;
              for (int q = 0; q < nv; q++) { so += Lm[a][q] * uOtherIn[r][q]; st += Lm[a][q] * uThisIn[r][q]; }
              cO[r][a] = so; cT[r][a] = st;
            }
          // FWBAP_L2_Biway(uThis, uOther, out, 1)
          for (int r = 0; r < nr; r++)
            for (int a = 0; a < nv; a++) {
              double u1 = cT[r][a], u2 = cO[r][a];
              double frac = u1 / (std::fabs(u2) + 1e-12) * signE(u2);
              double th1 = frac * frac * frac, th2 = sqr(frac) * sqr(frac);
              lim[r][a] = u1 * (1.0 + th1) / (1.0 + th2);
            }
          for (int r = 0; r < nr; r++)
            for (int a = 0; a < nv; a++) {
              double s = 0;
              for (int q = 0; q < nv; q++) s += Rm[a][q] * lim[r][q];
              uFaces[k][ls + r][a] = s;
              uOthers[nO][r][a] = s;
            }
          nO++;
        }
        // FWBAP_L2_Multiway(uOthers, nO, out, nStd)
        for (int r = 0; r < nr; r++)
          for (int v = 0; v < nv; v++) {
            double up = 0, down = 0, u0 = uOthers[0][r][v];
            for (int o = 1; o < nO; o++) {
              double uo = uOthers[o][r][v];
              double ti = u0 / (std::fabs(uo) + sm4) * signE(uo);
              down += sqr(ti) * sqr(ti);
              up += ti * ti * ti;
            }
            out[(i * 5 + ls + r) * nv + v] = u0 * (up + nStd) / (down + nStd);
          }
      }
    }
  });
  for (int64_t i = 0; i < c.N; i++) {
    if (ind[i] < scale && !ifAll) continue;
    for (int k = 0; k < 5 * nv; k++) c.urec[i * 5 * nv + k] = c.urec1[i * 5 * nv + k];
  }
}

// ReconstructionWBAPLimitFacialV2 (DNDS_FV_VR.hpp:1749-2047, "3WBAP", limiterProcedure 0), normWBAP=false.
// The indicator as V3.  Then order by order over all cells -- P2 rows 2..4, then P1 rows 0..1 -- each pass
// reading the coefficients as the previous one left them (uRecNewBuf; after the P2 pass the listed
// cells' rows 2..4 are limited): against every neighbour j, the secondary reconstruction of j's whole
// coefficient set in this cell's basis (matrixSecondary * uRecNewBuf[j], rows of the pass), both sides
// projected to characteristic space (M = L(face mean)), FWBAP_L2_Biway with n = WBAP_nStd, back with R;
// then FWBAP_L2_Multiway over those results with n = 1, centred on the FIRST neighbour's result (the
// reference's uOthers holds only the neighbours' results, in cell2face order).  A cell with no
// interior face keeps its coefficients (the reference would read past an empty list there).
void limiter_wbap_v2(orc_ctx& c, bool ifAll, double* indicator_out) {
  const int nv = c.nv;
  std::vector<double> ind = limiter_indicator(c);
  if (indicator_out) std::memcpy(indicator_out, ind.data(), sizeof(double) * c.N);
  const double scale = c.s.wbap_smooth_indicator_scale;
  const double nStd = c.s.wbap_n_std;
  const double sm4 = std::pow(kVerySmall, 1.0 / 4);
  std::vector<double>& buf = c.urec;   // uRecNewBuf (starts as uRec)
  std::vector<double>& out = c.urec1;  // uRecNewBuf1
  for (int pass = 0; pass < 2; pass++) {
    const int ls = pass == 0 ? 2 : 0, le = pass == 0 ? 4 : 1, nr = le - ls + 1;
    parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; i++) {
        if (ind[i] < scale && !ifAll) continue;
        const CellGeo& g = c.cg[i];
        double first[3][kMaxV], up[3][kMaxV], down[3][kMaxV];
        for (int r = 0; r < 3; r++) for (int v = 0; v < kMaxV; v++) { first[r][v] = up[r][v] = down[r][v] = 0; }
        int nO = 0;
        for (int k = 0; k < g.nface; k++) {
          const FaceGeo& f = c.fg[g.faces[k]];
          const int side = f.L == i ? 0 : 1;
          const int j = side == 0 ? f.R : f.L;
          if (j < 0) continue;
          const double nn = std::sqrt(sqr(f.ncenter[0]) + sqr(f.ncenter[1]));
          const double un[2] = {f.ncenter[0] / nn, f.ncenter[1] / nn};
          const double(*ms)[5] = side ? f.msL2R : f.msR2L;  // other -> this
          double uOtherIn[3][kMaxV], uThisIn[3][kMaxV];
          for (int r = 0; r < nr; r++)
            for (int v = 0; v < nv; v++) {
              double s = 0;
              for (int q = 0; q < 5; q++) s += ms[ls + r][q] * buf[(j * 5 + q) * nv + v];
              uOtherIn[r][v] = s;
              uThisIn[r][v] = buf[(i * 5 + ls + r) * nv + v];
            }
          const double* uR = side ? &c.u[i * nv] : &c.u[j * nv];
          const double* uL = side ? &c.u[j * nv] : &c.u[i * nv];
          double Lm[4][4], Rm[4][4];
          char_matrices(c.s.gamma, uL, uR, un, Lm, Rm);
          double cO[3][kMaxV], cT[3][kMaxV], lim[3][kMaxV];
          for (int r = 0; r < nr; r++)
            for (int a = 0; a < nv; a++) {
              double so = 0, st = 0;
              for (int q = 0; q < nv; q++) { so += Lm[a][q] * uOtherIn[r][q]; st += Lm[a][q] * uThisIn[r][q]; }
              cO[r][a] = so; cT[r][a] = st;
            }
          // FWBAP_L2_Biway(uThis, uOther, out, WBAP_nStd)
          for (int r = 0; r < nr; r++)
            for (int a = 0; a < nv; a++) {
              const double u1 = cT[r][a], u2 = cO[r][a];
              const double frac = u1 / (std::fabs(u2) + 1e-12) * signE(u2);
              const double th1 = frac * frac * frac, th2 = sqr(frac) * sqr(frac);
              lim[r][a] = u1 * (nStd + th1) / (nStd + th2);
            }
          for (int r = 0; r < nr; r++)
            for (int a = 0; a < nv; a++) {
              double s = 0;
              for (int q = 0; q < nv; q++) s += Rm[a][q] * lim[r][q];
              if (nO == 0) {
                first[r][a] = s;
              } else {  // FWBAP_L2_Multiway accumulation, uOthers[0] = the first neighbour's result
                const double ti = first[r][a] / (std::fabs(s) + sm4) * signE(s);
                down[r][a] += sqr(ti) * sqr(ti);
                up[r][a] += ti * ti * ti;
              }
            }
          nO++;
        }
        for (int r = 0; r < nr; r++)
          for (int v = 0; v < nv; v++)
            out[(i * 5 + ls + r) * nv + v] =
                nO ? first[r][v] * (up[r][v] + 1.0) / (down[r][v] + 1.0) : buf[(i * 5 + ls + r) * nv + v];
      }
    });
    for (int64_t i = 0; i < c.N; i++) {
      if (ind[i] < scale && !ifAll) continue;
      for (int k = ls * nv; k < (le + 1) * nv; k++) buf[i * 5 * nv + k] = out[i * 5 * nv + k];
    }
  }
}

// the limiter of the stage composition: limiterProcedure 1 (CWBAP, V3) or 0 (3WBAP, V2)
void limiter_stage(orc_ctx& c) {
  if (c.s.limiter == 2) limiter_wbap_v2(c, false, nullptr);
  else if (c.s.limiter) limiter_wbap(c, false, nullptr);
}

// ------------------------------------------------------------------ dt
// Sutherland's law at the mean state (fluxFace, DNDS_FV_EulerEvaluator.hpp:405-412):
// T = p / ((gamma - 1) / gamma * Cp * rho)
double sutherland_mu(const orc_settings& s, double p, double rho) {
  const double T = p / ((s.gamma - 1) / s.gamma * s.cp_gas * rho);
  return s.mu_gas * std::pow(T / s.t_ref, 1.5) * (s.t_ref + s.c_sutherland) / (T + s.c_sutherland);
}

// SA eddy-viscosity factor of fluxFace / EvaluateDt (DNDS_FV_EulerEvaluator.hpp:413-425,
// USE_NS_SA_NEGATIVE_MODEL): muf = mu (1 + Chi fnu1), Chi = U5 muRef / mu softened below 10
double sa_mu_factor(const orc_settings& s, double U5, double mufPhy) {
  const double cnu1 = 7.1;
  double Chi = U5 * s.mu_gas / mufPhy;
  if (Chi < 10) Chi = 0.05 * std::log(1 + std::exp(20 * Chi));
  const double Chi3 = Chi * Chi * Chi;
  const double fnu1 = Chi3 / (Chi3 + cnu1 * cnu1 * cnu1);
  return std::max(1 + Chi * fnu1, 1.0);
}

void eval_dt(orc_ctx& c, double cfl, double maxDt, bool useLocal, double* dtMinOut) {
  const int nv = c.nv;
  const double gamma = c.s.gamma;
  std::fill(c.lambdaCell.begin(), c.lambdaCell.end(), 0.0);
  parallel_for(c.nthreads, c.F, [&](int64_t b, int64_t e) {
    for (int64_t f = b; f < e; f++) {
      const FaceGeo& fg = c.fg[f];
      double nn = std::sqrt(sqr(fg.ncenter[0]) + sqr(fg.ncenter[1]));
      double un[2] = {fg.ncenter[0] / nn, fg.ncenter[1] / nn};
      const double* UL = &c.u[fg.L * nv];
      double uMean[kMaxV];
      for (int k = 0; k < nv; k++) uMean[k] = UL[k];
      double vL[2] = {UL[1] / UL[0], UL[2] / UL[0]}, vR[2] = {vL[0], vL[1]};
      double pL, aL2, HL, pR, aR2, HR;
      thermal(UL[3], UL[0], vL[0] * vL[0] + vL[1] * vL[1], gamma, pL, aL2, HL);
      pR = pL; HR = HL; aR2 = aL2;
      double volR = c.cg[fg.L].vol;
      if (fg.R >= 0) {
        const double* UR = &c.u[fg.R * nv];
        for (int k = 0; k < nv; k++) uMean[k] = (uMean[k] + UR[k]) * 0.5;
        vR[0] = UR[1] / UR[0]; vR[1] = UR[2] / UR[0];
        thermal(UR[3], UR[0], vR[0] * vR[0] + vR[1] * vR[1], gamma, pR, aR2, HR);
        volR = c.cg[fg.R].vol;
      }
      double vnMean = 0.5 * ((vL[0] + vR[0]) * un[0] + (vL[1] + vR[1]) * un[1]);
      double pMean = (pL + pR) * 0.5;
      double aMean = std::sqrt(gamma * pMean / uMean[0]);
      double lamConv = std::fabs(vnMean) + aMean;
      // viscous part (DNDS_FV_EulerEvaluator.cpp:80-99): muf at the mean state
      double lamVis = 0.0;
      if (c.s.mu_gas > 0) {
        double muf = sutherland_mu(c.s, pMean, uMean[0]);
        if (nv > 4) muf *= sa_mu_factor(c.s, uMean[4], muf);
        lamVis = muf / uMean[0] * std::max(4. / 3., gamma / c.s.pr_gas);
      }
      double area = fg.area;
      c.lambdaFace[f] = lamConv + lamVis * area * (1. / c.cg[fg.L].vol + 1. / volR);
      c.deltaLambdaFace[f] = std::fabs((vR[0] - vL[0]) * un[0] + (vR[1] - vL[1]) * un[1]) +
                             std::sqrt(std::fabs(aR2 - aL2)) * 0.7071;
    }
  });
  for (int64_t f = 0; f < c.F; f++) {
    const FaceGeo& fg = c.fg[f];
    c.lambdaCell[fg.L] += c.lambdaFace[f] * fg.area;
    if (fg.R >= 0) c.lambdaCell[fg.R] += c.lambdaFace[f] * fg.area;
  }
  double dtMin = 3e200;
  for (int64_t i = 0; i < c.N; i++) {
    c.dtCell[i] = std::min(cfl * c.cg[i].vol / (c.lambdaCell[i] + 1e-100), maxDt);
    dtMin = std::min(dtMin, c.dtCell[i]);
  }
  if (!useLocal)
    for (int64_t i = 0; i < c.N; i++) c.dtCell[i] = dtMin;
  if (dtMinOut) *dtMinOut = dtMin;
}

// ------------------------------------------------------------------ RHS
// Gas::ViscousFlux_IdealGas (DNDS_Gas.hpp:795-826) for dim 2, contracted with the unit normal:
// Fn[k] = sum_i n_i Flux(i, k).  G[i][v] = d U_v / d x_i (conservative gradients).
void viscous_flux_n(const double* U, const double G[2][4], const double* n, bool adiabatic, double gamma,
                    double mu, double k, double cp, double* Fn) {
  const double v[2] = {U[1] / U[0], U[2] / U[0]};
  double S[2][2];  // strainRate(i, j) = d u_j / d x_i
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) S[i][j] = (U[0] * G[i][1 + j] - G[i][0] * U[1 + j]) / (U[0] * U[0]);
  double gradP[2], gradT[2];
  for (int i = 0; i < 2; i++)
    gradP[i] = (gamma - 1) * (G[i][3] - 0.5 * (G[i][1] * v[0] + G[i][2] * v[1] + S[i][0] * U[1] + S[i][1] * U[2]));
  const double p = (gamma - 1) * (U[3] - U[0] * 0.5 * (v[0] * v[0] + v[1] * v[1]));
  for (int i = 0; i < 2; i++) gradT[i] = gamma / ((gamma - 1) * cp * U[0] * U[0]) * (U[0] * gradP[i] - p * G[i][0]);
  if (adiabatic) {
    const double d = gradT[0] * n[0] + gradT[1] * n[1];
    gradT[0] -= d * n[0];
    gradT[1] -= d * n[1];
  }
  const double lambda = -2. / 3., tr = S[0][0] + S[1][1];
  double F[2][4];
  for (int i = 0; i < 2; i++) {
    F[i][0] = 0;
    for (int j = 0; j < 2; j++) F[i][1 + j] = (S[i][j] + S[j][i]) * mu + (i == j ? lambda * mu * tr : 0.0);
    F[i][3] = F[i][1] * v[0] + F[i][2] * v[1] + k * gradT[i];
  }
  for (int q = 0; q < 4; q++) Fn[q] = n[0] * F[0][q] + n[1] * F[1][q];
}

// one face: fluxEs (3 columns: flux, FLfix, FRfix) integrated over the 3 GPs
// (EvaluateRHS face loop, DNDS_FV_EulerEvaluator.cpp:215-514, and fluxFace,
// DNDS_FV_EulerEvaluator.hpp:371-591); nv = 4 (NS_2D) or 5 (SA, the last variable rho nu~ / muRef)
void face_flux(const orc_ctx& c, int64_t f, double t, double fl[3][kMaxV], double* gpvals /*[3][2][nv] or null*/,
               int* reduced) {
  const int nv = c.nv;
  const FaceGeo& fg = c.fg[f];
  const double gamma = c.s.gamma;
  for (int a = 0; a < 3; a++) for (int k = 0; k < kMaxV; k++) fl[a][k] = 0;
  const double* uL = &c.u[fg.L * nv];
  const double* uR = fg.R >= 0 ? &c.u[fg.R * nv] : nullptr;
  for (int ig = 0; ig < 3; ig++) {
    double nn = std::sqrt(sqr(fg.n[ig][0]) + sqr(fg.n[ig][1]));
    double un[2] = {fg.n[ig][0] / nn, fg.n[ig][1] / nn};
    double inc[kMaxV] = {}, ULxy[kMaxV] = {}, URxy[kMaxV] = {}, ULm[kMaxV] = {}, URm[kMaxV] = {};
    bool redL = false, redR = false;
    for (int v = 0; v < nv; v++) {
      double s = 0;
      for (int q = 0; q < 5; q++) s += fg.D[ig][0][0][q + 1] * c.urec[(fg.L * 5 + q) * nv + v];
      inc[v] = s;
    }
    compress_rec_part(uL, inc, ULxy, redL, nv);
    for (int v = 0; v < nv; v++) ULm[v] = uL[v];
    if (fg.R >= 0) {
      for (int v = 0; v < nv; v++) {
        double s = 0;
        for (int q = 0; q < 5; q++) s += fg.D[ig][1][0][q + 1] * c.urec[(fg.R * 5 + q) * nv + v];
        inc[v] = s;
      }
      compress_rec_part(uR, inc, URxy, redR, nv);
      for (int v = 0; v < nv; v++) URm[v] = uR[v];
    } else {
      boundary_value(c, ULxy, un, fg.center, t, fg.bc, URxy, true);
      boundary_value(c, ULm, un, fg.center, t, fg.bc, URm, false);
    }
    if (reduced) *reduced += int(redL) + int(redR);
    if (gpvals)
      for (int v = 0; v < nv; v++) { gpvals[(ig * 2 + 0) * nv + v] = ULxy[v]; gpvals[(ig * 2 + 1) * nv + v] = URxy[v]; }
    // fluxFace (DNDS_FV_EulerEvaluator.hpp:371-591)
    double nb[2][2] = {{un[0], -un[1]}, {un[1], un[0]}};
    double UL[kMaxV] = {ULxy[0], nb[0][0] * ULxy[1] + nb[1][0] * ULxy[2], nb[0][1] * ULxy[1] + nb[1][1] * ULxy[2], ULxy[3]};
    double UR[kMaxV] = {URxy[0], nb[0][0] * URxy[1] + nb[1][0] * URxy[2], nb[0][1] * URxy[1] + nb[1][1] * URxy[2], URxy[3]};
    for (int v = 4; v < nv; v++) { UL[v] = ULxy[v]; UR[v] = URxy[v]; }
    double FLf[kMaxV] = {0}, FRf[kMaxV] = {0};
    {
      double Lm[4] = {ULm[0], nb[0][0] * ULm[1] + nb[1][0] * ULm[2], nb[0][1] * ULm[1] + nb[1][1] * ULm[2], ULm[3]};
      double Rm[4] = {URm[0], nb[0][0] * URm[1] + nb[1][0] * URm[2], nb[0][1] * URm[1] + nb[1][1] * URm[2], URm[3]};
      double wL[4], wR[4];
      cons2prim(Lm, wL, gamma); cons2prim(Rm, wR, gamma);
      inviscid_flux(Lm, wL[1], wL[3], FLf);
      inviscid_flux(Rm, wR[1], wR[3], FRf);
      double a1 = FLf[1], a2 = FLf[2];
      FLf[1] = nb[0][0] * a1 + nb[0][1] * a2; FLf[2] = nb[1][0] * a1 + nb[1][1] * a2;
      a1 = FRf[1]; a2 = FRf[2];
      FRf[1] = nb[0][0] * a1 + nb[0][1] * a2; FRf[2] = nb[1][0] * a1 + nb[1][1] * a2;
      if (nv > 4) { FLf[4] = wL[1] * ULm[4]; FRf[4] = wR[1] * URm[4]; }  // F_5 = rhoNut * un
    }
    double F[kMaxV] = {0};
    if (c.s.riemann == 2) hllc_flux(UL, UR, gamma, F);
    else roe_flux(UL, UR, gamma, F, c.deltaLambdaFace[f]);
    if (nv > 4) {
      // the SA variable: central flux with upwinding by the contact wave, |Roe normal velocity|
      // (Roe) or |mean normal velocity| (HLLC) (DNDS_FV_EulerEvaluator.hpp:540-553)
      double lam123;
      if (c.s.riemann == 2) {
        lam123 = std::fabs(UL[1] / UL[0] + UR[1] / UR[0]) * 0.5;
      } else {
        double sL = std::sqrt(UL[0]), sR = std::sqrt(UR[0]);
        lam123 = std::fabs((sL * UL[1] / UL[0] + sR * UR[1] / UR[0]) / (sL + sR));
      }
      F[4] = ((UL[1] / UL[0] * UL[4] + UR[1] / UR[0] * UR[4]) - (UR[4] - UL[4]) * lam123) * 0.5;
    }
    double a1 = F[1], a2 = F[2];
    F[1] = nb[0][0] * a1 + nb[0][1] * a2; F[2] = nb[1][0] * a1 + nb[1][1] * a2;
    if (c.s.mu_gas > 0) {
      // the viscous flux at the mean state with the face gradient of EvaluateRHS
      // (DNDS_FV_EulerEvaluator.cpp:279-370): the mean of both sides' reconstructed gradients
      // (the inner one's on a boundary) plus the jump (UR - UL) n / distGRP, distGRP =
      // 2 min(V_L, V_R) / A, made effectively infinite at walls
      double GL[2][kMaxV], GR[2][kMaxV], G[2][kMaxV];
      for (int d = 0; d < 2; d++)
        for (int v = 0; v < nv; v++) {
          double sL = 0, sR = 0;
          for (int q = 0; q < 5; q++) sL += fg.D[ig][0][1 + d][q + 1] * c.urec[(fg.L * 5 + q) * nv + v];
          if (fg.R >= 0)
            for (int q = 0; q < 5; q++) sR += fg.D[ig][1][1 + d][q + 1] * c.urec[(fg.R * 5 + q) * nv + v];
          GL[d][v] = sL;
          GR[d][v] = fg.R >= 0 ? sR : sL;
        }
      double minVol = c.cg[fg.L].vol;
      if (fg.R >= 0) minVol = std::min(minVol, c.cg[fg.R].vol);
      double distGRP = minVol / fg.area * 2;
      if (fg.bc == kWallEuler || fg.bc == kWallNoSlip) distGRP += 3e200;
      for (int d = 0; d < 2; d++)
        for (int v = 0; v < nv; v++) G[d][v] = (GR[d][v] + GL[d][v]) * 0.5 + (1.0 / distGRP) * un[d] * (URxy[v] - ULxy[v]);
      double Um[kMaxV];
      for (int v = 0; v < nv; v++) Um[v] = 0.5 * (ULxy[v] + URxy[v]);
      double pm, am, Hm;
      thermal(Um[3], Um[0], sqr(Um[1] / Um[0]) + sqr(Um[2] / Um[0]), gamma, pm, am, Hm);
      const double mufPhy = sutherland_mu(c.s, pm, Um[0]);
      double muf = mufPhy;
      if (nv > 4) muf *= sa_mu_factor(c.s, Um[4], mufPhy);
      const double kc = c.s.cp_gas * (muf - mufPhy) / 0.9 + c.s.cp_gas * mufPhy / c.s.pr_gas;
      double Gf[2][4];
      for (int d = 0; d < 2; d++) for (int v = 0; v < 4; v++) Gf[d][v] = G[d][v];
      double Fv[4];
      viscous_flux_n(Um, Gf, un, fg.bc == kWallNoSlip, gamma, muf, kc, c.s.cp_gas, Fv);
      for (int k = 0; k < 4; k++) F[k] -= Fv[k];
      if (nv > 4) {
        // the SA diffusion (DNDS_FV_EulerEvaluator.hpp:463-480)
        const double muRef = c.s.mu_gas, sigma = 2. / 3., cn1 = 16;
        double fn = 1;
        if (Um[4] < 0) {
          const double Chi = Um[4] * muRef / mufPhy;
          fn = (cn1 + Chi * Chi * Chi) / (cn1 - Chi * Chi * Chi);
        }
        double dn = 0;
        for (int d = 0; d < 2; d++) {
          const double diffNu = (G[d][4] * muRef - Um[4] * muRef / Um[0] * G[d][0]) / Um[0];
          dn += un[d] * diffNu * (mufPhy + Um[4] * muRef * fn) / sigma / muRef;
        }
        F[4] -= dn;
      }
    }
    double w = nn * fg.wq[ig];
    for (int k = 0; k < nv; k++) {
      fl[0][k] += -F[k] * w;
      fl[1][k] += FLf[k] * w;
      fl[2][k] += FRf[k] * w;
    }
  }
}

// EulerEvaluator::source and sourceJacobianDiag for NS_SA (DNDS_FV_EulerEvaluator.hpp:593-864,
// USE_NS_SA_NEGATIVE_MODEL): the SA-neg production, destruction and cb2 diffusion of the
// last variable at one point; U is the (compressed) reconstructed state, G[d][v] its gradient
void sa_source(const orc_ctx& c, const double* U, const double G[2][kMaxV], double dWall, double& src,
               double& jac) {
  const double d = std::min(dWall, std::pow(3e200, 1. / 6.));
  const double cb1 = 0.1355, cb2 = 0.622, sigma = 2. / 3., cnu1 = 7.1, cnu2 = 0.7, cnu3 = 0.9, cw2 = 0.3, cw3 = 2,
               kappa = 0.41, rlim = 10, ct3 = 1.2, ct4 = 0.5;
  const double cw1 = cb1 / sqr(kappa) + (1 + cb2) / sigma;
  const double gamma = c.s.gamma;
  double p, a2, H;
  thermal(U[3], U[0], sqr(U[1] / U[0]) + sqr(U[2] / U[0]), gamma, p, a2, H);
  const double muRef = c.s.mu_gas;
  const double nuh = U[4] * muRef / U[0];
  const double mufPhy = sutherland_mu(c.s, p, U[0]);
  const double Chi = U[4] * muRef / mufPhy;
  const double fnu1 = std::pow(Chi, 3) / (std::pow(Chi, 3) + std::pow(cnu1, 3));
  const double fnu2 = 1 - Chi / (1 + Chi * fnu1);
  const double velo[2] = {U[1] / U[0], U[2] / U[0]};
  double diffNu[2], diffRho[2], diffU[2][2];
  for (int i = 0; i < 2; i++) {
    diffRho[i] = G[i][0];
    diffNu[i] = (G[i][4] * muRef - nuh * G[i][0]) / U[0];
    for (int j = 0; j < 2; j++) diffU[i][j] = (G[i][1 + j] - G[i][0] * velo[j]) / U[0];
  }
  // Omega = (diffU^T - diffU) / 2, S = |Omega|_F sqrt(2)
  const double w01 = 0.5 * (diffU[1][0] - diffU[0][1]);
  const double S = std::sqrt(2 * w01 * w01) * std::sqrt(2.0);
  const double Sbar = nuh / (sqr(kappa) * sqr(d)) * fnu2;
  double Sh;
  if (Sbar < -cnu2 * S) Sh = S + S * (sqr(cnu2) * S + cnu3 * Sbar) / ((cnu3 - 2 * cnu2) * S - Sbar);
  else Sh = S + Sbar;
  const double r = std::min(nuh / (Sh * sqr(kappa * d) + kVerySmall), rlim);
  const double g = r + cw2 * (std::pow(r, 6) - r);
  const double fw = g * std::pow((1 + std::pow(cw3, 6)) / (std::pow(g, 6) + std::pow(cw3, 6)), 1. / 6.);
  const double ft2 = ct3 * std::exp(-ct4 * sqr(Chi));
  double D = (cw1 * fw - cb1 / sqr(kappa) * ft2) * sqr(nuh / d);
  double P = cb1 * (1 - ft2) * Sh * nuh;
  double fn = 1;
  if (U[4] < 0) {
    const double cn1 = 16;
    fn = (cn1 + std::pow(Chi, 3)) / (cn1 - std::pow(Chi, 3));
    P = cb1 * (1 - ct3) * S * nuh;
    D = -cw1 * sqr(nuh / d);
  }
  const double dn2 = diffNu[0] * diffNu[0] + diffNu[1] * diffNu[1];
  const double rn = diffRho[0] * diffNu[0] + diffRho[1] * diffNu[1];
  src = U[0] * (P - D + dn2 * cb2 / sigma) / muRef - (U[4] * fn * muRef + mufPhy) / (U[0] * sigma) * rn / muRef;
  jac = -std::min(U[0] * (P * 0 - D * 2) / muRef / (U[4] + kVerySmall), -kVerySmall);
}

void eval_rhs(orc_ctx& c, double t, double* rhs, double* wallFlux, int* nreduced) {
  const int nv = c.nv;
  const int FW = 3 * kMaxV;
  std::vector<double> buf(c.F * FW);
  std::atomic<int> red{0};
  parallel_for(c.nthreads, c.F, [&](int64_t b, int64_t e) {
    int r = 0;
    for (int64_t f = b; f < e; f++) {
      double fl[3][kMaxV];
      face_flux(c, f, t, fl, nullptr, &r);
      std::memcpy(&buf[f * FW], fl, sizeof(fl));
    }
    red += r;
  });
  for (int64_t k = 0; k < c.N * nv; k++) rhs[k] = 0;
  double wf[kMaxV] = {0};
  // scatter in face order (DNDS_FV_EulerEvaluator.cpp:501-516)
  for (int64_t f = 0; f < c.F; f++) {
    const FaceGeo& fg = c.fg[f];
    const double* fl = &buf[f * FW];
    double vL = c.cg[fg.L].vol;
    for (int k = 0; k < nv; k++) rhs[fg.L * nv + k] += fl[k] / vL;
    if (fg.R >= 0) {
      double vR = c.cg[fg.R].vol;
      for (int k = 0; k < nv; k++) rhs[fg.R * nv + k] -= fl[k] / vR;
    }
    for (int k = 0; k < nv; k++) rhs[fg.L * nv + k] -= fl[kMaxV + k] / vL;
    if (fg.R >= 0) {
      double vR = c.cg[fg.R].vol;
      for (int k = 0; k < nv; k++) rhs[fg.R * nv + k] += fl[2 * kMaxV + k] / vR;
    }
    if (fg.bc == kWallNoSlip || fg.bc == kWallEuler)
      for (int k = 0; k < nv; k++) wf[k] -= fl[k];
  }
  if (wallFlux) for (int k = 0; k < nv; k++) wallFlux[k] = wf[k];
  if (nreduced) *nreduced = red.load();
  // cell source loop (DNDS_FV_EulerEvaluator.cpp:520-638): the SA source and its diagonal Jacobian
  // integrated over the cell's quadrature with the reconstructed value and gradient
  c.srcJac.assign(c.N * nv, 0.0);
  if (nv < 5) return;
  const Quad q3 = tri4(), q4 = quad9();
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      const CellGeo& g = c.cg[i];
      const Quad& q = g.nn == 3 ? q3 : q4;
      double sv = 0, sj = 0;
      for (int ig = 0; ig < q.n; ig++) {
        double N[4], dN[2][4], x = 0, y = 0, J[2][2] = {{0, 0}, {0, 0}};
        shape(g.nn, q.p[ig][0], q.p[ig][1], N, dN);
        for (int k = 0; k < g.nn; k++) {
          x += N[k] * g.xy[k][0]; y += N[k] * g.xy[k][1];
          for (int d = 0; d < 2; d++) { J[d][0] += dN[d][k] * g.xy[k][0]; J[d][1] += dN[d][k] * g.xy[k][1]; }
        }
        const double wdet = q.w[ig] * (J[0][0] * J[1][1] - J[0][1] * J[1][0]);
        double D[kND][kND];
        diff_base_value(c, g, x, y, g.moment, D);
        double inc[kMaxV] = {}, U[kMaxV] = {}, G[2][kMaxV] = {};
        for (int v = 0; v < nv; v++) {
          double s0 = 0, s1 = 0, s2 = 0;
          for (int r = 0; r < 5; r++) {
            const double a = c.urec[(i * 5 + r) * nv + v];
            s0 += D[0][r + 1] * a; s1 += D[1][r + 1] * a; s2 += D[2][r + 1] * a;
          }
          inc[v] = s0; G[0][v] = s1; G[1][v] = s2;
        }
        bool red2 = false;
        compress_rec_part(&c.u[i * nv], inc, U, red2, nv);
        double src, jac;
        sa_source(c, U, G, c.dWall[i], src, jac);
        sv += src * wdet;
        sj += jac * wdet;
      }
      rhs[i * nv + 4] += sv / g.vol;
      c.srcJac[i * nv + 4] = sj / g.vol;
    }
  });
}

// first-order wall distance (USE_FIRST_ORDER_WALL_DIST, DNDS_FV_EulerEvaluator.hpp:227-363): from
// each cell's barycentre to the nearest Wall_NoSlip face segment
void wall_distance(orc_ctx& c, const orc_mesh& m) {
  std::vector<std::array<double, 4>> seg;
  for (int64_t f = 0; f < c.F; f++)
    if (c.fg[f].bc == kWallNoSlip) {
      const int a = m.face_nodes[2 * f], b = m.face_nodes[2 * f + 1];
      seg.push_back({m.node_xy[2 * a], m.node_xy[2 * a + 1], m.node_xy[2 * b], m.node_xy[2 * b + 1]});
    }
  c.dWall.assign(c.N, std::pow(3e200, 1. / 6.));
  parallel_for(c.nthreads, c.N, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      const double px = c.cg[i].bary[0], py = c.cg[i].bary[1];
      double best = std::pow(3e200, 1. / 6.);
      for (const auto& sg : seg) {
        const double ex = sg[2] - sg[0], ey = sg[3] - sg[1];
        const double L2 = std::sqrt(ex * ex + ey * ey);
        const double bx = px - sg[0], by = py - sg[1];
        const double LB = (bx * ex + by * ey) / L2;
        double d;
        if (LB >= 0 && LB <= L2) d = std::sqrt(sqr(bx - LB * ex / L2) + sqr(by - LB * ey / L2));
        else d = std::min(std::sqrt(bx * bx + by * by), std::sqrt(sqr(px - sg[2]) + sqr(py - sg[3])));
        best = std::min(best, d);
      }
      c.dWall[i] = best;
    }
  });
}

// ------------------------------------------------------------------ implicit path
// EulerEvaluator::fluxJacobian0_Right_Times_du (DNDS_FV_EulerEvaluator.hpp:928-956) for NS_2D:
// the inviscid flux increment of dU about U through the unit normal n
// (Gas::IdealGasUIncrement, GasInviscidFluxFacialIncrement, DNDS_Gas.hpp:122-146),
// minus lambdaMain * dU
void flux_jac_times_du(const double* U, const double* n, const double* dU, double lam, double gamma, double* dF,
                       int nv = 4) {
  const double vx = U[1] / U[0], vy = U[2] / U[0];
  double p, a2, H;
  thermal(U[3], U[0], vx * vx + vy * vy, gamma, p, a2, H);
  const double dvx = (dU[1] - U[1] / U[0] * dU[0]) / U[0], dvy = (dU[2] - U[2] / U[0] * dU[0]) / U[0];
  const double dp = (gamma - 1) * (dU[3] - 0.5 * (dU[1] * vx + dU[2] * vy + U[1] * dvx + U[2] * dvy));
  const double vn = vx * n[0] + vy * n[1], dvn = dvx * n[0] + dvy * n[1];
  dF[0] = dU[1] * n[0] + dU[2] * n[1];
  dF[1] = dU[1] * vn + U[1] * dvn + n[0] * dp;
  dF[2] = dU[2] * vn + U[2] * dvn + n[1] * dp;
  dF[3] = (dU[3] + dp) * vn + (U[3] + p) * dvn;
  for (int k = 0; k < 4; k++) dF[k] -= lam * dU[k];
  for (int k = 4; k < nv; k++) dF[k] = dU[k] * vn + U[k] * dvn - dU[k] * lam;  // the SA variable
}

// CompressInc (DNDS_FV_EulerEvaluator.hpp:1362-1406): the SA variable may not go negative; an
// increment that would make it so is replaced by an exponential decay, floored at 1e-6
void compress_inc(const orc_ctx& c, const double* u, double* inc) {
  if (c.nv < 5) return;
  if (u[4] + inc[4] < 0) {
    const double declineV = inc[4] / (u[4] + 1e-6);
    const double newu5 = std::max(1e-6, u[4] * std::exp(declineV));
    inc[4] = newu5 - u[4];
  }
}

// LUSGSMatrixInit (DNDS_FV_EulerEvaluator.cpp:995-1047), jacobianCode 0:
// D_i = 1/dTau_i + 1/dt + sum_f (alpha/2) A_f lambdaFace_f / V_i, kept as its inverse
void lusgs_matrix_init(orc_ctx& c, const double* dTau, double dt, double alpha) {
  const int nv = c.nv;
  c.Dinv.assign(c.N * nv, 0.0);
  c.Dmat.assign(c.N * nv, 0.0);
  const bool src = c.srcJac.size() == (size_t)(c.N * nv);
  for (int64_t i = 0; i < c.N; i++) {
    const CellGeo& g = c.cg[i];
    double d = 1.0 / dTau[i] + 1.0 / dt;
    for (int k = 0; k < g.nface; k++) {
      const int f = g.faces[k];
      d += (0.5 * alpha) * c.fg[f].area * c.lambdaFace[f] / g.vol;
    }
    // + alpha * jacobianCellSourceDiag, kept diagonal
    for (int v = 0; v < nv; v++) {
      c.Dmat[i * nv + v] = d + (src ? alpha * c.srcJac[i * nv + v] : 0.0);
      c.Dinv[i * nv + v] = 1.0 / c.Dmat[i * nv + v];
    }
  }
}

// the off-diagonal sum of UpdateLUSGSForward / Backward (DNDS_FV_EulerEvaluator.cpp:1149-1357)
// over the neighbours j with scan position before (forward) or after (backward) cell i.  With a
// partition (the reference run on several MPI ranks): a neighbour in another part is a ghost, whose
// scan position counts as after every local cell (iScanOther = iScan + 1, :1177-1181, 1313-1317): it
// enters the backward sweep only, with its value as pulled after the forward sweep (ghostInc)
void lusgs_offdiag(const orc_ctx& c, int64_t i, int64_t si, const std::vector<int64_t>& pos, bool forward,
                   double alpha, const double* inc, double* buf, const double* ghostInc = nullptr) {
  const CellGeo& g = c.cg[i];
  const bool parts = !c.lusgsPart.empty();
  for (int k = 0; k < g.nface; k++) {
    const int f = g.faces[k];
    const FaceGeo& fg = c.fg[f];
    const int64_t j = fg.L == i ? fg.R : fg.L;
    if (j < 0) continue;
    const bool ghost = parts && c.lusgsPart[j] != c.lusgsPart[i];
    if (ghost ? forward : (forward ? !(pos[j] < si) : !(pos[j] > si))) continue;
    const double nn = std::sqrt(sqr(fg.ncenter[0]) + sqr(fg.ncenter[1]));
    const double sg = fg.L == i ? 1.0 : -1.0;  // faces out of i
    const double n[2] = {sg * fg.ncenter[0] / nn, sg * fg.ncenter[1] / nn};
    const int nv = c.nv;
    double dF[kMaxV];
    flux_jac_times_du(&c.u[j * nv], n, ghost ? &ghostInc[j * nv] : &inc[j * nv], c.lambdaFace[f], c.s.gamma, dF,
                      nv);
    for (int v = 0; v < nv; v++) buf[v] -= (0.5 * alpha) * fg.area / g.vol * dF[v];
  }
}

void scan_positions(const orc_ctx& c, const int64_t* scan2cell, std::vector<int64_t>& order,
                    std::vector<int64_t>& pos) {
  order.resize(c.N);
  pos.resize(c.N);
  for (int64_t s = 0; s < c.N; s++) order[s] = scan2cell ? scan2cell[s] : s;
  for (int64_t s = 0; s < c.N; s++) pos[order[s]] = s;
}

// forward then backward sweep in place on inc (the reference calls both with uInc == uIncNew)
void lusgs_sweeps(const orc_ctx& c, double alpha, const double* rhs, double* inc, const int64_t* scan2cell,
                  bool doForward, bool doBackward) {
  std::vector<int64_t> order, pos;
  scan_positions(c, scan2cell, order, pos);
  if (doForward)
    for (int64_t s = 0; s < c.N; s++) {
      const int64_t i = order[s];
      const int nv = c.nv;
      double buf[kMaxV];
      for (int v = 0; v < nv; v++) buf[v] = rhs[i * nv + v];
      lusgs_offdiag(c, i, s, pos, true, alpha, inc, buf);
      for (int v = 0; v < nv; v++) inc[i * nv + v] = c.Dinv[i * nv + v] * buf[v];
    }
  if (doBackward) {
    std::vector<double> ghostInc;  // the ghosts' increments as pulled after the forward sweep
    if (!c.lusgsPart.empty()) ghostInc.assign(inc, inc + c.N * c.nv);
    for (int64_t s = c.N - 1; s >= 0; s--) {
      const int64_t i = order[s];
      const int nv = c.nv;
      double buf[kMaxV] = {0};
      lusgs_offdiag(c, i, s, pos, false, alpha, inc, buf, ghostInc.data());
      for (int v = 0; v < nv; v++) inc[i * nv + v] += c.Dinv[i * nv + v] * buf[v];
    }
  }
}


// LUSGSMatrixVec (DNDS_FV_EulerEvaluator.cpp:1062-1143): Ax_i = D_i x_i - buf,
// buf -= (alpha/2) A_f / V_i fluxJacobian0_Right_Times_du(u_j, n_out, x_j) over every neighbour
void lusgs_matvec(const orc_ctx& c, double alpha, const double* x, double* Ax) {
  const int nv = c.nv;
  for (int64_t i = 0; i < c.N; i++) {
    const CellGeo& g = c.cg[i];
    double buf[kMaxV] = {0};
    for (int k = 0; k < g.nface; k++) {
      const int f = g.faces[k];
      const FaceGeo& fg = c.fg[f];
      const int64_t j = fg.L == i ? fg.R : fg.L;
      if (j < 0) continue;
      const double nn = std::sqrt(sqr(fg.ncenter[0]) + sqr(fg.ncenter[1]));
      const double sg = fg.L == i ? 1.0 : -1.0;
      const double n[2] = {sg * fg.ncenter[0] / nn, sg * fg.ncenter[1] / nn};
      double dF[kMaxV];
      flux_jac_times_du(&c.u[j * nv], n, &x[j * nv], c.lambdaFace[f], c.s.gamma, dF, nv);
      for (int v = 0; v < nv; v++) buf[v] -= (0.5 * alpha) * fg.area / g.vol * dF[v];
    }
    for (int v = 0; v < nv; v++) Ax[i * nv + v] = c.Dmat[i * nv + v] * x[i * nv + v] - buf[v];
  }
}

double vdot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (size_t k = 0; k < a.size(); k++) s += a[k] * b[k];
  return s;
}

// least squares min |H y - rhs| for an m x n matrix (row-major) by Householder QR
void lsq_householder(std::vector<double> H, int m, int n, std::vector<double> rhs, double* y) {
  for (int j = 0; j < n; j++) {
    double nrm = 0;
    for (int i = j; i < m; i++) nrm += H[i * n + j] * H[i * n + j];
    nrm = std::sqrt(nrm);
    if (nrm == 0) continue;
    const double alpha = H[j * n + j] > 0 ? -nrm : nrm;
    std::vector<double> v(m, 0.0);
    for (int i = j; i < m; i++) v[i] = H[i * n + j];
    v[j] -= alpha;
    double vv = 0;
    for (int i = j; i < m; i++) vv += v[i] * v[i];
    if (vv == 0) continue;
    for (int q = j; q < n; q++) {
      double d = 0;
      for (int i = j; i < m; i++) d += v[i] * H[i * n + q];
      for (int i = j; i < m; i++) H[i * n + q] -= 2 * d / vv * v[i];
    }
    double d = 0;
    for (int i = j; i < m; i++) d += v[i] * rhs[i];
    for (int i = j; i < m; i++) rhs[i] -= 2 * d / vv * v[i];
  }
  for (int j = n - 1; j >= 0; j--) {
    double r = rhs[j];
    for (int q = j + 1; q < n; q++) r -= H[j * n + q] * y[q];
    y[j] = r / H[j * n + j];
  }
}

// GMRES_LeftPreconditioned::solve (DNDS_Linear.hpp:47-105) with the EulerSolver's FStop (never
// stops early): FA = LUSGSMatrixVec, FML = LU-SGS forward + backward with the argument as rhs
void gmres_solve(const orc_ctx& c, int K, int nRestart, double alpha, const std::vector<double>& b,
                 std::vector<double>& x, const int64_t* scan2cell) {
  const size_t n = b.size();
  auto FML = [&](const std::vector<double>& in, std::vector<double>& out) {
    out.assign(n, 0.0);
    lusgs_sweeps(c, alpha, in.data(), out.data(), scan2cell, true, true);
  };
  std::vector<double> MLb, tmp(n);
  std::vector<std::vector<double>> V(K + 1, std::vector<double>(n));
  FML(b, MLb);
  for (int iRestart = 0; iRestart <= nRestart; iRestart++) {
    lusgs_matvec(c, alpha, x.data(), tmp.data());
    FML(tmp, V[0]);
    for (size_t e = 0; e < n; e++) V[0][e] += MLb[e] * -1.0;
    const double beta = std::sqrt(vdot(V[0], V[0]));
    if (std::abs(beta) < 1e-200 || iRestart == nRestart) break;
    for (size_t e = 0; e < n; e++) V[0][e] *= -1.0 / beta;
    std::vector<double> h((size_t)(K + 1) * K, 0.0);  // row-major (K+1) x K
    for (int j = 0; j < K; j++) {
      lusgs_matvec(c, alpha, V[j].data(), tmp.data());
      FML(tmp, V[j + 1]);
      for (int i = 0; i <= j; i++) h[i * K + j] = vdot(V[j + 1], V[i]);
      for (int i = 0; i <= j; i++)
        for (size_t e = 0; e < n; e++) V[j + 1][e] += V[i][e] * -h[i * K + j];
      h[(j + 1) * K + j] = std::sqrt(vdot(V[j + 1], V[j + 1]));
      for (size_t e = 0; e < n; e++) V[j + 1][e] *= 1.0 / h[(j + 1) * K + j];
    }
    std::vector<double> eb(K + 1, 0.0), y(K);
    eb[0] = beta;
    lsq_householder(h, K + 1, K, eb, y.data());
    for (int j = 0; j < K; j++)
      for (size_t e = 0; e < n; e++) x[e] += V[j][e] * y[j];
  }
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int orc_create(const orc_mesh* mesh, const orc_settings* s, orc_ctx** out) {
  if (!mesh || !s || !out) return 1;
  auto* c = new orc_ctx();
  c->s = *s;
  c->nv = s->nvars;
  if (c->nv != 4 && c->nv != 5) { c->err = "nvars must be 4 (NS_2D) or 5 (NS_2D with SA)"; *out = c; return 2; }
  if (c->nv == 5 && !(s->mu_gas > 0)) { c->err = "the SA model needs mu_gas > 0"; *out = c; return 2; }
  if (s->rec_order != 2) { c->err = "only rec_order=2 (P2) is restated"; *out = c; return 2; }
  c->nthreads = s->n_threads > 0 ? s->n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
  int rc = setup(*c, *mesh);
  if (rc == 0 && c->nv == 5) wall_distance(*c, *mesh);
  *out = c;
  return rc;
}

void orc_destroy(orc_ctx* c) { delete c; }
const char* orc_last_error(orc_ctx* c) { return c ? c->err.c_str() : "null ctx"; }

int orc_set_u(orc_ctx* c, const double* u) { std::memcpy(c->u.data(), u, sizeof(double) * c->N * c->nv); return 0; }
int orc_get_u(orc_ctx* c, double* u) { std::memcpy(u, c->u.data(), sizeof(double) * c->N * c->nv); return 0; }
int orc_set_urec(orc_ctx* c, const double* r) { std::memcpy(c->urec.data(), r, sizeof(double) * c->N * 5 * c->nv); return 0; }
int orc_get_urec(orc_ctx* c, double* r) { std::memcpy(r, c->urec.data(), sizeof(double) * c->N * 5 * c->nv); return 0; }

int orc_get_geometry(orc_ctx* c, double* vol, double* bary, double* area) {
  for (int64_t i = 0; i < c->N; i++) {
    if (vol) vol[i] = c->cg[i].vol;
    if (bary) { bary[2 * i] = c->cg[i].bary[0]; bary[2 * i + 1] = c->cg[i].bary[1]; }
  }
  if (area) for (int64_t f = 0; f < c->F; f++) area[f] = c->fg[f].area;
  return 0;
}

int orc_init_isentropic_vortex(orc_ctx* c) {
  Quad q3 = tri4(), q4 = quad9();
  for (int64_t i = 0; i < c->N; i++) {
    const CellGeo& g = c->cg[i];
    const Quad& q = g.nn == 3 ? q3 : q4;
    double um[4] = {0, 0, 0, 0};
    for (int ig = 0; ig < q.n; ig++) {
      double N[4], dN[2][4];
      shape(g.nn, q.p[ig][0], q.p[ig][1], N, dN);
      double x = 0, y = 0, J[2][2] = {{0, 0}, {0, 0}};
      for (int k = 0; k < g.nn; k++) {
        x += N[k] * g.xy[k][0]; y += N[k] * g.xy[k][1];
        for (int d = 0; d < 2; d++) { J[d][0] += dN[d][k] * g.xy[k][0]; J[d][1] += dN[d][k] * g.xy[k][1]; }
      }
      double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      double U[4];
      vortex_state(x, y, 5, 5, c->s.gamma, true, U);
      for (int k = 0; k < 4; k++) um[k] += U[k] * det * q.w[ig];
    }
    for (int k = 0; k < 4; k++) c->u[i * c->nv + k] = um[k] / g.vol;
  }
  return 0;
}

int orc_exact_isentropic_vortex(orc_ctx* c, double t, double* out) {
  // exact solution on the periodic [0,10]^2 domain: the vortex centre moves by (t, t)
  Quad q3 = tri4(), q4 = quad9();
  for (int64_t i = 0; i < c->N; i++) {
    const CellGeo& g = c->cg[i];
    const Quad& q = g.nn == 3 ? q3 : q4;
    double um[4] = {0, 0, 0, 0};
    for (int ig = 0; ig < q.n; ig++) {
      double N[4], dN[2][4];
      shape(g.nn, q.p[ig][0], q.p[ig][1], N, dN);
      double x = 0, y = 0, J[2][2] = {{0, 0}, {0, 0}};
      for (int k = 0; k < g.nn; k++) {
        x += N[k] * g.xy[k][0]; y += N[k] * g.xy[k][1];
        for (int d = 0; d < 2; d++) { J[d][0] += dN[d][k] * g.xy[k][0]; J[d][1] += dN[d][k] * g.xy[k][1]; }
      }
      double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      double xc = std::fmod(5 + t, 10.0), yc = std::fmod(5 + t, 10.0);
      // nearest periodic image of the centre
      double dx = x - xc, dy = y - yc;
      dx -= 10.0 * std::round(dx / 10.0); dy -= 10.0 * std::round(dy / 10.0);
      double U[4];
      vortex_state(xc + dx, yc + dy, xc, yc, c->s.gamma, true, U);
      for (int k = 0; k < 4; k++) um[k] += U[k] * det * q.w[ig];
    }
    for (int k = 0; k < 4; k++) out[i * c->nv + k] = um[k] / g.vol;
  }
  return 0;
}

int orc_init_quadrants(orc_ctx* c, double xs, double ys, const double* q) {
  for (int64_t i = 0; i < c->N; i++) {
    double x = c->cg[i].bary[0], y = c->cg[i].bary[1];
    int k = (x > xs) ? ((y > ys) ? 0 : 3) : ((y > ys) ? 1 : 2);
    prim2cons(&q[4 * k], &c->u[i * c->nv], c->s.gamma);
  }
  return 0;
}

int orc_vr_step(orc_ctx* c, int nsweeps) {
  for (int k = 0; k < nsweeps; k++) vr_sweep(*c);
  return 0;
}
double orc_vr_last_increment(orc_ctx* c) { return c->lastInc; }

int orc_limiter_wbap_v2(orc_ctx* c, int if_all, double* ind) {
  limiter_wbap_v2(*c, if_all != 0, ind);
  return 0;
}
int orc_limiter_wbap(orc_ctx* c, int if_all, double* ind) {
  limiter_wbap(*c, if_all != 0, ind);
  return 0;
}

int orc_eval_dt(orc_ctx* c, double cfl, double max_dt, int use_local, double* dt_out, double* dt_min) {
  eval_dt(*c, cfl, max_dt, use_local != 0, dt_min);
  if (dt_out) std::memcpy(dt_out, c->dtCell.data(), sizeof(double) * c->N);
  return 0;
}

int orc_eval_rhs(orc_ctx* c, double t, double* rhs_out, double* wall_flux) {
  eval_rhs(*c, t, rhs_out, wall_flux, nullptr);
  return 0;
}

int orc_face_values(orc_ctx* c, double t, double* out) {
  parallel_for(c->nthreads, c->F, [&](int64_t b, int64_t e) {
    for (int64_t f = b; f < e; f++) {
      double fl[3][kMaxV];
      face_flux(*c, f, t, fl, &out[f * 6 * c->nv], nullptr);
    }
  });
  return 0;
}

// frhs (DNDS_FV_EulerSolver.hpp:713-837) composed with
// ExplicitSSPRK3LocalDt::Step (DNDS_ODE.hpp:131-177); the dt comes from the
// caller (EvaluateDt with UseLocaldt=false, clipped to t_end)
int orc_ssprk3_step(orc_ctx* c, double dt, double t) {
  const int64_t n = c->N * c->nv;
  std::vector<double> xLast = c->u, rhs(n);
  const double cst[3] = {0.0, 1.0, 0.5};
  const double coef[3] = {1.0, 0.25, 2.0 / 3.0};
  for (int st = 0; st < 3; st++) {
    vr_sweep(*c);
    if (c->s.limiter) limiter_stage(*c);
    eval_rhs(*c, t + cst[st] * dt, rhs.data(), nullptr, nullptr);
    for (int64_t k = 0; k < n; k++) rhs[k] *= dt;
    for (int64_t k = 0; k < n; k++) c->u[k] += rhs[k];
    if (st > 0) {
      double cf = coef[st];
      for (int64_t k = 0; k < n; k++) {
        double x = c->u[k] * (cf / (1 - cf));
        x += xLast[k];
        c->u[k] = x * (1 - cf);
      }
    }
  }
  return 0;
}

int orc_residual(orc_ctx* c, const double* rhs, int p, int vol_wise, double* out) {
  const int nv = c->nv;
  for (int k = 0; k < nv; k++) out[k] = 0;
  if (p < 3) {
    for (int64_t i = 0; i < c->N; i++)
      for (int k = 0; k < nv; k++) {
        double v = std::pow(std::fabs(rhs[i * nv + k]), double(p));
        out[k] += vol_wise ? v * c->cg[i].vol : v;
      }
    for (int k = 0; k < nv; k++) out[k] = std::pow(out[k], 1.0 / p);
  } else {
    for (int64_t i = 0; i < c->N; i++)
      for (int k = 0; k < nv; k++) out[k] = std::max(out[k], std::fabs(rhs[i * nv + k]));
  }
  return 0;
}

int orc_lusgs_matrix_init(orc_ctx* c, const double* dtau, double dt, double alpha) {
  std::vector<double> d(c->N);
  for (int64_t i = 0; i < c->N; i++) d[i] = dtau ? dtau[i] : c->dtCell[i] / alpha;
  lusgs_matrix_init(*c, d.data(), dt, alpha);
  return 0;
}

int orc_lusgs_forward(orc_ctx* c, double alpha, const double* rhs, double* inc, const int64_t* scan2cell) {
  if (c->Dinv.size() != (size_t)(c->N * c->nv)) return 1;
  lusgs_sweeps(*c, alpha, rhs, inc, scan2cell, true, false);
  return 0;
}

int orc_lusgs_backward(orc_ctx* c, double alpha, const double* rhs, double* inc, const int64_t* scan2cell) {
  if (c->Dinv.size() != (size_t)(c->N * c->nv)) return 1;
  lusgs_sweeps(*c, alpha, rhs, inc, scan2cell, false, true);
  return 0;
}

// one pseudo-time iteration of ImplicitBDFDualTimeStep::Step (DNDS_ODE.hpp:444-486) at BDF order 1
// with the EulerSolver lambdas fdtau / frhs / fsolve (DNDS_FV_EulerSolver.hpp:713-925):
// dTau = EvaluateDt(CFL, local)/alpha; nInternalRecStep Jacobi sweeps; [limiter]; EvaluateRHS;
// rhs = alpha R - (x - xLast)/dt; LU-SGS forward + backward from zero; x += inc
int orc_implicit_iteration(orc_ctx* c, double cfl, double dt, double alpha, const double* x_last,
                           const int64_t* scan2cell, double t, int n_rec, double* inc_out) {
  const int64_t n = c->N * c->nv;
  double dtMin;
  eval_dt(*c, cfl, 1e100, true, &dtMin);
  std::vector<double> dTau(c->N), rhs(n), inc(n, 0.0);
  for (int64_t i = 0; i < c->N; i++) dTau[i] = c->dtCell[i] / alpha;
  for (int k = 0; k < n_rec; k++) vr_sweep(*c);
  if (c->s.limiter) limiter_stage(*c);
  eval_rhs(*c, t, rhs.data(), nullptr, nullptr);
  for (int64_t k = 0; k < n; k++) {
    rhs[k] *= alpha;
    rhs[k] += -c->u[k] / dt;
    rhs[k] += x_last[k] / dt;
  }
  lusgs_matrix_init(*c, dTau.data(), dt, alpha);
  const int nv = c->nv;
  // fsolve's positivity fixes (DNDS_FV_EulerSolver.hpp:874-912): CompressInc on rhs * dTau, then
  // on the increment
  for (int64_t i = 0; i < c->N; i++) {
    double r[kMaxV];
    for (int v = 0; v < nv; v++) r[v] = rhs[i * nv + v] * dTau[i];
    compress_inc(*c, &c->u[i * nv], r);
    for (int v = 0; v < nv; v++) rhs[i * nv + v] = r[v] / dTau[i];
  }
  lusgs_sweeps(*c, alpha, rhs.data(), inc.data(), scan2cell, true, true);
  for (int64_t i = 0; i < c->N; i++) compress_inc(*c, &c->u[i * nv], &inc[i * nv]);
  for (int64_t k = 0; k < n; k++) c->u[k] += inc[k];
  if (inc_out) std::memcpy(inc_out, inc.data(), sizeof(double) * n);
  return 0;
}

int orc_set_lusgs_parts(orc_ctx* c, const int32_t* part) {
  if (!part) c->lusgsPart.clear();
  else c->lusgsPart.assign(part, part + c->N);
  return 0;
}

int orc_lusgs_matvec(orc_ctx* c, double alpha, const double* x, double* ax) {
  if (c->Dmat.size() != (size_t)(c->N * c->nv)) return 1;
  lusgs_matvec(*c, alpha, x, ax);
  return 0;
}

int orc_gmres_lusgs(orc_ctx* c, double alpha, int n_space, int n_restart, const double* b, double* x,
                    const int64_t* scan2cell) {
  if (c->Dmat.size() != (size_t)(c->N * c->nv) || n_space < 1) return 1;
  const size_t n = (size_t)(c->N * c->nv);
  std::vector<double> bv(b, b + n), xv(x, x + n);
  gmres_solve(*c, n_space, n_restart, alpha, bv, xv, scan2cell);
  std::memcpy(x, xv.data(), sizeof(double) * n);
  return 0;
}

int orc_dual_reset(orc_ctx* c) {
  c->odeOrder = c->odeCnPrev = c->odePrevStart = 0;
  c->odeDtPrev = 0;
  return 0;
}

// one physical step of ImplicitBDFDualTimeStep (order k, DNDS_ODE.hpp:392-497) or
// ImplicitSDIRK4DualTimeStep (DNDS_ODE.hpp:269-390) with the EulerSolver lambdas
// (DNDS_FV_EulerSolver.hpp:713-1061): fdtau = local EvaluateDt / alphaDiag; frhs = Jacobi sweeps,
// [limiter], EvaluateRHS at t + ct dt; fsolve = LUSGSMatrixInit, CompressInc of rhs dTau, LU-SGS
// and / or GMRES, CompressInc of the increment; fstop = the L1 (volume-weighted) increment norm
// over its running maximum, density entry against the threshold
int orc_dual_step(orc_ctx* c, const orc_dual_settings* d, double dt, double t, const int64_t* scan2cell,
                  int* iters_out, double* res_out) {
  static const double bdf[4][5] = {{1.0, 1.0, 0, 0, 0},
                                   {2. / 3., 4. / 3., -1. / 3., 0, 0},
                                   {6. / 11., 18. / 11., -9. / 11., 2. / 11., 0},
                                   {12. / 25., 48. / 25., -36. / 25., 16. / 25., -3. / 25.}};
  const double z = 0.128886400515;
  const double A[3][3] = {{z, 0, 0}, {0.5 - z, z, 0}, {2 * z, 1 - 4 * z, z}};
  const double C[3] = {z, 0.5, 1 - z};
  const double B[3] = {1. / (6 * sqr(2 * z - 1)), (4 * sqr(z) - 4 * z + 2. / 3.) / sqr(2 * z - 1),
                       1. / (6 * sqr(2 * z - 1))};
  const int nv = c->nv;
  const int64_t n = c->N * nv;
  const bool bdfScheme = d->scheme == 1;
  if (bdfScheme && (d->bdf_order < 1 || d->bdf_order > 4)) return 1;
  if (bdfScheme && c->odeOrder != d->bdf_order) {
    c->odeOrder = d->bdf_order;
    c->odeCnPrev = 0;
    c->odePrevStart = std::max(0, d->bdf_order - 2);
  }
  const size_t nOde = bdfScheme ? (size_t)(d->bdf_order - 1) : 3;
  while (c->odeVec.size() < nOde) c->odeVec.emplace_back(n, 0.0);
  std::vector<double> xLast = c->u, rhs(n), inc(n), dTau(c->N);
  double base[kMaxV] = {0}, rel[kMaxV] = {0};
  // one internal iteration; true when fstop says stop
  auto iteration = [&](int iter, double alphaDiag, double ct, const std::function<void(std::vector<double>&)>& compose) {
    double dtMin;
    eval_dt(*c, d->cfl, 1e100, true, &dtMin);
    for (int64_t i = 0; i < c->N; i++) dTau[i] = c->dtCell[i] / alphaDiag;
    for (int k = 0; k < d->n_rec; k++) vr_sweep(*c);
    if (c->s.limiter) limiter_stage(*c);
    eval_rhs(*c, t + ct * dt, rhs.data(), nullptr, nullptr);
    compose(rhs);
    lusgs_matrix_init(*c, dTau.data(), dt, alphaDiag);
    for (int64_t i = 0; i < c->N; i++) {
      double r[kMaxV] = {};
      for (int v = 0; v < nv; v++) r[v] = rhs[i * nv + v] * dTau[i];
      compress_inc(*c, &c->u[i * nv], r);
      for (int v = 0; v < nv; v++) rhs[i * nv + v] = r[v] / dTau[i];
    }
    std::fill(inc.begin(), inc.end(), 0.0);
    if (d->gmres_code == 0 || d->gmres_code == 2) {
      lusgs_sweeps(*c, alphaDiag, rhs.data(), inc.data(), scan2cell, true, true);
      for (int64_t i = 0; i < c->N; i++) compress_inc(*c, &c->u[i * nv], &inc[i * nv]);
    }
    if (d->gmres_code != 0) {
      gmres_solve(*c, d->n_gmres_space, d->n_gmres_iter, alphaDiag, rhs, inc, scan2cell);
      for (int64_t i = 0; i < c->N; i++) compress_inc(*c, &c->u[i * nv], &inc[i * nv]);
    }
    double res[kMaxV] = {0};
    for (int64_t i = 0; i < c->N; i++)
      for (int v = 0; v < nv; v++) res[v] += std::abs(inc[i * nv + v]) * (d->vol_wise ? c->cg[i].vol : 1.0);
    for (int64_t k = 0; k < n; k++) c->u[k] += inc[k];
    for (int v = 0; v < nv; v++) {
      base[v] = iter == 1 ? res[v] : std::max(base[v], res[v]);
      rel[v] = res[v] / base[v];
    }
    return rel[0] < d->threshold;
  };
  if (bdfScheme) {
    const int prevSiz = d->bdf_order - 1, kCur = c->odeCnPrev + 1;
    if (c->odeCnPrev > 0 && !(std::abs(c->odeDtPrev - dt) < dt * 1e-8)) return 1;
    int iter = 1;
    for (; iter <= d->max_iter; iter++) {
      const bool stop = iteration(iter, bdf[kCur - 1][0], 1.0, [&](std::vector<double>& r) {
        for (int64_t k = 0; k < n; k++) {
          r[k] *= bdf[kCur - 1][0];
          r[k] += c->u[k] * (-1. / dt);
          r[k] += xLast[k] * (bdf[kCur - 1][1] / dt);
          for (int ip = 0; ip < c->odeCnPrev; ip++)
            r[k] += c->odeVec[(ip + c->odePrevStart) % prevSiz][k] * (bdf[kCur - 1][2 + ip] / dt);
        }
      });
      if (stop) break;
    }
    if (iters_out) iters_out[0] = std::min(iter, d->max_iter);
    if (prevSiz) {
      c->odePrevStart = ((c->odePrevStart - 1) % prevSiz + prevSiz) % prevSiz;
      c->odeVec[c->odePrevStart] = xLast;
      c->odeDtPrev = dt;
      c->odeCnPrev = std::min(c->odeCnPrev + 1, prevSiz);
    }
  } else {
    for (int iB = 0; iB < 3; iB++) {
      c->u = xLast;
      int iter = 1;
      for (; iter <= d->max_iter; iter++) {
        const bool stop = iteration(iter, A[iB][iB], C[iB], [&](std::vector<double>& r) {
          c->odeVec[iB] = r;
          for (int64_t k = 0; k < n; k++) {
            double v = xLast[k];
            v -= c->u[k];
            v *= 1.0 / dt;
            for (int jB = 0; jB <= iB; jB++) v += c->odeVec[jB][k] * A[iB][jB];
            r[k] = v;
          }
        });
        if (stop) break;
      }
      if (iters_out) iters_out[iB] = std::min(iter, d->max_iter);
    }
    c->u = xLast;
    for (int jB = 0; jB < 3; jB++)
      for (int64_t k = 0; k < n; k++) c->u[k] += c->odeVec[jB][k] * (B[jB] * dt);
  }
  if (res_out)
    for (int v = 0; v < nv; v++) res_out[v] = rel[v];
  return 0;
}

int orc_get_vr_blocks(orc_ctx* c, double* ainv, double* ainvb, double* ainv_b) {
  if (ainv) std::memcpy(ainv, c->Ainv.data(), sizeof(double) * c->N * 25);
  if (ainvb) std::memcpy(ainvb, c->AinvB.data(), sizeof(double) * c->N * 100);
  if (ainv_b) std::memcpy(ainv_b, c->Ainvb.data(), sizeof(double) * c->N * 20);
  return 0;
}

int orc_get_face_dibj(orc_ctx* c, double* out) {
  for (int64_t f = 0; f < c->F; f++) std::memcpy(&out[f * 216], c->fg[f].D, sizeof(double) * 216);
  return 0;
}

void orc_riemann_flux(int riemann, const double* ul, const double* ur, double gamma, double dlambda, double* f) {
  if (riemann == 2) hllc_flux(ul, ur, gamma, f);
  else roe_flux(ul, ur, gamma, f, dlambda);
}

}  // extern "C"
