// dndsg_sa.cuh -- the Spalart-Allmaras (SA-neg) model on the GPU, as the reference's NS_SA model
// restricted to 2-D (w = 0): a fifth conserved variable U5 = rho nu~ / muRef carried in its own
// arrays next to the unchanged 4-variable flow state, so that the flow kernels stay as they are.
//
//   VR sweep of U5                    ReconstructionJacobiStep, DNDS_FV_VR.hpp:1474-1713
//   face flux (flow with the eddy     fluxFace, DNDS_FV_EulerEvaluator.hpp:371-591
//     viscosity, U5 transport and
//     diffusion)
//   source and its diagonal Jacobian  source / sourceJacobianDiag, DNDS_FV_EulerEvaluator.hpp:593-864,
//     over the cell quadrature        integrated as in DNDS_FV_EulerEvaluator.cpp:520-638
//   first-order wall distance         DNDS_FV_EulerEvaluator.hpp:227-363 (USE_FIRST_ORDER_WALL_DIST)
//   EvaluateDt with the eddy viscosity DNDS_FV_EulerEvaluator.cpp:80-99
//   LU-SGS on 5 variables             DNDS_FV_EulerEvaluator.cpp:995-1357, .hpp:928-956
//   CompressInc                       DNDS_FV_EulerEvaluator.hpp:1362-1406
#pragma once
#include "dndsg_bodies.cuh"

namespace dg {

constexpr int kSaGp = 9;       // cell quadrature points per cell (QUAD_9; TRI_4 pads with zero weights)
constexpr int kSaGpE = 16;     // per point: weight x det J, value row (5), d/dx row (5), d/dy row (5)

template <class T>
struct SaView {
  double* u;             // [N] U5
  double* uLast;         // [N]
  const T* urec;         // [N][5]
  T* urecNew;            // [N][5]
  double* rhs;           // [N]
  double* flux;          // [F] integrated U5 face flux
  double* inc;           // [N] LU-SGS increment
  double* Dinv;          // [N] LU-SGS diagonal inverse of U5
  double* srcJac;        // [N] jacobianCellSourceDiag of U5
  const double* dWall;   // [N]
  const double* cellGp;  // [N][kSaGp][kSaGpE]
  double far5;           // farFieldStaticValue[4]
};

// SA eddy-viscosity factor (fluxFace, DNDS_FV_EulerEvaluator.hpp:413-425, SA-neg softening below 10)
DG_HD double sa_mu_factor(double U5, double muRef, double mufPhy) {
  const double cnu1 = 7.1;
  double Chi = U5 * muRef / mufPhy;
  if (Chi < 10) Chi = 0.05 * log(1 + exp(20 * Chi));
  const double Chi3 = Chi * Chi * Chi;
  const double fnu1 = Chi3 / (Chi3 + cnu1 * cnu1 * cnu1);
  return dmax(1 + Chi * fnu1, 1.0);
}

// cell quadrature of the reference (TRI_4 / QUAD_9, DNDS_Elements.hpp:326-430) and the Tri3 / Quad4
// shape functions (DNDS_Elements.hpp:1020-1090)
DG_HD int cell_gp(int nn, int ig, double& xi, double& eta, double& w) {
  if (nn == 3) {
    const double P[4][2] = {{1. / 3., 1. / 3.}, {0.6, 0.2}, {0.2, 0.6}, {0.2, 0.2}};
    const double W[4] = {-27. / 96., 25. / 96., 25. / 96., 25. / 96.};
    if (ig >= 4) return 0;
    xi = P[ig][0]; eta = P[ig][1]; w = W[ig];
    return 1;
  }
  const double a = sqrt(0.6);
  const double l[3] = {-a, 0.0, a}, lw[3] = {5. / 9., 8. / 9., 5. / 9.};
  xi = l[ig % 3]; eta = l[ig / 3]; w = lw[ig % 3] * lw[ig / 3];
  return 1;
}

// per cell: weight x det J and the basis value / gradient rows at each cell quadrature point
DG_HD void setup_sa_cell_gp(int64_t i, const CellSetup* cells, double* gp) {
  const CellSetup& c = cells[i];
  for (int ig = 0; ig < kSaGp; ig++) {
    double* o = &gp[(i * kSaGp + ig) * kSaGpE];
    double xi, eta, w;
    if (!cell_gp(c.nn, ig, xi, eta, w)) {
      for (int e = 0; e < kSaGpE; e++) o[e] = 0;
      continue;
    }
    double N[4], dN[2][4];
    if (c.nn == 3) {
      N[0] = 1 - xi - eta; N[1] = xi; N[2] = eta; N[3] = 0;
      dN[0][0] = -1; dN[0][1] = 1; dN[0][2] = 0; dN[0][3] = 0;
      dN[1][0] = -1; dN[1][1] = 0; dN[1][2] = 1; dN[1][3] = 0;
    } else {
      N[0] = (1 - xi) * (1 - eta) * 0.25; N[1] = (1 + xi) * (1 - eta) * 0.25;
      N[2] = (1 + xi) * (1 + eta) * 0.25; N[3] = (1 - xi) * (1 + eta) * 0.25;
      dN[0][0] = -(1 - eta) * 0.25; dN[0][1] = (1 - eta) * 0.25; dN[0][2] = (1 + eta) * 0.25; dN[0][3] = -(1 + eta) * 0.25;
      dN[1][0] = -(1 - xi) * 0.25; dN[1][1] = -(1 + xi) * 0.25; dN[1][2] = (1 + xi) * 0.25; dN[1][3] = (1 - xi) * 0.25;
    }
    double x = 0, y = 0, J[2][2] = {{0, 0}, {0, 0}};
    for (int k = 0; k < c.nn; k++) {
      x += N[k] * c.xy[k][0]; y += N[k] * c.xy[k][1];
      for (int d = 0; d < 2; d++) { J[d][0] += dN[d][k] * c.xy[k][0]; J[d][1] += dN[d][k] * c.xy[k][1]; }
    }
    o[0] = w * (J[0][0] * J[1][1] - J[0][1] * J[1][0]);
    double D[6][5];
    p2_diffs(c.fr, x, y, D);
    for (int r = 0; r < 3; r++)
      for (int k = 0; k < 5; k++) o[1 + r * 5 + k] = D[r][k];
  }
}

// first-order wall distance: from the cell barycentre to the nearest wall segment [nw][4]
DG_HD double sa_wall_distance(double px, double py, const double* seg, int64_t nw) {
  double best = pow(3e200, 1. / 6.);
  for (int64_t s = 0; s < nw; s++) {
    const double x1 = seg[4 * s], y1 = seg[4 * s + 1], x2 = seg[4 * s + 2], y2 = seg[4 * s + 3];
    const double ex = x2 - x1, ey = y2 - y1, L2 = sqrt(ex * ex + ey * ey);
    const double bx = px - x1, by = py - y1, LB = (bx * ex + by * ey) / L2;
    double d;
    if (LB >= 0 && LB <= L2) {
      const double qx = bx - LB * ex / L2, qy = by - LB * ey / L2;
      d = sqrt(qx * qx + qy * qy);
    } else {
      d = dmin(sqrt(bx * bx + by * by), sqrt((px - x2) * (px - x2) + (py - y2) * (py - y2)));
    }
    best = dmin(best, d);
  }
  return best;
}

// the VR sweep of U5: the reference's sweep for one variable, wall corrections included
// (a no-slip wall holds U5 = 0, USE_FIX_ZERO_SA_NUT_AT_WALL; a slip wall keeps the inner value)
template <class T>
DG_HD void sa_vr_cell(int64_t i, const HotView<T>& h, const SaView<T>& sa) {
  const int E = h.nfmax * 30;
  const double ui = sa.u[i];
  double acc[5];
  const T* ri = &sa.urec[i * 5];
  for (int r = 0; r < 5; r++) acc[r] = (1 - h.relax) * (double)ri[r];
  for (int k = 0; k < h.nfmax; k++) {
    const int mode = h.vrMode[aos(i, k, h.nfmax)];
    if (mode == VR_EMPTY) continue;
    const int64_t j = h.vrNbr[aos(i, k, h.nfmax)];
    auto op = [&](int e) { return (double)h.vrOp[aos(i, k * 30 + e, E)]; };
    if (mode == VR_INNER || mode == VR_FAR) {
      const T* rj = &sa.urec[j * 5];
      for (int r = 0; r < 5; r++) {
        double s = 0;
        for (int q = 0; q < 5; q++) s += op(r * 5 + q) * (double)rj[q];
        acc[r] += h.relax * s;
      }
    }
    if (mode == VR_INNER || mode == VR_WALL) {
      const double du = mode == VR_INNER ? sa.u[j] - ui : 0.0 - ui;
      for (int r = 0; r < 5; r++) acc[r] += h.relax * du * op(25 + r);
    }
    if (mode == VR_WALLCORR) {
      const int32_t f = h.vrFace[aos(i, k, h.nfmax)];
      const double w0 = h.faceW0[f], area = h.faceArea[f];
      const bool noslip = h.faceBC[f] == BC_WALL_NOSLIP;
      double corr[5] = {0, 0, 0, 0, 0};
      const FaceBasisSide<T> fb(h.faceBasis, f, 0);
      for (int g = 0; g < 3; g++) {
        double phi[5], uBL = ui;
        T pg[5];
        fb.at(g, pg);
        for (int q = 0; q < 5; q++) {
          phi[q] = (double)pg[q];
          uBL += phi[q] * (double)ri[q];
        }
        const double uBV = noslip ? 0.0 : uBL;
        const double jw = 0.5 * area * l3_weight(g);
        for (int q = 0; q < 5; q++) corr[q] += phi[q] * w0 * w0 * (uBV - ui) * jw;
      }
      const double* Ai = &h.Ainv[i * 25];
      for (int r = 0; r < 5; r++) {
        double s = 0;
        for (int q = 0; q < 5; q++) s += Ai[r * 5 + q] * corr[q];
        acc[r] += h.relax * s;
      }
    }
  }
  for (int r = 0; r < 5; r++) sa.urecNew[i * 5 + r] = (T)acc[r];
}

// positivity-compressed flow and SA states at one face point, the SA boundary value, and the
// SA gradient (CompressRecPart replaces all five variables by the mean when the flow state is bad)
template <class T>
DG_HD void sa_point(const HotView<T>& h, const SaView<T>& sa, int64_t f, int g, int32_t L, int32_t R, bool inner,
                    const double uL[4], const double uR[4], const T incL[4], const T incR[4], double UL[4],
                    double UR[4], double& sL, double& sR, int& nred) {
  const double sLm = sa.u[L];
  double incS = 0;
  T pg[5];
  FaceBasisSide<T>(h.faceBasis, f, 0).at(g, pg);
  for (int q = 0; q < 5; q++) incS += (double)pg[q] * (double)sa.urec[(int64_t)L * 5 + q];
  double inc[4];
  for (int v = 0; v < 4; v++) inc[v] = (double)incL[v];
  bool cL = compress_rec_part(uL, inc, UL);
  sL = cL ? sLm : sLm + incS;
  nred += cL ? 1 : 0;
  if (inner) {
    double incSR = 0;
    FaceBasisSide<T>(h.faceBasis, f, 1).at(g, pg);
    for (int q = 0; q < 5; q++) incSR += (double)pg[q] * (double)sa.urec[(int64_t)R * 5 + q];
    for (int v = 0; v < 4; v++) inc[v] = (double)incR[v];
    bool cR = compress_rec_part(uR, inc, UR);
    sR = cR ? sa.u[R] : sa.u[R] + incSR;
    nred += cR ? 1 : 0;
  } else {
    const int bc = h.faceBC[f];
    const double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1];
    const double far[4] = {h.farU[0], h.farU[1], h.farU[2], h.farU[3]};
    boundary_value(bc, UL, nx, ny, h.faceCenter[2 * f], h.faceCenter[2 * f + 1], 0.0, h.gamma, far, UR);
    // the SA variable of generateBoundaryValue (DNDS_FV_EulerEvaluator.hpp:958-1275)
    if (bc == BC_FAR) {
      const double vn = (UL[1] * nx + UL[2] * ny) / UL[0];
      const double p = (h.gamma - 1) * (UL[3] - 0.5 * (UL[1] * UL[1] + UL[2] * UL[2]) / UL[0]);
      const double a = sqrt(h.gamma * p / UL[0]);
      sR = vn > 0 ? sL : sa.far5;  // outflow keeps the inner value, inflow takes the far one
      (void)a;
    } else if (bc == BC_WALL_NOSLIP) {
      sL = sR = 0.0;
    } else {
      sR = sL;
    }
  }
}

// the reconstruction increments of both cells at face Gauss point g (face_increments for one point,
// the same sums)
template <class T>
DG_HD void face_increment_point(int64_t f, int g, int32_t L, int32_t R, const HotView<T>& h, T incL[4], T incR[4]) {
  for (int v = 0; v < 4; v++) incL[v] = incR[v] = T(0);
  T phi[5];
  FaceBasisSide<T>(h.faceBasis, f, 0).at(g, phi);
  const T* rl = &h.urec[(int64_t)L * 20];
  for (int q = 0; q < 5; q++) {
    T row[4];
    load_row(rl + 4 * q, row);
    for (int v = 0; v < 4; v++) incL[v] += phi[q] * row[v];
  }
  if (R >= 0) {
    FaceBasisSide<T>(h.faceBasis, f, 1).at(g, phi);
    const T* rr = &h.urec[(int64_t)R * 20];
    for (int q = 0; q < 5; q++) {
      T row[4];
      load_row(rr + 4 * q, row);
      for (int v = 0; v < 4; v++) incR[v] += phi[q] * row[v];
    }
  }
}

// face flux of an SA context at Gauss point g: the flow flux with the eddy viscosity and the U5
// transport and diffusion (fluxFace, DNDS_FV_EulerEvaluator.hpp:371-591, SA branches), weighted;
// the face flux is minus the sum of the three points' c / cS in point order
template <class T, int RIEMANN, bool BND>
DG_HD int face_flux_sa_point(int64_t f, int g, const HotView<T>& h, const SaView<T>& sa, double c[4], double& cS,
                             bool& bad) {
  const int32_t L = h.faceL[f], R = h.faceR[f];
  const double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1], area = h.faceArea[f];
  double uL[4], uR[4] = {0, 0, 0, 0};
  load4<T>(&h.u[(int64_t)L * 4], uL);
  const bool inner = !BND || R >= 0;
  if (inner) load4<T>(&h.u[(int64_t)R * 4], uR);
  const int bc = BND ? h.faceBC[f] : BC_INNER;
  const bool wall = bc == BC_WALL_EULER || bc == BC_WALL_NOSLIP;
  double minVol = h.vol[L];
  if (inner) minVol = dmin(minVol, h.vol[R]);
  const double invD = wall ? 0.0 : area / (2.0 * minVol);
  const double dl = h.dLam[f];
  const double muRef = h.mu;
  T incL[4], incR[4];
  face_increment_point(f, g, L, inner ? R : -1, h, incL, incR);
  int nred = 0;
  {
    double UL[4], UR[4], a[4], b[4], F[4], sL, sR;
    sa_point(h, sa, f, g, L, R, inner, uL, uR, incL, incR, UL, UR, sL, sR, nred);
    to_normal_frame(UL, nx, ny, a);
    to_normal_frame(UR, nx, ny, b);
    if (!(a[0] > 0 && b[0] > 0)) bad = true;
    if (RIEMANN == 2) hllc_flux(a, b, h.gamma, F);
    else roe_flux(a, b, h.gamma, dl, F);
    from_normal_frame(F, nx, ny);
    double lam123;
    if (RIEMANN == 2) {
      lam123 = fabs(a[1] / a[0] + b[1] / b[0]) * 0.5;
    } else {
      const double qL = sqrt(a[0]), qR = sqrt(b[0]);
      lam123 = fabs((qL * a[1] / a[0] + qR * b[1] / b[0]) / (qL + qR));
    }
    double FS = ((a[1] / a[0] * sL + b[1] / b[0] * sR) - (sR - sL) * lam123) * 0.5;
    // gradients of the 5 variables at the point
    double GL[2][4], GR[2][4], G[2][4], Um[4], Fv[4], gS[2];
    face_grad(f, 0, g, L, h, GL);
    if (inner) face_grad(f, 1, g, R, h, GR);
    double gSL[2] = {0, 0}, gSR[2] = {0, 0};
    for (int d = 0; d < 2; d++)
      for (int q = 0; q < 5; q++) {
        gSL[d] += (double)h.faceGrad[aos(f, ((0 * 3 + g) * 2 + d) * 5 + q, 60)] * (double)sa.urec[(int64_t)L * 5 + q];
        if (inner)
          gSR[d] += (double)h.faceGrad[aos(f, ((1 * 3 + g) * 2 + d) * 5 + q, 60)] * (double)sa.urec[(int64_t)R * 5 + q];
      }
    for (int v = 0; v < 4; v++) {
      const double jump = invD * (UR[v] - UL[v]);
      G[0][v] = 0.5 * (GL[0][v] + (inner ? GR[0][v] : GL[0][v])) + jump * nx;
      G[1][v] = 0.5 * (GL[1][v] + (inner ? GR[1][v] : GL[1][v])) + jump * ny;
      Um[v] = 0.5 * (UL[v] + UR[v]);
    }
    const double jS = invD * (sR - sL);
    gS[0] = 0.5 * (gSL[0] + (inner ? gSR[0] : gSL[0])) + jS * nx;
    gS[1] = 0.5 * (gSL[1] + (inner ? gSR[1] : gSL[1])) + jS * ny;
    const double Sm = 0.5 * (sL + sR);
    const double pm = (h.gamma - 1) * (Um[3] - 0.5 * (Um[1] * Um[1] + Um[2] * Um[2]) / Um[0]);
    const double mufPhy = sutherland_mu(h, pm, Um[0]);
    const double muf = mufPhy * sa_mu_factor(Sm, muRef, mufPhy);
    const double kc = h.cp * (muf - mufPhy) / 0.9 + h.cp * mufPhy / h.pr;
    viscous_flux_n(Um, G, nx, ny, bc == BC_WALL_NOSLIP, h.gamma, muf, kc, h.cp, Fv);
    // the U5 diffusion (DNDS_FV_EulerEvaluator.hpp:463-480)
    double fn = 1;
    if (Sm < 0) {
      const double Chi = Sm * muRef / mufPhy, cn1 = 16;
      fn = (cn1 + Chi * Chi * Chi) / (cn1 - Chi * Chi * Chi);
    }
    double FvS = 0;
    const double gn[2] = {nx, ny};
    for (int d = 0; d < 2; d++) {
      const double diffNu = (gS[d] * muRef - Sm * muRef / Um[0] * G[d][0]) / Um[0];
      FvS += gn[d] * diffNu * (mufPhy + Sm * muRef * fn) / (2. / 3.) / muRef;
    }
    const double jw = 0.5 * area * l3_weight(g);
    for (int k = 0; k < 4; k++) c[k] = (F[k] - Fv[k]) * jw;
    cS = (FS - FvS) * jw;
  }
  return nred;
}

// the SA source and its diagonal Jacobian at one point (source / sourceJacobianDiag for NS_SA,
// DNDS_FV_EulerEvaluator.hpp:593-864, USE_NS_SA_NEGATIVE_MODEL)
template <class T>
DG_HD void sa_source_point(const HotView<T>& h, const double U[4], double U5, const double G[2][4],
                           const double gS[2], double dWall, double& src, double& jac) {
  const double d = dmin(dWall, pow(3e200, 1. / 6.));
  const double cb1 = 0.1355, cb2 = 0.622, sigma = 2. / 3., cnu1 = 7.1, cnu2 = 0.7, cnu3 = 0.9, cw2 = 0.3, cw3 = 2,
               kappa = 0.41, rlim = 10, ct3 = 1.2, ct4 = 0.5;
  const double cw1 = cb1 / (kappa * kappa) + (1 + cb2) / sigma;
  const double p = (h.gamma - 1) * (U[3] - 0.5 * (U[1] * U[1] + U[2] * U[2]) / U[0]);
  const double muRef = h.mu;
  const double nuh = U5 * muRef / U[0];
  const double mufPhy = sutherland_mu(h, p, U[0]);
  const double Chi = U5 * muRef / mufPhy;
  const double Chi3 = Chi * Chi * Chi;
  const double fnu1 = Chi3 / (Chi3 + cnu1 * cnu1 * cnu1);
  const double fnu2 = 1 - Chi / (1 + Chi * fnu1);
  const double vx = U[1] / U[0], vy = U[2] / U[0];
  double diffNu[2], diffRho[2];
  for (int i = 0; i < 2; i++) {
    diffRho[i] = G[i][0];
    diffNu[i] = (gS[i] * muRef - nuh * G[i][0]) / U[0];
  }
  // diffU[i][j] = d u_j / d x_i; Omega = (diffU^T - diffU) / 2, S = |Omega|_F sqrt 2
  const double d10 = (G[1][1] - G[1][0] * vx) / U[0], d01 = (G[0][2] - G[0][0] * vy) / U[0];
  const double w01 = 0.5 * (d10 - d01);
  const double S = sqrt(2 * w01 * w01) * sqrt(2.0);
  const double Sbar = nuh / (kappa * kappa * d * d) * fnu2;
  double Sh;
  if (Sbar < -cnu2 * S) Sh = S + S * (cnu2 * cnu2 * S + cnu3 * Sbar) / ((cnu3 - 2 * cnu2) * S - Sbar);
  else Sh = S + Sbar;
  const double r = dmin(nuh / (Sh * (kappa * d) * (kappa * d) + 1e-200), rlim);
  const double r6 = r * r * r * r * r * r;
  const double g = r + cw2 * (r6 - r);
  const double g6 = g * g * g * g * g * g, c6 = cw3 * cw3 * cw3 * cw3 * cw3 * cw3;
  const double fw = g * pow((1 + c6) / (g6 + c6), 1. / 6.);
  const double ft2 = ct3 * exp(-ct4 * Chi * Chi);
  double D = (cw1 * fw - cb1 / (kappa * kappa) * ft2) * (nuh / d) * (nuh / d);
  double P = cb1 * (1 - ft2) * Sh * nuh;
  double fn = 1;
  if (U5 < 0) {
    const double cn1 = 16;
    fn = (cn1 + Chi3) / (cn1 - Chi3);
    P = cb1 * (1 - ct3) * S * nuh;
    D = -cw1 * (nuh / d) * (nuh / d);
  }
  const double dn2 = diffNu[0] * diffNu[0] + diffNu[1] * diffNu[1];
  const double rn = diffRho[0] * diffNu[0] + diffRho[1] * diffNu[1];
  src = U[0] * (P - D + dn2 * cb2 / sigma) / muRef - (U5 * fn * muRef + mufPhy) / (U[0] * sigma) * rn / muRef;
  jac = -dmin(U[0] * (P * 0 - D * 2) / muRef / (U5 + 1e-200), -1e-200);
}

// the SA source and its Jacobian at cell quadrature point ig of cell i, times the point's weight
// (0 for the zero-weight padding of a triangle's 4 points)
template <class T>
DG_HD void sa_cell_point(int64_t i, int ig, const HotView<T>& h, const SaView<T>& sa, double& src, double& jac) {
  src = jac = 0;
  const double* gp = &sa.cellGp[(i * kSaGp + ig) * kSaGpE];
  const double wdet = gp[0];
  if (wdet == 0.0) return;
  double U[4];
  load4<T>(&h.u[i * 4], U);
  const T* rc = &h.urec[i * 20];
  const T* rs = &sa.urec[i * 5];
  double inc[4] = {0, 0, 0, 0}, G[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, incS = 0, gS[2] = {0, 0};
  for (int q = 0; q < 5; q++) {
    const double b0 = gp[1 + q], bx = gp[6 + q], by = gp[11 + q];
    for (int v = 0; v < 4; v++) {
      const double a = (double)rc[4 * q + v];
      inc[v] += b0 * a; G[0][v] += bx * a; G[1][v] += by * a;
    }
    const double a = (double)rs[q];
    incS += b0 * a; gS[0] += bx * a; gS[1] += by * a;
  }
  double Ug[4];
  const double u5 = sa.u[i];
  const bool comp = compress_rec_part(U, inc, Ug);
  const double U5g = comp ? u5 : u5 + incS;
  double s, j;
  sa_source_point(h, Ug, U5g, G, gS, sa.dWall[i], s, j);
  src = s * wdet;
  jac = j * wdet;
}

// U5 rhs of cell i: the face fluxes, the flux-balance term -U5_i (v_i . closure_i) / V_i, and the
// source integrated over the cell quadrature (src / jac: the kSaGp weighted point values, summed in
// point order); the source Jacobian into srcJac
template <class T>
DG_HD void sa_cell_rhs(int64_t i, const HotView<T>& h, const SaView<T>& sa, const double* src, const double* jac) {
  double s = 0;
  for (int k = 0; k < h.nfmax; k++) {
    const int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    s += sf >= 0 ? sa.flux[sf] : -sa.flux[~sf];
  }
  double U[4];
  load4<T>(&h.u[i * 4], U);
  const double u5 = sa.u[i];
  const double vn = (U[1] * h.closure[2 * i] + U[2] * h.closure[2 * i + 1]) / U[0];
  double r = (s - u5 * vn) / h.vol[i];
  double sv = 0, sj = 0;
  for (int ig = 0; ig < kSaGp; ig++) {
    sv += src[ig];
    sj += jac[ig];
  }
  sa.rhs[i] = r + sv / h.vol[i];
  sa.srcJac[i] = sj / h.vol[i];
}

// EvaluateDt face part for an SA context (DNDS_FV_EulerEvaluator.cpp:25-137): the viscous spectral
// radius uses the eddy viscosity of the mean U5
template <class T>
DG_HD void dt_face_sa(int64_t f, const HotView<T>& h, const SaView<T>& sa) {
  const int32_t L = h.faceL[f], R = h.faceR[f];
  const double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1], area = h.faceArea[f];
  double UL[4];
  load4<T>(&h.u[(int64_t)L * 4], UL);
  double pL, aL2, HL, pR, aR2, HR;
  double uL = UL[1] / UL[0], vL = UL[2] / UL[0], uR = uL, vR = vL;
  thermal(UL[3], UL[0], uL * uL + vL * vL, h.gamma, pL, aL2, HL);
  pR = pL; aR2 = aL2;
  double rhoMean = UL[0], s5 = sa.u[L];
  if (R >= 0) {
    double UR[4];
    load4<T>(&h.u[(int64_t)R * 4], UR);
    rhoMean = (UL[0] + UR[0]) * 0.5;
    s5 = (s5 + sa.u[R]) * 0.5;
    uR = UR[1] / UR[0]; vR = UR[2] / UR[0];
    thermal(UR[3], UR[0], uR * uR + vR * vR, h.gamma, pR, aR2, HR);
  }
  const double vn = 0.5 * ((uL + uR) * nx + (vL + vR) * ny);
  const double pMean = (pL + pR) * 0.5;
  double lam = fabs(vn) + sqrt(h.gamma * pMean / rhoMean);
  double muf = sutherland_mu(h, pMean, rhoMean);
  muf *= sa_mu_factor(s5, h.mu, muf);
  const double lamVis = muf / rhoMean * dmax(4. / 3., h.gamma / h.pr);
  lam += lamVis * area * (1.0 / h.vol[L] + 1.0 / (R >= 0 ? h.vol[R] : h.vol[L]));
  h.lamA[f] = lam * area;
  h.dLam[f] = fabs((uR - uL) * nx + (vR - vL) * ny) + sqrt(fabs(aR2 - aL2)) * 0.7071;
}

// one cell of an LU-SGS sweep on the 5 variables of an SA context (flow in inc, U5 in sa.inc)
template <class T, bool FWD>
DG_HD void lusgs_cell_sa(const HotView<T>& h, const SaView<T>& sa, const int32_t* rankOf, int64_t i, double alpha,
                         const double* Dinv, const double* rhs, double* inc) {
  const int ci = rankOf[i];
  double buf[4], bufS;
  if (FWD) { load4<T>(&rhs[i * 4], buf); bufS = sa.rhs[i]; }
  else { buf[0] = buf[1] = buf[2] = buf[3] = 0.0; bufS = 0.0; }
  const double scale = -0.5 * alpha / h.vol[i];
  for (int k = 0; k < h.nfmax; k++) {
    const int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    const int32_t f = sf >= 0 ? sf : ~sf;
    const int32_t j = sf >= 0 ? h.faceR[f] : h.faceL[f];
    if (j < 0) continue;
    const int cj = rankOf[j];
    if (FWD ? !(cj < ci) : !(cj > ci)) continue;
    const double sg = sf >= 0 ? 1.0 : -1.0;
    const double area = h.faceArea[f], lam = h.lamA[f] / area;
    const double nx = sg * h.faceNormal[2 * f], ny = sg * h.faceNormal[2 * f + 1];
    double U[4], dU[4];
    load4<T>(&h.u[(int64_t)j * 4], U);
    load4<T>(&inc[(int64_t)j * 4], dU);
    // fluxJacobian0_Right_Times_du (DNDS_FV_EulerEvaluator.hpp:928-956) with the U5 row
    const double ir = 1.0 / U[0];
    const double vx = U[1] * ir, vy = U[2] * ir;
    const double p = (h.gamma - 1) * (U[3] - 0.5 * U[0] * (vx * vx + vy * vy));
    const double dvx = (dU[1] - vx * dU[0]) * ir, dvy = (dU[2] - vy * dU[0]) * ir;
    const double dp = (h.gamma - 1) * (dU[3] - 0.5 * (dU[1] * vx + dU[2] * vy + U[1] * dvx + U[2] * dvy));
    const double vn = vx * nx + vy * ny, dvn = dvx * nx + dvy * ny;
    const double dF[4] = {dU[1] * nx + dU[2] * ny - lam * dU[0], dU[1] * vn + U[1] * dvn + nx * dp - lam * dU[1],
                          dU[2] * vn + U[2] * dvn + ny * dp - lam * dU[2], (dU[3] + dp) * vn + (U[3] + p) * dvn - lam * dU[3]};
    const double dS = sa.inc[j];
    const double dFS = dS * vn + sa.u[j] * dvn - dS * lam;
    for (int v = 0; v < 4; v++) buf[v] += scale * area * dF[v];
    bufS += scale * area * dFS;
  }
  const double di = Dinv[i], dS = sa.Dinv[i];
  double* o = &inc[i * 4];
  if (FWD) {
    for (int v = 0; v < 4; v++) o[v] = di * buf[v];
    sa.inc[i] = dS * bufS;
  } else {
    for (int v = 0; v < 4; v++) o[v] += di * buf[v];
    sa.inc[i] += dS * bufS;
  }
}

// CompressInc (DNDS_FV_EulerEvaluator.hpp:1362-1406): U5 may not go negative
DG_HD double sa_compress_inc(double u5, double inc5) {
  if (u5 + inc5 < 0) {
    const double declineV = inc5 / (u5 + 1e-6);
    const double newu5 = dmax(1e-6, u5 * exp(declineV));
    return newu5 - u5;
  }
  return inc5;
}

}  // namespace dg
