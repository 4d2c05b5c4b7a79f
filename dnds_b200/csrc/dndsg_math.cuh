// dndsg_math.cuh -- host/device arithmetic of the DNDS hot path (2-D, P2, Euler).
//
// Everything here is plain straight-line arithmetic on registers, usable from
// CUDA kernels and from host code.  Reference functions are cited per item.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define DG_HD __host__ __device__ __forceinline__
#else
#define DG_HD inline
#endif

namespace dg {

constexpr double kVerySmall = 1e-200;  // verySmallReal (DNDS_Defines.h:70)
constexpr double kPi = 3.14159265358979323846;

// BoundaryType (DNDS_Mesh.hpp:21-35)
enum : int { BC_INNER = -1, BC_WALL = 1, BC_FAR = 2, BC_WALL_EULER = 3, BC_WALL_NOSLIP = 4,
             BC_DMR_FAR = -2, BC_RT_FAR = -3, BC_IV_FAR = -4, BC_RIEMANN_FAR = -5 };
DG_HD bool is_far_type(int b) {
  return b == BC_FAR || b == BC_DMR_FAR || b == BC_RT_FAR || b == BC_IV_FAR || b == BC_RIEMANN_FAR;
}

template <class T> DG_HD T sq(T x) { return x * x; }
template <class T> DG_HD T dmax(T a, T b) { return a > b ? a : b; }
template <class T> DG_HD T dmin(T a, T b) { return a < b ? a : b; }

// ---------------------------------------------------------------- gas (2-D)
// Gas::IdealGasThermal (DNDS_Gas.hpp:73-79)
template <class T>
DG_HD void thermal(T E, T rho, T vsqr, T gamma, T& p, T& asqr, T& H) {
  p = (gamma - T(1)) * (E - rho * T(0.5) * vsqr);
  asqr = gamma * p / rho;
  H = (E + p) / rho;
}

// rotate the momentum of U into the (n, t) frame of NormBuildLocalBaseV
// (DNDS_Elements.hpp:1467-1488): base = [n, (-ny, nx)]; U_local = base^T U
template <class T>
DG_HD void to_normal_frame(const T* U, T nx, T ny, T* R) {
  R[0] = U[0];
  R[1] = nx * U[1] + ny * U[2];
  R[2] = -ny * U[1] + nx * U[2];
  R[3] = U[3];
}
template <class T>
DG_HD void from_normal_frame(T* F, T nx, T ny) {
  T a = F[1], b = F[2];
  F[1] = nx * a - ny * b;
  F[2] = ny * a + nx * b;
}

// x-direction inviscid flux F(U) (Gas::GasInviscidFlux, DNDS_Gas.hpp:113-119)
template <class T>
DG_HD void inviscid_flux_x(const T* U, T gamma, T* F) {
  T ir = T(1) / U[0];
  T vx = U[1] * ir, vy = U[2] * ir;
  T p = (gamma - T(1)) * (U[3] - U[0] * T(0.5) * (vx * vx + vy * vy));
  F[0] = U[1];
  F[1] = U[1] * vx + p;
  F[2] = U[2] * vx;
  F[3] = (U[3] + p) * vx;
}

// Roe flux with the Harten-Yee entropy fix, normal frame
// (Gas::RoeFlux_IdealGas_HartenYee<2,0>, DNDS_Gas.hpp:406-654)
template <class T>
DG_HD void roe_flux(const T* UL, const T* UR, T gamma, T dLambda, T* F) {
  const T scaleHY = T(0.05);
  T irL = T(1) / UL[0], irR = T(1) / UR[0];
  T uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
  T pL, aL2, HL, pR, aR2, HR;
  thermal(UL[3], UL[0], uL * uL + vL * vL, gamma, pL, aL2, HL);
  thermal(UR[3], UR[0], uR * uR + vR * vR, gamma, pR, aR2, HR);
  T sL = sqrt(UL[0]), sR = sqrt(UR[0]);
  T isum = T(1) / (sL + sR);
  T u = (sL * uL + sR * uR) * isum, v = (sL * vL + sR * vR) * isum;
  T vs = u * u + v * v;
  T H = (sL * HL + sR * HR) * isum;
  T a2 = (gamma - T(1)) * (H - T(0.5) * vs);
  T a = sqrt(a2);
  T lam0 = fabs(u - a), lam1 = fabs(u), lam3 = fabs(u + a);
  T thr = dmax(scaleHY * (sqrt(vs) + a), dLambda);
  T thrS = thr * thr;
  if (lam0 < thr) lam0 = (lam0 * lam0 + thrS) / (T(2) * thr);
  if (lam3 < thr) lam3 = (lam3 * lam3 + thrS) / (T(2) * thr);
  T d0 = UR[0] - UL[0], d1 = UR[1] - UL[1], d2 = UR[2] - UL[2], d3 = UR[3] - UL[3];
  T al2 = d2 - v * d0;
  T d3b = d3 - al2 * v;
  T al1 = (gamma - T(1)) / a2 * (d0 * (H - u * u) + u * d1 - d3b);
  T al0 = (d0 * (u + a) - d1 - a * al1) / (T(2) * a);
  T al3 = d0 - (al0 + al1);
  T w0 = lam0 * al0, w1 = lam1 * al1, w2 = lam1 * al2, w3 = lam3 * al3;
  // ReV = [[1,1,0,1],[u-a,u,0,u+a],[v,v,1,v],[H-ua, vs/2, v, H+ua]]
  T i0 = w0 + w1 + w3;
  T i1 = (u - a) * w0 + u * w1 + (u + a) * w3;
  T i2 = v * w0 + v * w1 + w2 + v * w3;
  T i3 = (H - u * a) * w0 + T(0.5) * vs * w1 + v * w2 + (H + u * a) * w3;
  T FL0 = UL[1], FL1 = UL[1] * uL + pL, FL2 = UL[2] * uL, FL3 = (UL[3] + pL) * uL;
  T FR0 = UR[1], FR1 = UR[1] * uR + pR, FR2 = UR[2] * uR, FR3 = (UR[3] + pR) * uR;
  F[0] = (FL0 + FR0) * T(0.5) - T(0.5) * i0;
  F[1] = (FL1 + FR1) * T(0.5) - T(0.5) * i1;
  F[2] = (FL2 + FR2) * T(0.5) - T(0.5) * i2;
  F[3] = (FL3 + FR3) * T(0.5) - T(0.5) * i3;
}

// HLLC flux (Gas::HLLCFlux_IdealGas_HartenYee<2>, DNDS_Gas.hpp:312-403)
template <class T>
DG_HD void hllc_flux(const T* UL, const T* UR, T gamma, T* F) {
  T irL = T(1) / UL[0], irR = T(1) / UR[0];
  T uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
  T pL, aL2, HL, pR, aR2, HR;
  thermal(UL[3], UL[0], uL * uL + vL * vL, gamma, pL, aL2, HL);
  thermal(UR[3], UR[0], uR * uR + vR * vR, gamma, pR, aR2, HR);
  T sL = sqrt(UL[0]), sR = sqrt(UR[0]);
  T u = (sL * uL + sR * uR) / (sL + sR);
  T eta2 = T(0.5) * (sL * sR) / sq(sL + sR);
  T dsqr = (aL2 * sL + aR2 * sR) / (sL + sR) + eta2 * sq(uR - uL);
  T SL = u - sqrt(dsqr), SR = u + sqrt(dsqr);
  T FL[4] = {UL[1], UL[1] * uL + pL, UL[2] * uL, (UL[3] + pL) * uL};
  T FR[4] = {UR[1], UR[1] * uR + pR, UR[2] * uR, (UR[3] + pR) * uR};
  if (T(0) <= SL) { for (int k = 0; k < 4; k++) F[k] = FL[k]; return; }
  if (SR <= T(0)) { for (int k = 0; k < 4; k++) F[k] = FR[k]; return; }
  const T tiny = T(sizeof(T) == 8 ? 1e-200 : 1e-37);
  T SS = 0;
  T div = UL[0] * (SL - uL) - UR[0] * (SR - uR);
  if (fabs(div) > tiny) SS = (pR - pL + UL[1] * (SL - uL) - UR[1] * (SR - uR)) / div;
  T DS[4] = {T(0), T(1), T(0), SS};
  if (SS >= T(0)) {
    T d = SL - SS;
    if (fabs(d) < tiny) { for (int k = 0; k < 4; k++) F[k] = FL[k]; }
    else {
      T sc = (pL + UL[0] * (SL - uL) * (SS - uL)) * SL;
      for (int k = 0; k < 4; k++) F[k] = ((UL[k] * SL - FL[k]) * SS + DS[k] * sc) / d;
    }
  } else {
    T d = SR - SS;
    if (fabs(d) < tiny) { for (int k = 0; k < 4; k++) F[k] = FR[k]; }
    else {
      T sc = (pR + UR[0] * (SR - uR) * (SS - uR)) * SR;
      for (int k = 0; k < 4; k++) F[k] = ((UR[k] * SR - FR[k]) * SS + DS[k] * sc) / d;
    }
  }
}

DG_HD void cons_to_prim(const double* U, double* W, double gamma) {
  double ir = 1.0 / U[0];
  W[0] = U[0]; W[1] = U[1] * ir; W[2] = U[2] * ir;
  W[3] = (gamma - 1) * (U[3] - U[0] * 0.5 * (W[1] * W[1] + W[2] * W[2]));
}
DG_HD void prim_to_cons(const double* W, double* U, double gamma) {
  U[0] = W[0]; U[1] = W[1] * W[0]; U[2] = W[2] * W[0];
  U[3] = W[3] / (gamma - 1) + W[0] * 0.5 * (W[1] * W[1] + W[2] * W[2]);
}

// exact isentropic vortex (centre (xc,yc), chi = 5), as used by Special_IVFar
// (DNDS_FV_EulerEvaluator.hpp:1100-1125)
DG_HD void vortex_state(double x, double y, double xc, double yc, double gamma, double* U) {
  const double chi = 5.0;
  double r2 = sq(x - xc) + sq(y - yc);
  double dT = -(gamma - 1) / (8 * gamma * sq(kPi)) * sq(chi) * exp(1 - r2);
  double e2 = chi / 2 / kPi * exp((1 - r2) / 2);
  double ux = 1 + e2 * -(y - yc), uy = 1 + e2 * (x - xc);
  double Tm = 1 + dT;
  double rho = pow(Tm, 1 / (gamma - 1));
  double p = Tm * rho;
  U[0] = rho; U[1] = rho * ux; U[2] = rho * uy;
  U[3] = 0.5 * (ux * ux + uy * uy) * rho + p / (gamma - 1);
}

// EulerEvaluator::generateBoundaryValue for the 2-D Euler model
// (DNDS_FV_EulerEvaluator.hpp:958-1275); n = unit outward normal, pc = face centre
DG_HD void boundary_value(int bc, const double* UL, double nx, double ny, double pcx, double pcy, double t,
                          double gamma, const double* farU, double* UR) {
  if (bc == BC_FAR) {
    double ir = 1.0 / UL[0];
    double vn = (UL[1] * nx + UL[2] * ny) * ir;
    double vs = sq(UL[1] * ir) + sq(UL[2] * ir);
    double p, a2, H;
    thermal(UL[3], UL[0], vs, gamma, p, a2, H);
    double a = sqrt(a2);
    if (vn - a > 0) {
      for (int k = 0; k < 4; k++) UR[k] = UL[k];
    } else if (vn > 0) {
      double fp[4], lp[4];
      cons_to_prim(farU, fp, gamma);
      cons_to_prim(UL, lp, gamma);
      lp[3] = fp[3];
      prim_to_cons(lp, UR, gamma);
    } else if (vn + a > 0) {
      double fp[4], lp[4];
      cons_to_prim(farU, fp, gamma);
      cons_to_prim(UL, lp, gamma);
      fp[3] = lp[3];
      prim_to_cons(fp, UR, gamma);
    } else {
      for (int k = 0; k < 4; k++) UR[k] = farU[k];
    }
  } else if (bc == BC_IV_FAR) {
    vortex_state(pcx, pcy, 5 + t, 5 + t, gamma, UR);
  } else if (bc == BC_RIEMANN_FAR) {
    const double phi2 = -0.422115882408869, loc = 0.8, bTol = 1e-9;
    double p2 = loc + phi2 * t;
    double lp[4];
    cons_to_prim(UL, lp, gamma);
    double W[4] = {lp[0], lp[1], lp[2], lp[3]};
    if (fabs(pcx) < bTol) {
      if (pcy <= p2) { W[0] = 0.137992831541219; W[1] = 1.206045378311055; W[2] = 1.206045378311055; W[3] = 0.029032258064516; }
      else { W[0] = 0.532258064516129; W[1] = 1.206045378311055; W[2] = 0.0; W[3] = 0.3; }
    } else if (fabs(pcx - 1.0) < bTol) {
      W[1] = -lp[1];
    } else if (fabs(pcy - 1.0) < bTol) {
      W[2] = -lp[2];
    } else if (fabs(pcy) < bTol) {
      if (pcx <= p2) { W[0] = 0.137992831541219; W[1] = 1.206045378311055; W[2] = 1.206045378311055; W[3] = 0.029032258064516; }
      else { W[0] = 0.532258064516129; W[1] = 0.0; W[2] = 1.206045378311055; W[3] = 0.3; }
    } else {
      W[0] = W[1] = W[2] = W[3] = NAN;
    }
    prim_to_cons(W, UR, gamma);
  } else if (bc == BC_WALL_EULER) {
    double d = UL[1] * nx + UL[2] * ny;
    UR[0] = UL[0]; UR[1] = UL[1] - d * nx; UR[2] = UL[2] - d * ny; UR[3] = UL[3];
  } else if (bc == BC_WALL_NOSLIP) {
    UR[0] = UL[0]; UR[1] = -UL[1]; UR[2] = -UL[2]; UR[3] = UL[3];
  } else {
    for (int k = 0; k < 4; k++) UR[k] = NAN;
  }
}

// EulerEvaluator::CompressRecPart (DNDS_FV_EulerEvaluator.hpp:1277-1360):
// mean + increment, falling back to the mean if density or internal energy < 0
DG_HD bool compress_rec_part(const double* um, const double* inc, double* r) {
  for (int k = 0; k < 4; k++) r[k] = um[k] + inc[k];
  bool red = false;
  if (r[0] < 0) { for (int k = 0; k < 4; k++) r[k] = um[k]; red = true; }
  double eK = (r[1] * r[1] + r[2] * r[2]) * 0.5 / (kVerySmall + r[0]);
  if (r[3] - eK < 0) { for (int k = 0; k < 4; k++) r[k] = um[k]; red = true; }
  return red;
}

// ---------------------------------------------------------------- P2 basis
// A cell's zero-mean P2 basis phi_k(x) = m_k(xi) - moment_k, k = 1..5, with
// m = {xi, eta, xi^2, xi*eta, eta^2} and xi = Pinv (x - c).  This is the
// basis of VRFiniteVolume2D::FDiffBaseValue (DNDS_FV_VR.hpp:300-1019): Pinv
// is diag(1/sx, 1/sy) in global coordinates or the inverse of the scaled
// inertia frame when useLocalCoord.  D[r][k] are the derivatives
// {value, d/dx, d/dy, d2/dx2, d2/dxdy, d2/dy2} of phi_{k+1} in global coordinates.
struct CellFrame {
  double c[2];
  double Pinv[2][2];
  double moment[5];  // moments of m_1..m_5 (m_0 = 1 has moment 1)
};

template <class C>
DG_HD void p2_monomials(C xi, C eta, C m[5]) {
  m[0] = xi; m[1] = eta; m[2] = xi * xi; m[3] = xi * eta; m[4] = eta * eta;
}

// the frame coordinates of a point: xi = Pinv (x - c)
DG_HD void p2_frame_coords(const CellFrame& f, double x, double y, double& xi, double& eta) {
  const double dx = x - f.c[0], dy = y - f.c[1];
  xi = f.Pinv[0][0] * dx + f.Pinv[0][1] * dy;
  eta = f.Pinv[1][0] * dx + f.Pinv[1][1] * dy;
}

// value, gradient and Hessian rows of the basis at frame coordinates (xi, eta), from the frame's
// Pinv and moments alone
// basis value and derivative rows at frame coordinates (xi, eta), in the arithmetic type C
template <class C>
DG_HD void p2_diffs_at(const C Q[2][2], const C moment[5], C xi, C eta, C D[6][5]) {
  C m[5];
  p2_monomials(xi, eta, m);
  for (int k = 0; k < 5; k++) D[0][k] = m[k] - moment[k];
  // d(xi)/dx = Q[0][0], d(xi)/dy = Q[0][1], d(eta)/dx = Q[1][0], d(eta)/dy = Q[1][1]
  const C gxi[5] = {C(1), C(0), 2 * xi, eta, C(0)};  // dm/dxi
  const C get[5] = {C(0), C(1), C(0), xi, 2 * eta};  // dm/deta
  for (int k = 0; k < 5; k++) {
    D[1][k] = gxi[k] * Q[0][0] + get[k] * Q[1][0];
    D[2][k] = gxi[k] * Q[0][1] + get[k] * Q[1][1];
  }
  // second derivatives: Hxi = {m_xixi, m_xieta, m_etaeta} per monomial
  const C hxx[5] = {C(0), C(0), C(2), C(0), C(0)}, hxy[5] = {C(0), C(0), C(0), C(1), C(0)},
          hyy[5] = {C(0), C(0), C(0), C(0), C(2)};
  for (int k = 0; k < 5; k++) {
    // d2/dxa dxb = sum_ij H_ij Q[i][a] Q[j][b]
    D[3][k] = hxx[k] * Q[0][0] * Q[0][0] + 2 * hxy[k] * Q[0][0] * Q[1][0] + hyy[k] * Q[1][0] * Q[1][0];
    D[4][k] = hxx[k] * Q[0][0] * Q[0][1] + hxy[k] * (Q[0][0] * Q[1][1] + Q[1][0] * Q[0][1]) + hyy[k] * Q[1][0] * Q[1][1];
    D[5][k] = hxx[k] * Q[0][1] * Q[0][1] + 2 * hxy[k] * Q[0][1] * Q[1][1] + hyy[k] * Q[1][1] * Q[1][1];
  }
}

DG_HD void p2_diffs(const CellFrame& f, double x, double y, double D[6][5]) {
  double xi, eta;
  p2_frame_coords(f, x, y, xi, eta);
  p2_diffs_at(f.Pinv, f.moment, xi, eta, D);
}

// only the value row (what the flux needs)
DG_HD void p2_values(const CellFrame& f, double x, double y, double v[5]) {
  double dx = x - f.c[0], dy = y - f.c[1];
  double xi = f.Pinv[0][0] * dx + f.Pinv[0][1] * dy, eta = f.Pinv[1][0] * dx + f.Pinv[1][1] * dy;
  double m[5];
  p2_monomials(xi, eta, m);
  for (int k = 0; k < 5; k++) v[k] = m[k] - f.moment[k];
}

// ---------------------------------------------------------------- VR functional
// FFaceFunctional (DNDS_FV_VR.hpp:1021-1293), the 6-weight (P2) branch, written
// as a sum of squares: conj(I,J) = sum_a (T_a D_I)^T (T_a D_J).  proj() forms
// the six rows T_a D for one side.  The mixed second-derivative row keeps the
// reference's coefficients {n0 t0, 2 n0 t1, n1 t1}.
template <class C>
struct FaceFunctionalT {
  C t[6][6];  // t[a][r]: weight of derivative row r in term a
};
using FaceFunctional = FaceFunctionalT<double>;

// the functional's rows, in the arithmetic type C (the weights' zero test and 1e-50 threshold are the
// reference's; in FP32 a weight below 1e-50 is zero already)
template <class C>
DG_HD FaceFunctionalT<C> make_functional(const C W[6], C unx, C uny, C tangWeight, C tangModifier, int modLoc) {
  FaceFunctionalT<C> F;
  for (int a = 0; a < 6; a++) for (int r = 0; r < 6; r++) F.t[a][r] = C(0);
  C w2r = C(0), length = C(0);
  if (fabs((double)W[1]) >= 1e-50 || fabs((double)W[2]) >= 1e-50) {
    w2r = fabs(W[1]) >= fabs(W[2]) ? W[3] / (W[1] * W[1]) : W[5] / (W[2] * W[2]);
    length = sqrt(W[1] * W[1] + W[2] * W[2]);
  }
  const C n0 = unx * length, n1 = uny * length;
  const C tf = tangWeight * tangModifier * (modLoc == 1 ? tangModifier : C(1));
  const C t0 = -n1 * tf, t1 = n0 * tf;
  const C tm = modLoc == 0 ? tangModifier : C(1);  // sqrt of the reference's sqr(tangModifier)
  F.t[0][0] = W[0];
  F.t[1][1] = n0; F.t[1][2] = n1;
  F.t[2][1] = t0 * tm; F.t[2][2] = t1 * tm;
  F.t[3][3] = n0 * n0 * w2r; F.t[3][4] = 2 * n0 * n1 * w2r; F.t[3][5] = n1 * n1 * w2r;
  const C s2 = sqrt(C(2)) * tm;
  F.t[4][3] = n0 * t0 * w2r * s2; F.t[4][4] = 2 * n0 * t1 * w2r * s2; F.t[4][5] = n1 * t1 * w2r * s2;
  F.t[5][3] = t0 * t0 * w2r * tm; F.t[5][4] = 2 * t0 * t1 * w2r * tm; F.t[5][5] = t1 * t1 * w2r * tm;
  return F;
}

DG_HD void functional_proj(const FaceFunctional& F, const double D[6][5], double P[6][5]) {
  for (int a = 0; a < 6; a++)
    for (int k = 0; k < 5; k++) {
      double s = 0;
      for (int r = 0; r < 6; r++) s += F.t[a][r] * D[r][k];
      P[a][k] = s;
    }
}

// Cholesky solve A X = B for SPD 5x5 A, B 5 x m (in place)
DG_HD bool chol5(double A[5][5]) {
  for (int j = 0; j < 5; j++) {
    double s = A[j][j];
    for (int k = 0; k < j; k++) s -= A[j][k] * A[j][k];
    if (!(s > 0)) return false;
    double d = sqrt(s);
    A[j][j] = d;
    for (int i = j + 1; i < 5; i++) {
      double t = A[i][j];
      for (int k = 0; k < j; k++) t -= A[i][k] * A[j][k];
      A[i][j] = t / d;
    }
  }
  return true;
}
DG_HD void chol5_solve_vec(const double L[5][5], double* b) {
  for (int i = 0; i < 5; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= L[i][k] * b[k];
    b[i] = s / L[i][i];
  }
  for (int i = 4; i >= 0; i--) {
    double s = b[i];
    for (int k = i + 1; k < 5; k++) s -= L[k][i] * b[k];
    b[i] = s / L[i][i];
  }
}

// LU with partial pivoting, solve A X = B (5x5, B 5x5), used for the secondary
// reconstruction matrices (HardEigen::EigenLeastSquareSolve on a square system)
DG_HD bool lu5_solve(double A[5][5], double B[5][5]) {
  for (int k = 0; k < 5; k++) {
    int p = k;
    for (int i = k + 1; i < 5; i++) if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
    if (A[p][k] == 0.0) return false;
    if (p != k)
      for (int j = 0; j < 5; j++) {
        double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t;
        t = B[k][j]; B[k][j] = B[p][j]; B[p][j] = t;
      }
    for (int i = k + 1; i < 5; i++) {
      double f = A[i][k] / A[k][k];
      for (int j = k; j < 5; j++) A[i][j] -= f * A[k][j];
      for (int j = 0; j < 5; j++) B[i][j] -= f * B[k][j];
    }
  }
  for (int k = 4; k >= 0; k--)
    for (int j = 0; j < 5; j++) {
      double s = B[k][j];
      for (int i = k + 1; i < 5; i++) s -= A[k][i] * B[i][j];
      B[k][j] = s / A[k][k];
    }
  return true;
}

}  // namespace dg
