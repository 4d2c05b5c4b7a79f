// dndsg_bodies.cuh -- per-cell / per-face bodies of the setup and hot kernels.
//
// Each body processes one cell or one face and touches only its own outputs,
// so a kernel is "one thread per item" around a body.  Data layouts:
//   * per-cell and per-face operator data: tile-major AoSoA, element e of item
//     i at ((i/32)*E + e)*32 + i%32 -> a warp reads one contiguous 32-wide row
//     per element (fully coalesced without shared-memory staging);
//   * u  [N][4] double, urec [N][5][4] (T), flux [F][4] double: one item's
//     values are contiguous, so neighbour gathers use whole 16-byte vectors.
#pragma once
#include "dndsg_math.cuh"

namespace dg {

DG_HD int64_t aos(int64_t i, int e, int E) { return ((i >> 5) * (int64_t)E + e) * 32 + (i & 31); }
DG_HD int64_t aos_size(int64_t n, int E) { return ((n + 31) / 32) * 32 * (int64_t)E; }

// VR slot modes (what a cell's face contributes to its Jacobi update,
// DNDS_FV_VR.hpp:1520-1665)
enum : int32_t { VR_INNER = 0, VR_FAR = 1, VR_WALL = 2, VR_WALLCORR = 3, VR_EMPTY = 4 };
constexpr int32_t kEmptySlot = INT32_MIN;  // cellFace slot without a face

// LINE_3 Gauss-Legendre on [-1, 1]
DG_HD double l3_point(int g) { return g == 0 ? -0.7745966692414834 : (g == 1 ? 0.0 : 0.7745966692414834); }
DG_HD double l3_weight(int g) { return g == 1 ? 8.0 / 9.0 : 5.0 / 9.0; }

// The value-row basis of a face's two cells at its 3 gauss points, stored compactly (AoSoA, E = 18):
// per side 9 values, the 5 basis values v1 at the face centre (gauss point 1), the centre's frame
// coordinates (xi, eta) and the frame offset (dxi, deta) from the centre to gauss point 2 (gauss
// point 0 is at the opposite offset).  The quadratic monomials m = (xi, eta, xi^2, xi eta, eta^2)
// give the other points exactly: the basis at gauss points 0 and 2 is v1 + C -+ B, where
// B = (dxi, deta, 2 xi dxi, xi deta + eta dxi, 2 eta deta) and C = (0, 0, dxi^2, dxi deta, deta^2)
// are the odd and even parts of m(xi + s dxi, eta + s deta) - m(xi, eta) at s = +-1.  18 values per
// face instead of the 30 of a table of the basis at every point.
constexpr int kFaceBasisSide = 9, kFaceBasisE = 18;

template <class T>
struct FaceBasisSide {
  T v1[5], B[5], C[5];
  DG_HD FaceBasisSide(const T* fb, int64_t f, int side) {
    const int o = side * kFaceBasisSide;
    for (int k = 0; k < 5; k++) v1[k] = fb[aos(f, o + k, kFaceBasisE)];
    const T xi = fb[aos(f, o + 5, kFaceBasisE)], eta = fb[aos(f, o + 6, kFaceBasisE)];
    const T dxi = fb[aos(f, o + 7, kFaceBasisE)], det = fb[aos(f, o + 8, kFaceBasisE)];
    B[0] = dxi; B[1] = det; B[2] = T(2) * xi * dxi; B[3] = xi * det + eta * dxi; B[4] = T(2) * eta * det;
    C[0] = T(0); C[1] = T(0); C[2] = dxi * dxi; C[3] = dxi * det; C[4] = det * det;
  }
  // the basis values at gauss point g
  DG_HD void at(int g, T phi[5]) const {
    for (int k = 0; k < 5; k++) phi[k] = g == 1 ? v1[k] : (g == 0 ? (v1[k] + C[k]) - B[k] : (v1[k] + C[k]) + B[k]);
  }
};

// ---------------------------------------------------------------- setup
struct SetupParams {
  int use_local_coord, anisotropic_lengths, base_center_type;
  int weight_scheme_geom, weight_scheme_dir, tang_weight_direction, tang_weight_mod_loc;
  double weight_len_scale, wall_weight, far_weight, tang_weight, tang_weight_mod_min, tang_weight_mod_power;
};

struct CellSetup {
  int nn;
  double xy[4][2];
  double vol;
  double bary[2];
  CellFrame fr;
};

struct MeshView {
  int64_t N, F;
  const double* node_xy;
  const int32_t* cell_nodes;
  const int32_t* face_nodes;
  const int32_t* face_cells;
  const int32_t* face_bc;
  const double* face_shift;  // may be null
};

// Tri3 / Quad4 map at parametric (a, b): point and jacobian determinant
DG_HD void elem_map(const CellSetup& c, double a, double b, double& x, double& y, double& det) {
  if (c.nn == 3) {
    x = c.xy[0][0] * (1 - a - b) + c.xy[1][0] * a + c.xy[2][0] * b;
    y = c.xy[0][1] * (1 - a - b) + c.xy[1][1] * a + c.xy[2][1] * b;
    det = (c.xy[1][0] - c.xy[0][0]) * (c.xy[2][1] - c.xy[0][1]) - (c.xy[1][1] - c.xy[0][1]) * (c.xy[2][0] - c.xy[0][0]);
  } else {
    double N[4] = {(1 - a) * (1 - b) * 0.25, (1 + a) * (1 - b) * 0.25, (1 + a) * (1 + b) * 0.25, (1 - a) * (1 + b) * 0.25};
    double da[4] = {-(1 - b) * 0.25, (1 - b) * 0.25, (1 + b) * 0.25, -(1 + b) * 0.25};
    double db[4] = {-(1 - a) * 0.25, -(1 + a) * 0.25, (1 + a) * 0.25, (1 - a) * 0.25};
    x = y = 0;
    double xa = 0, ya = 0, xb = 0, yb = 0;
    for (int k = 0; k < 4; k++) {
      x += N[k] * c.xy[k][0]; y += N[k] * c.xy[k][1];
      xa += da[k] * c.xy[k][0]; ya += da[k] * c.xy[k][1];
      xb += db[k] * c.xy[k][0]; yb += db[k] * c.xy[k][1];
    }
    det = xa * yb - ya * xb;
  }
}
// cell quadrature: TRI_4 (Hammer) / QUAD_9 (Gauss) -- the reconstruction's cell schemes
DG_HD int cell_nq(int nn) { return nn == 3 ? 4 : 9; }
DG_HD void cell_qp(int nn, int g, double& a, double& b, double& w) {
  if (nn == 3) {
    const double P[4][2] = {{1. / 3., 1. / 3.}, {0.6, 0.2}, {0.2, 0.6}, {0.2, 0.2}};
    a = P[g][0]; b = P[g][1]; w = g == 0 ? -27. / 96. : 25. / 96.;
  } else {
    int i = g % 3, j = g / 3;
    a = l3_point(i); b = l3_point(j); w = l3_weight(i) * l3_weight(j);
  }
}

// initMoment (DNDS_FV_VR.cpp:82-181) + the basis frame of FDiffBaseValue
DG_HD bool setup_cell(int64_t i, const MeshView& m, const SetupParams& p, CellSetup& c) {
  c.nn = m.cell_nodes[4 * i + 3] < 0 ? 3 : 4;
  for (int k = 0; k < c.nn; k++) {
    int32_t nd = m.cell_nodes[4 * i + k];
    c.xy[k][0] = m.node_xy[2 * nd]; c.xy[k][1] = m.node_xy[2 * nd + 1];
  }
  int nq = cell_nq(c.nn);
  double vol = 0, bx = 0, by = 0;
  bool ok = true;
  for (int g = 0; g < nq; g++) {
    double a, b, w, x, y, det;
    cell_qp(c.nn, g, a, b, w);
    elem_map(c, a, b, x, y, det);
    if (!(det > 0)) ok = false;
    vol += det * w; bx += x * det * w; by += y * det * w;
  }
  c.vol = vol;
  c.bary[0] = bx / vol; c.bary[1] = by / vol;
  double ixx = 0, ixy = 0, iyy = 0;
  for (int g = 0; g < nq; g++) {
    double a, b, w, x, y, det;
    cell_qp(c.nn, g, a, b, w);
    elem_map(c, a, b, x, y, det);
    double rx = x - c.bary[0], ry = y - c.bary[1];
    ixx += rx * rx * det * w; ixy += rx * ry * det * w; iyy += ry * ry * det * w;
  }
  ixx /= vol; ixy /= vol; iyy /= vol;
  // basis centre
  if (p.base_center_type == 0) { c.fr.c[0] = c.bary[0]; c.fr.c[1] = c.bary[1]; }
  else {
    double x, y, det;
    elem_map(c, c.nn == 3 ? 1. / 3. : 0., c.nn == 3 ? 1. / 3. : 0., x, y, det);
    c.fr.c[0] = x; c.fr.c[1] = y;
  }
  if (!p.use_local_coord) {
    // CoordMinMaxScale: half extents
    double mnx = c.xy[0][0], mxx = mnx, mny = c.xy[0][1], mxy = mny;
    for (int k = 1; k < c.nn; k++) {
      mnx = dmin(mnx, c.xy[k][0]); mxx = dmax(mxx, c.xy[k][0]);
      mny = dmin(mny, c.xy[k][1]); mxy = dmax(mxy, c.xy[k][1]);
    }
    double sx = (mxx - mnx) * 0.5, sy = (mxy - mny) * 0.5;
    if (!p.anisotropic_lengths) { double s = sqrt(sx * sx + sy * sy); sx = sy = s; }
    c.fr.Pinv[0][0] = 1.0 / sx; c.fr.Pinv[0][1] = 0; c.fr.Pinv[1][0] = 0; c.fr.Pinv[1][1] = 1.0 / sy;
  } else {
    // principal axes of the inertia (largest first), then scale each axis by
    // the cell's half extent along it (DNDS_FV_VR.hpp:358-410)
    double hm = 0.5 * (ixx + iyy), hd = 0.5 * (ixx - iyy);
    double rr = sqrt(hd * hd + ixy * ixy);
    double e0x = 1, e0y = 0;
    if (rr > 1e-14 * fabs(hm)) {
      double lmax = hm + rr;
      double vx, vy;
      if (ixx >= iyy) { vx = lmax - iyy; vy = ixy; } else { vx = ixy; vy = lmax - ixx; }
      double nr = sqrt(vx * vx + vy * vy);
      e0x = vx / nr; e0y = vy / nr;
    }
    double e1x = -e0y, e1y = e0x;
    // coordinates along e0, e1 are projections (orthonormal frame)
    double mn0 = 1e300, mx0 = -1e300, mn1 = 1e300, mx1 = -1e300;
    for (int k = 0; k < c.nn; k++) {
      double rx = c.xy[k][0] - c.fr.c[0], ry = c.xy[k][1] - c.fr.c[1];
      double s0 = e0x * rx + e0y * ry, s1 = e1x * rx + e1y * ry;
      mn0 = dmin(mn0, s0); mx0 = dmax(mx0, s0); mn1 = dmin(mn1, s1); mx1 = dmax(mx1, s1);
    }
    double a0 = (mx0 - mn0) * 0.5, a1 = (mx1 - mn1) * 0.5;
    if (!p.anisotropic_lengths) { double s = sqrt(a0 * a0 + a1 * a1); a0 = a1 = s; }
    // P = [e0*a0, e1*a1]; Pinv rows = e_k^T / a_k
    c.fr.Pinv[0][0] = e0x / a0; c.fr.Pinv[0][1] = e0y / a0;
    c.fr.Pinv[1][0] = e1x / a1; c.fr.Pinv[1][1] = e1y / a1;
  }
  for (int k = 0; k < 5; k++) c.fr.moment[k] = 0;
  double mom[5] = {0, 0, 0, 0, 0};
  for (int g = 0; g < nq; g++) {
    double a, b, w, x, y, det, v[5];
    cell_qp(c.nn, g, a, b, w);
    elem_map(c, a, b, x, y, det);
    p2_values(c.fr, x, y, v);
    for (int k = 0; k < 5; k++) mom[k] += v[k] * det * w;
  }
  for (int k = 0; k < 5; k++) c.fr.moment[k] = mom[k] / vol;
  return ok;
}

// face geometry: nodes -> unit normal (out of L), length, centre, gauss points
struct FaceGeom {
  double nx, ny, area, cx, cy;
  double gx[3], gy[3];
};
DG_HD FaceGeom face_geom(int64_t f, const MeshView& m) {
  FaceGeom g;
  int32_t a = m.face_nodes[2 * f], b = m.face_nodes[2 * f + 1];
  double x0 = m.node_xy[2 * a], y0 = m.node_xy[2 * a + 1], x1 = m.node_xy[2 * b], y1 = m.node_xy[2 * b + 1];
  double dx = x1 - x0, dy = y1 - y0;
  g.area = sqrt(dx * dx + dy * dy);
  g.nx = dy / g.area; g.ny = -dx / g.area;
  g.cx = 0.5 * (x0 + x1); g.cy = 0.5 * (y0 + y1);
  for (int q = 0; q < 3; q++) {
    double s = l3_point(q);
    g.gx[q] = x0 * (1 - s) * 0.5 + x1 * (1 + s) * 0.5;
    g.gy[q] = y0 * (1 - s) * 0.5 + y1 * (1 + s) * 0.5;
  }
  return g;
}

// faceWeights (DNDS_FV_VR.cpp:716-888) for P2
DG_HD void face_weights(int64_t f, const MeshView& m, const SetupParams& p, const FaceGeom& g, const CellSetup* cells,
                        double W[6]) {
  int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
  int bc = m.face_bc[f];
  double dx, dy;
  for (int k = 0; k < 6; k++) W[k] = 1.0;
  if (R >= 0) {
    double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
    dx = cells[R].bary[0] + sx - cells[L].bary[0];
    dy = cells[R].bary[1] + sy - cells[L].bary[1];
  } else {
    for (int k = 0; k < 6; k++) W[k] = 0.0;
    dx = g.cx - cells[L].bary[0];
    dy = g.cy - cells[L].bary[1];
    if (bc == BC_WALL || bc == BC_WALL_EULER) W[0] = p.wall_weight;
    else if (is_far_type(bc)) W[0] = p.far_weight;
    else if (bc == BC_WALL_NOSLIP) {
      W[0] = p.wall_weight;
      double d = g.nx * dx + g.ny * dy;  // first-order wall delta
      dx = g.nx * d; dy = g.ny * d;
    }
  }
  double D = sqrt(dx * dx + dy * dy), S = g.area, GW = 1;
  if (p.weight_scheme_geom == 1) GW = pow(1.0 / D, 0.5);
  else if (p.weight_scheme_geom == 2) GW = pow(1.0 / S, 0.5);
  else if (p.weight_scheme_geom == 3) GW = pow(S / D, 0.25);
  if (p.tang_weight_direction == 0) { dx = g.nx * D; dy = g.ny * D; }
  dx *= p.weight_len_scale; dy *= p.weight_len_scale;
  // diffs {1, x, y, xx, xy, yy}
  const int ox[6] = {0, 1, 0, 2, 1, 0}, oy[6] = {0, 0, 1, 0, 1, 2};
  const double fac[3] = {1, 1, 2}, ncomb[6] = {1, 1, 1, 1, 2, 1}, hqm[3] = {1, 0.4643, 0.1559};
  for (int k = 0; k < 6; k++) {
    double pw = pow(dx, ox[k]) * pow(dy, oy[k]);
    if (p.weight_scheme_dir == 0) W[k] *= GW * pw * ncomb[k] / fac[ox[k] + oy[k]];
    else W[k] *= GW * pw * hqm[ox[k] + oy[k]];
  }
}

DG_HD double tang_modifier(const SetupParams& p, double volL, double volR, double area) {
  double sL = sqrt(volL) / area, sR = sqrt(volR) / area;
  double arMax = dmax(1.0, dmax(sL, sR));
  return pow((1.0 / arMax) * (1 - p.tang_weight_mod_min) + p.tang_weight_mod_min, p.tang_weight_mod_power);
}

// ---------------------------------------------------------------- hot path
template <class T>
struct HotView {
  int64_t N, F;
  int nfmax;
  // cells
  const double* vol;
  const double* closure;    // [N][2]
  const int32_t* cellFace;  // AoSoA E = nfmax: f (cell is left) or ~f (cell is right)
  const T* vrOp;            // AoSoA E = nfmax*30: per slot 25 A^-1B (row-major) + 5 A^-1b
  const int32_t* vrNbr;     // AoSoA E = nfmax
  const int32_t* vrMode;    // AoSoA E = nfmax
  const int32_t* vrFace;    // AoSoA E = nfmax (face id of the slot)
  const double* Ainv;       // [N][25] or null
  // faces
  const int32_t* faceL;
  const int32_t* faceR;
  const int32_t* faceBC;
  const T* faceBasis;       // AoSoA E = kFaceBasisE: per side the compact record of face_phi below
  const double* faceNormal; // [F][2] unit, out of L
  const double* faceArea;   // [F]
  const double* faceCenter; // [F][2]
  const double* faceW0;     // [F] weight 0 (wall corrections)
  // state
  double* u;
  double* uLast;
  double* rhs;
  double* dt;
  const T* urec;
  T* urecNew;
  double* flux;             // [F][4]
  double* lamA;             // [F]
  double* dLam;             // [F]
  const uint8_t* owned;     // [N] 1 for cells this context owns, or null (all owned); partitioned runs
  double gamma;
  double farU[4];
  double relax;
  // Navier-Stokes (mu > 0): gradient rows of both cells' basis at the face gauss points,
  // AoSoA E = 60: [side][gp][d/dx, d/dy][5], and the gas properties
  const T* faceGrad;
  double mu, cp, pr, tRef, cSuth;
};

template <class T>
DG_HD void load4(const double* p, double* v) {
#if defined(__CUDA_ARCH__)
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
#else
  for (int k = 0; k < 4; k++) v[k] = p[k];
#endif
}
// one 4-variable row of a cell's coefficient block (16 B for float, 32 B for double)
DG_HD void load_row(const float* p, float r[4]) {
#if defined(__CUDA_ARCH__)
  const float4 a = *reinterpret_cast<const float4*>(p);
  r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
#else
  for (int k = 0; k < 4; k++) r[k] = p[k];
#endif
}
DG_HD void load_row(const double* p, double r[4]) { load4<double>(p, r); }
DG_HD void store_row(float* p, const float r[4]) {
#if defined(__CUDA_ARCH__)
  *reinterpret_cast<float4*>(p) = make_float4(r[0], r[1], r[2], r[3]);
#else
  for (int k = 0; k < 4; k++) p[k] = r[k];
#endif
}
DG_HD void store_row(double* p, const double r[4]) {
#if defined(__CUDA_ARCH__)
  reinterpret_cast<double2*>(p)[0] = make_double2(r[0], r[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(r[2], r[3]);
#else
  for (int k = 0; k < 4; k++) p[k] = r[k];
#endif
}
template <class T>
DG_HD void load_rec(const T* p, T r[5][4]) {
  for (int q = 0; q < 5; q++) load_row(p + 4 * q, r[q]);
}

// accessor of the per-slot VR operator (25 A^-1B entries then 5 A^-1b entries) in global memory
template <class T>
struct VrOpGlobal {
  const T* op;
  int64_t i;
  int E;
  DG_HD T operator()(int k, int e) const { return op[aos(i, k * 30 + e, E)]; }
};

// one cell of ReconstructionJacobiStep (Jacobi form, DNDS_FV_VR.hpp:1500-1712)
template <class T, bool RELAX1>
DG_HD void vr_cell(int64_t i, const HotView<T>& h);
template <class T, bool RELAX1, class Op>
DG_HD void vr_cell_op(int64_t i, const HotView<T>& h, const Op& opk) {
  double ui[4];
  load4<T>(&h.u[i * 4], ui);
  T acc[5][4];
  if (RELAX1) {
    for (int q = 0; q < 5; q++) for (int v = 0; v < 4; v++) acc[q][v] = T(0);
  } else {
    T r0[5][4];
    load_rec(&h.urec[i * 20], r0);
    for (int q = 0; q < 5; q++) for (int v = 0; v < 4; v++) acc[q][v] = T(1 - h.relax) * r0[q][v];
  }
  const T relax = T(h.relax);
  for (int k = 0; k < h.nfmax; k++) {
    int mode = h.vrMode[aos(i, k, h.nfmax)];
    if (mode == VR_EMPTY) continue;
    int32_t j = h.vrNbr[aos(i, k, h.nfmax)];
    T b[5];
    for (int r = 0; r < 5; r++) b[r] = opk(k, 25 + r);
    if (mode == VR_INNER || mode == VR_FAR) {
      // stream the neighbour's coefficient rows: acc[r][:] += sum_q (A^-1B)[r][q] * urec_j[q][:]
      const T* rj = &h.urec[(int64_t)j * 20];
      for (int q = 0; q < 5; q++) {
        T row[4], col[5];
        load_row(rj + 4 * q, row);
        for (int r = 0; r < 5; r++) col[r] = relax * opk(k, r * 5 + q);
        for (int r = 0; r < 5; r++)
          for (int v = 0; v < 4; v++) acc[r][v] += col[r] * row[v];
      }
    }
    if (mode == VR_INNER || mode == VR_WALL) {
      T du[4];
      if (mode == VR_INNER) {
        double uj[4];
        load4<T>(&h.u[(int64_t)j * 4], uj);
        for (int v = 0; v < 4; v++) du[v] = T(uj[v] - ui[v]);
      } else {
        for (int v = 0; v < 4; v++) du[v] = T(0.0 - ui[v]);
      }
      for (int r = 0; r < 5; r++)
        for (int v = 0; v < 4; v++) acc[r][v] += relax * (du[v] * b[r]);
    }
    if (mode == VR_WALLCORR) {
      // Wall_Euler / Wall_NoSlip: A^-1 * integral of the weighted jump to the wall state
      int32_t f = h.vrFace[aos(i, k, h.nfmax)];
      double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1];
      double w0 = h.faceW0[f], area = h.faceArea[f];
      int bc = h.faceBC[f];
      T ri[5][4];
      load_rec(&h.urec[i * 20], ri);
      double corr[5][4];
      for (int q = 0; q < 5; q++) for (int v = 0; v < 4; v++) corr[q][v] = 0;
      const FaceBasisSide<T> fb(h.faceBasis, f, 0);
      for (int g = 0; g < 3; g++) {
        double phi[5];
        T pg[5];
        fb.at(g, pg);
        for (int q = 0; q < 5; q++) phi[q] = (double)pg[q];
        double uBL[4], uBV[4];
        for (int v = 0; v < 4; v++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += phi[q] * (double)ri[q][v];
          uBL[v] = s + ui[v];
        }
        if (bc == BC_WALL_EULER) {
          double d = nx * uBL[1] + ny * uBL[2];
          uBV[0] = uBL[0]; uBV[1] = uBL[1] - nx * d; uBV[2] = uBL[2] - ny * d; uBV[3] = uBL[3];
        } else {
          uBV[0] = uBL[0]; uBV[1] = -uBL[1]; uBV[2] = -uBL[2]; uBV[3] = uBL[3];
        }
        double jw = 0.5 * area * l3_weight(g);
        for (int q = 0; q < 5; q++)
          for (int v = 0; v < 4; v++) corr[q][v] += phi[q] * w0 * w0 * (uBV[v] - ui[v]) * jw;
      }
      const double* Ai = &h.Ainv[i * 25];
      for (int r = 0; r < 5; r++)
        for (int v = 0; v < 4; v++) {
          double s = 0;
          for (int q = 0; q < 5; q++) s += Ai[r * 5 + q] * corr[q][v];
          acc[r][v] += relax * T(s);
        }
    }
  }
  T* out = &h.urecNew[i * 20];
  for (int q = 0; q < 5; q++) store_row(out + 4 * q, acc[q]);
}
template <class T, bool RELAX1>
DG_HD void vr_cell(int64_t i, const HotView<T>& h) {
  vr_cell_op<T, RELAX1>(i, h, VrOpGlobal<T>{h.vrOp, i, h.nfmax * 30});
}

// reconstruction increments phi(gp) . urec of one cell at the 3 gauss points of a face, from the
// side's compact basis: the dot products of the coefficient rows with v1, B and C (rows 2..4 only),
// combined per point as phi . r = v1.r + C.r -+ B.r; gauss point 1 is the plain sum v1.r
template <class T>
DG_HD void side_increments(const FaceBasisSide<T>& b, const T* rec, T inc[3][4]) {
  T a[4] = {T(0), T(0), T(0), T(0)}, o[4] = {T(0), T(0), T(0), T(0)}, e[4] = {T(0), T(0), T(0), T(0)};
  for (int q = 0; q < 5; q++) {
    T row[4];
    load_row(rec + 4 * q, row);
    for (int v = 0; v < 4; v++) {
      a[v] += b.v1[q] * row[v];
      o[v] += b.B[q] * row[v];
      if (q >= 2) e[v] += b.C[q] * row[v];
    }
  }
  for (int v = 0; v < 4; v++) {
    const T p = a[v] + e[v];
    inc[0][v] = p - o[v]; inc[1][v] = a[v]; inc[2][v] = p + o[v];
  }
}

// reconstruction increments phi(gp) . urec of both cells at the 3 gauss points of
// face f; the coefficient rows are streamed once (EvaluateRHS, DNDS_FV_EulerEvaluator.cpp:250-360)
template <class T>
DG_HD void face_increments(int64_t f, int32_t L, int32_t R, const HotView<T>& h, T incL[3][4], T incR[3][4]) {
  side_increments(FaceBasisSide<T>(h.faceBasis, f, 0), &h.urec[(int64_t)L * 20], incL);
  if (R >= 0) side_increments(FaceBasisSide<T>(h.faceBasis, f, 1), &h.urec[(int64_t)R * 20], incR);
  else for (int g = 0; g < 3; g++) for (int v = 0; v < 4; v++) incR[g][v] = T(0);
}

// positivity-compressed states at gauss point g (CompressRecPart, boundary state on a boundary face)
template <class T, bool BND = true>
DG_HD int gp_states(int64_t f, int32_t R, const HotView<T>& h, double t, double nx, double ny, const double uL[4],
                    const double uR[4], const T incL[4], const T incR[4], double UL[4], double UR[4]) {
  double inc[4];
  for (int v = 0; v < 4; v++) inc[v] = (double)incL[v];
  int nred = compress_rec_part(uL, inc, UL) ? 1 : 0;
  if (!BND || R >= 0) {
    for (int v = 0; v < 4; v++) inc[v] = (double)incR[v];
    nred += compress_rec_part(uR, inc, UR) ? 1 : 0;
  } else {
    const double far[4] = {h.farU[0], h.farU[1], h.farU[2], h.farU[3]};  // keeps the view out of local memory
    boundary_value(h.faceBC[f], UL, nx, ny, h.faceCenter[2 * f], h.faceCenter[2 * f + 1], t, h.gamma, far, UR);
  }
  return nred;
}

// all gauss-point states of face f (diagnostic)
template <class T>
DG_HD int face_states(int64_t f, const HotView<T>& h, double t, double UL[3][4], double UR[3][4], double& nx,
                      double& ny, double& area) {
  int32_t L = h.faceL[f], R = h.faceR[f];
  nx = h.faceNormal[2 * f]; ny = h.faceNormal[2 * f + 1]; area = h.faceArea[f];
  double uL[4], uR[4] = {0, 0, 0, 0};
  load4<T>(&h.u[(int64_t)L * 4], uL);
  if (R >= 0) load4<T>(&h.u[(int64_t)R * 4], uR);
  T incL[3][4], incR[3][4];
  face_increments(f, L, R, h, incL, incR);
  int nred = 0;
  for (int g = 0; g < 3; g++) nred += gp_states(f, R, h, t, nx, ny, uL, uR, incL[g], incR[g], UL[g], UR[g]);
  return nred;
}

// face flux: sum over gauss points of -F(UL,UR).n |n| w (fluxFace, DNDS_FV_EulerEvaluator.hpp:371-591)
// returns the reduced-order count; *bad is set on non-physical input
// BND = false: an interior (or periodic) face, so no boundary-state code is compiled in
template <class T, int RIEMANN, bool BND>
DG_HD int face_flux(int64_t f, const HotView<T>& h, double t, double out[4], bool& bad) {
  int32_t L = h.faceL[f], R = h.faceR[f];
  double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1], area = h.faceArea[f];
  double uL[4], uR[4] = {0, 0, 0, 0};
  load4<T>(&h.u[(int64_t)L * 4], uL);
  if (!BND || R >= 0) load4<T>(&h.u[(int64_t)R * 4], uR);
  double dl = h.dLam[f];
  T incL[3][4], incR[3][4];
  face_increments(f, L, R, h, incL, incR);
  int nred = 0;
  double acc[4] = {0, 0, 0, 0};
  for (int g = 0; g < 3; g++) {
    double UL[4], UR[4], a[4], b[4], F[4];
    nred += gp_states<T, BND>(f, R, h, t, nx, ny, uL, uR, incL[g], incR[g], UL, UR);
    to_normal_frame(UL, nx, ny, a);
    to_normal_frame(UR, nx, ny, b);
    if (!(a[0] > 0 && b[0] > 0)) bad = true;
    if (RIEMANN == 2) hllc_flux(a, b, h.gamma, F);
    else roe_flux(a, b, h.gamma, dl, F);
    from_normal_frame(F, nx, ny);
    double jw = 0.5 * area * l3_weight(g);
    for (int k = 0; k < 4; k++) acc[k] -= F[k] * jw;
  }
  for (int k = 0; k < 4; k++) {
    if (!(acc[k] == acc[k])) bad = true;
    out[k] = acc[k];
  }
  return nred;
}

// Sutherland's law at a state (fluxFace, DNDS_FV_EulerEvaluator.hpp:405-412): T = p / ((gamma-1)/gamma Cp rho)
template <class T>
DG_HD double sutherland_mu(const HotView<T>& h, double p, double rho) {
  const double Tm = p / ((h.gamma - 1) / h.gamma * h.cp * rho);
  return h.mu * pow(Tm / h.tRef, 1.5) * (h.tRef + h.cSuth) / (Tm + h.cSuth);
}

// Gas::ViscousFlux_IdealGas (DNDS_Gas.hpp:795-826), 2-D, contracted with the unit normal;
// G[i][v] = d U_v / d x_i of the conservative variables
DG_HD void viscous_flux_n(const double U[4], const double G[2][4], double nx, double ny, bool adiabatic,
                          double gamma, double mu, double k, double cp, double Fn[4]) {
  const double ir = 1.0 / U[0];
  const double v0 = U[1] * ir, v1 = U[2] * ir;
  double S[2][2];  // d u_j / d x_i
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) S[i][j] = (U[0] * G[i][1 + j] - G[i][0] * U[1 + j]) * ir * ir;
  const double p = (gamma - 1) * (U[3] - U[0] * 0.5 * (v0 * v0 + v1 * v1));
  double gT[2];
  for (int i = 0; i < 2; i++) {
    const double gP = (gamma - 1) * (G[i][3] - 0.5 * (G[i][1] * v0 + G[i][2] * v1 + S[i][0] * U[1] + S[i][1] * U[2]));
    gT[i] = gamma / ((gamma - 1) * cp * U[0] * U[0]) * (U[0] * gP - p * G[i][0]);
  }
  if (adiabatic) {
    const double d = gT[0] * nx + gT[1] * ny;
    gT[0] -= d * nx;
    gT[1] -= d * ny;
  }
  const double tr = S[0][0] + S[1][1];
  const double txx = 2 * S[0][0] * mu - 2.0 / 3.0 * mu * tr, tyy = 2 * S[1][1] * mu - 2.0 / 3.0 * mu * tr;
  const double txy = (S[0][1] + S[1][0]) * mu;
  Fn[0] = 0;
  Fn[1] = nx * txx + ny * txy;
  Fn[2] = nx * txy + ny * tyy;
  Fn[3] = nx * (txx * v0 + txy * v1 + k * gT[0]) + ny * (txy * v0 + tyy * v1 + k * gT[1]);
}

// reconstructed gradient of cell `cell` (side 0 = left, 1 = right) at gauss point g of face f
template <class T>
DG_HD void face_grad(int64_t f, int side, int g, int64_t cell, const HotView<T>& h, double G[2][4]) {
  const T* rc = &h.urec[cell * 20];
  for (int d = 0; d < 2; d++) {
    for (int v = 0; v < 4; v++) G[d][v] = 0.0;
    for (int q = 0; q < 5; q++) {
      const double b = (double)h.faceGrad[aos(f, ((side * 3 + g) * 2 + d) * 5 + q, 60)];
      for (int v = 0; v < 4; v++) G[d][v] += b * (double)rc[4 * q + v];
    }
  }
}

// face flux with the Navier-Stokes viscous term (fluxFace, DNDS_FV_EulerEvaluator.hpp:371-591, and
// the face gradient of EvaluateRHS, DNDS_FV_EulerEvaluator.cpp:279-370): the mean of both sides'
// reconstructed gradients (the inner one's on a boundary face) plus (UR - UL) n / distGRP with
// distGRP = 2 min(V_L, V_R) / A, no jump term at walls; viscous flux at the mean state, Sutherland
// viscosity, k = Cp mu / Pr, adiabatic at a no-slip wall
template <class T, int RIEMANN, bool BND>
DG_HD int face_flux_vis(int64_t f, const HotView<T>& h, double t, double out[4], bool& bad) {
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
  T incL[3][4], incR[3][4];
  face_increments(f, L, R, h, incL, incR);
  int nred = 0;
  double acc[4] = {0, 0, 0, 0};
  for (int g = 0; g < 3; g++) {
    double UL[4], UR[4], a[4], b[4], F[4];
    nred += gp_states<T, BND>(f, R, h, t, nx, ny, uL, uR, incL[g], incR[g], UL, UR);
    to_normal_frame(UL, nx, ny, a);
    to_normal_frame(UR, nx, ny, b);
    if (!(a[0] > 0 && b[0] > 0)) bad = true;
    if (RIEMANN == 2) hllc_flux(a, b, h.gamma, F);
    else roe_flux(a, b, h.gamma, dl, F);
    from_normal_frame(F, nx, ny);
    double GL[2][4], GR[2][4], G[2][4], Um[4], Fv[4];
    face_grad(f, 0, g, L, h, GL);
    if (inner) face_grad(f, 1, g, R, h, GR);
    for (int v = 0; v < 4; v++) {
      const double jump = invD * (UR[v] - UL[v]);
      G[0][v] = 0.5 * (GL[0][v] + (inner ? GR[0][v] : GL[0][v])) + jump * nx;
      G[1][v] = 0.5 * (GL[1][v] + (inner ? GR[1][v] : GL[1][v])) + jump * ny;
      Um[v] = 0.5 * (UL[v] + UR[v]);
    }
    const double pm = (h.gamma - 1) * (Um[3] - 0.5 * (Um[1] * Um[1] + Um[2] * Um[2]) / Um[0]);
    const double mu = sutherland_mu(h, pm, Um[0]);
    viscous_flux_n(Um, G, nx, ny, bc == BC_WALL_NOSLIP, h.gamma, mu, h.cp * mu / h.pr, h.cp, Fv);
    const double jw = 0.5 * area * l3_weight(g);
    for (int k = 0; k < 4; k++) acc[k] -= (F[k] - Fv[k]) * jw;
  }
  for (int k = 0; k < 4; k++) {
    if (!(acc[k] == acc[k])) bad = true;
    out[k] = acc[k];
  }
  return nred;
}

// F(U0 + d) - F(U0) of the normal-frame Euler flux, evaluated from the
// increments so that FP32 rounding scales with |d|, not with |F|
DG_HD void flux_delta_f32(const float U[4], const float d[4], float gamma, float D[4]) {
  const float rho = U[0], m = U[1], k = U[2], E = U[3];
  const float ir = 1.0f / rho, u = m * ir, v = k * ir;
  const float p = (gamma - 1.0f) * (E - 0.5f * (m * u + k * v));
  const float irn = 1.0f / (rho + d[0]);
  const float du = (d[1] - u * d[0]) * irn, dv = (d[2] - v * d[0]) * irn;
  const float un = u + du, vn = v + dv;
  const float dp = (gamma - 1.0f) * (d[3] - 0.5f * (m * du + d[1] * un + k * dv + d[2] * vn));
  D[0] = d[1];
  D[1] = m * du + d[1] * un + dp;
  D[2] = k * du + d[2] * un;
  D[3] = (E + p) * du + (d[3] + dp) * un;
}

// physical flux F(U).n of a cell mean in the x-y frame, FP64
DG_HD void flux_n_f64(const double U[4], double nx, double ny, double gamma, double F[4]) {
  const double ir = 1.0 / U[0];
  const double u = U[1] * ir, v = U[2] * ir;
  const double p = (gamma - 1) * (U[3] - 0.5 * (U[1] * u + U[2] * v));
  const double un = u * nx + v * ny;
  F[0] = U[0] * un;
  F[1] = U[1] * un + p * nx;
  F[2] = U[2] * un + p * ny;
  F[3] = (U[3] + p) * un;
}

// Roe flux of an interior face for the FP32-bulk path, in flux-difference form:
//   F(UL,UR) = 1/2 (F(uL) + F(uR))                      FP64, once per face
//            + 1/2 (F(UL) - F(uL) + F(UR) - F(uR))      FP32 from the increments
//            - 1/2 R |Lambda| L (UR - UL)               FP32, UR - UL formed from an FP64 mean difference
// uL/uR are the cell means, UL = uL + phi_L . urec_L at each gauss point.  The
// algebra is that of Gas::RoeFlux_IdealGas_HartenYee<2,0> (DNDS_Gas.hpp:406-654).
DG_HD int face_flux_roe_delta32(int64_t f, const HotView<float>& h, double out[4], bool& bad) {
  const int32_t L = h.faceL[f], R = h.faceR[f];
  const double nxd = h.faceNormal[2 * f], nyd = h.faceNormal[2 * f + 1], area = h.faceArea[f];
  double uL[4], uR[4];
  load4<float>(&h.u[(int64_t)L * 4], uL);
  load4<float>(&h.u[(int64_t)R * 4], uR);
  float incL[3][4], incR[3][4];
  face_increments(f, L, R, h, incL, incR);
  const float gamma = (float)h.gamma, dl = (float)h.dLam[f];
  const float nx = (float)nxd, ny = (float)nyd;
  // FP64 part: area * (F(uL) + F(uR)) / 2
  double FL[4], FR[4];
  flux_n_f64(uL, nxd, nyd, h.gamma, FL);
  flux_n_f64(uR, nxd, nyd, h.gamma, FR);
  // normal-frame FP32 bases and the mean jump
  float bL[4], bR[4], dmean[4];
  {
    float tL[4] = {(float)uL[0], (float)uL[1], (float)uL[2], (float)uL[3]};
    float tR[4] = {(float)uR[0], (float)uR[1], (float)uR[2], (float)uR[3]};
    float tD[4] = {(float)(uR[0] - uL[0]), (float)(uR[1] - uL[1]), (float)(uR[2] - uL[2]), (float)(uR[3] - uL[3])};
    to_normal_frame(tL, nx, ny, bL);
    to_normal_frame(tR, nx, ny, bR);
    to_normal_frame(tD, nx, ny, dmean);
  }
  int nred = 0;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int g = 0; g < 3; g++) {
    float dL[4], dR[4];
    to_normal_frame(incL[g], nx, ny, dL);
    to_normal_frame(incR[g], nx, ny, dR);
    // CompressRecPart: fall back to the mean where density or internal energy would be negative
    float UL[4], UR[4];
    for (int v = 0; v < 4; v++) { UL[v] = bL[v] + dL[v]; UR[v] = bR[v] + dR[v]; }
    // rho < 0 or internal energy E - |m|^2 / (2 rho) < 0, i.e. 2 rho E < |m|^2 for rho > 0
    if (UL[0] < 0.f || 2.f * UL[0] * UL[3] < UL[1] * UL[1] + UL[2] * UL[2]) {
      for (int v = 0; v < 4; v++) { dL[v] = 0.f; UL[v] = bL[v]; }
      nred++;
    }
    if (UR[0] < 0.f || 2.f * UR[0] * UR[3] < UR[1] * UR[1] + UR[2] * UR[2]) {
      for (int v = 0; v < 4; v++) { dR[v] = 0.f; UR[v] = bR[v]; }
      nred++;
    }
    if (!(UL[0] > 0.f && UR[0] > 0.f)) bad = true;
    float DL[4], DR[4];
    flux_delta_f32(bL, dL, gamma, DL);
    flux_delta_f32(bR, dR, gamma, DR);
    // Roe average and wave strengths of dU = (uR - uL) + (dR - dL)
    const float irL = 1.0f / UL[0], irR = 1.0f / UR[0];
    const float u1 = UL[1] * irL, v1 = UL[2] * irL, u2 = UR[1] * irR, v2 = UR[2] * irR;
    const float pL = (gamma - 1.0f) * (UL[3] - 0.5f * (UL[1] * u1 + UL[2] * v1));
    const float pR = (gamma - 1.0f) * (UR[3] - 0.5f * (UR[1] * u2 + UR[2] * v2));
    const float HL = (UL[3] + pL) * irL, HR = (UR[3] + pR) * irR;
    const float sL = sqrtf(UL[0]), sR = sqrtf(UR[0]), isum = 1.0f / (sL + sR);
    const float u = (sL * u1 + sR * u2) * isum, v = (sL * v1 + sR * v2) * isum;
    const float vs = u * u + v * v;
    const float H = (sL * HL + sR * HR) * isum;
    const float a2 = (gamma - 1.0f) * (H - 0.5f * vs);
    const float a = sqrtf(a2);
    float lam0 = fabsf(u - a), lam1 = fabsf(u), lam3 = fabsf(u + a);
    const float thr = fmaxf(0.05f * (sqrtf(vs) + a), dl), thrS = thr * thr;
    if (lam0 < thr) lam0 = (lam0 * lam0 + thrS) / (2.0f * thr);
    if (lam3 < thr) lam3 = (lam3 * lam3 + thrS) / (2.0f * thr);
    const float d0 = dmean[0] + (dR[0] - dL[0]), d1 = dmean[1] + (dR[1] - dL[1]);
    const float d2 = dmean[2] + (dR[2] - dL[2]), d3 = dmean[3] + (dR[3] - dL[3]);
    const float al2 = d2 - v * d0;
    const float d3b = d3 - al2 * v;
    const float al1 = (gamma - 1.0f) / a2 * (d0 * (H - u * u) + u * d1 - d3b);
    const float al0 = (d0 * (u + a) - d1 - a * al1) / (2.0f * a);
    const float al3 = d0 - (al0 + al1);
    const float w0 = lam0 * al0, w1 = lam1 * al1, w2 = lam1 * al2, w3 = lam3 * al3;
    float G[4];
    G[0] = 0.5f * (DL[0] + DR[0]) - 0.5f * (w0 + w1 + w3);
    G[1] = 0.5f * (DL[1] + DR[1]) - 0.5f * ((u - a) * w0 + u * w1 + (u + a) * w3);
    G[2] = 0.5f * (DL[2] + DR[2]) - 0.5f * (v * (w0 + w1 + w3) + w2);
    G[3] = 0.5f * (DL[3] + DR[3]) - 0.5f * ((H - u * a) * w0 + 0.5f * vs * w1 + v * w2 + (H + u * a) * w3);
    from_normal_frame(G, nx, ny);
    const float jw = (float)(0.5 * area * l3_weight(g));
    for (int k = 0; k < 4; k++) acc[k] += G[k] * jw;
  }
  for (int k = 0; k < 4; k++) {
    out[k] = -(area * 0.5 * (FL[k] + FR[k]) + (double)acc[k]);
    if (!(out[k] == out[k])) bad = true;
  }
  return nred;
}

// HLLC flux of an interior face for the FP32-bulk path, in flux-difference form.  With the flux
// jump dF = F(UR) - F(UL) and the contact-speed offset sigma = S* - u_L, the HLLC flux of
// Gas::HLLCFlux_IdealGas_HartenYee<2> (DNDS_Gas.hpp:312-403) is, exactly:
//   0 <= SL:      F = F_mid - dF / 2                      SR <= 0:  F = F_mid + dF / 2
//   S* >= 0:      F = F_mid - dF / 2 + SL (U*L - UL)      else:     F = F_mid + dF / 2 + SR (U*R - UR)
//   F_mid = (F(UL) + F(UR)) / 2,  U*K - UK = (sigma_K / (SK - S*)) UK + chi_K sigma_K (0, rho_K, 0, rho_K S* + p_K / (SK - u_K)),
//   chi_K = (SK - u_K) / (SK - S*),  sigma_L = (dp - rho_R (SR - u_R) du) / (rho_L (SL - u_L) - rho_R (SR - u_R)),
//   sigma_R = sigma_L - du
// (the reference's star flux ((UK SK - FK) S* + D* (p_K + rho_K (SK - u_K)(S* - u_K)) SK) / (SK - S*)
// written as FK + SK (U*K - UK)).  F_mid is 1/2 (F(uL) + F(uR)) in FP64 once per face plus the FP32
// increments 1/2 (F(UL) - F(uL) + F(UR) - F(uR)); the jumps dF, du, dp are formed from the FP64 mean
// difference plus the FP32 increment difference, so every FP32 term's rounding scales with the
// reconstruction increment or the jump across the face, not with the flux itself.
DG_HD int face_flux_hllc_delta32(int64_t f, const HotView<float>& h, double out[4], bool& bad) {
  const int32_t L = h.faceL[f], R = h.faceR[f];
  const double nxd = h.faceNormal[2 * f], nyd = h.faceNormal[2 * f + 1], area = h.faceArea[f];
  double uL[4], uR[4];
  load4<float>(&h.u[(int64_t)L * 4], uL);
  load4<float>(&h.u[(int64_t)R * 4], uR);
  float incL[3][4], incR[3][4];
  face_increments(f, L, R, h, incL, incR);
  const float gamma = (float)h.gamma, gm1 = gamma - 1.0f;
  const float nx = (float)nxd, ny = (float)nyd;
  double FL[4], FR[4];
  flux_n_f64(uL, nxd, nyd, h.gamma, FL);
  flux_n_f64(uR, nxd, nyd, h.gamma, FR);
  float bL[4], bR[4], dmean[4], dFmean[4];
  {
    const float tL[4] = {(float)uL[0], (float)uL[1], (float)uL[2], (float)uL[3]};
    const float tR[4] = {(float)uR[0], (float)uR[1], (float)uR[2], (float)uR[3]};
    const float tD[4] = {(float)(uR[0] - uL[0]), (float)(uR[1] - uL[1]), (float)(uR[2] - uL[2]), (float)(uR[3] - uL[3])};
    const float tF[4] = {(float)(FR[0] - FL[0]), (float)(FR[1] - FL[1]), (float)(FR[2] - FL[2]), (float)(FR[3] - FL[3])};
    to_normal_frame(tL, nx, ny, bL);
    to_normal_frame(tR, nx, ny, bR);
    to_normal_frame(tD, nx, ny, dmean);
    to_normal_frame(tF, nx, ny, dFmean);
  }
  int nred = 0;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int g = 0; g < 3; g++) {
    float dL[4], dR[4];
    to_normal_frame(incL[g], nx, ny, dL);
    to_normal_frame(incR[g], nx, ny, dR);
    float UL[4], UR[4];
    for (int v = 0; v < 4; v++) { UL[v] = bL[v] + dL[v]; UR[v] = bR[v] + dR[v]; }
    // CompressRecPart: the mean where density or internal energy would be negative
    if (UL[0] < 0.f || 2.f * UL[0] * UL[3] < UL[1] * UL[1] + UL[2] * UL[2]) {
      for (int v = 0; v < 4; v++) { dL[v] = 0.f; UL[v] = bL[v]; }
      nred++;
    }
    if (UR[0] < 0.f || 2.f * UR[0] * UR[3] < UR[1] * UR[1] + UR[2] * UR[2]) {
      for (int v = 0; v < 4; v++) { dR[v] = 0.f; UR[v] = bR[v]; }
      nred++;
    }
    if (!(UL[0] > 0.f && UR[0] > 0.f)) bad = true;
    float DL[4], DR[4];
    flux_delta_f32(bL, dL, gamma, DL);
    flux_delta_f32(bR, dR, gamma, DR);
    float J[4], dF[4], G[4];
    for (int v = 0; v < 4; v++) {
      J[v] = dmean[v] + (dR[v] - dL[v]);
      dF[v] = dFmean[v] + (DR[v] - DL[v]);
      G[v] = 0.5f * (DL[v] + DR[v]);
    }
    const float rL = UL[0], rR = UR[0], irL = 1.0f / rL, irR = 1.0f / rR;
    const float uL1 = UL[1] * irL, vL1 = UL[2] * irL, uR1 = UR[1] * irR, vR1 = UR[2] * irR;
    const float pL = gm1 * (UL[3] - 0.5f * (UL[1] * uL1 + UL[2] * vL1));
    const float pR = gm1 * (UR[3] - 0.5f * (UR[1] * uR1 + UR[2] * vR1));
    // exact jumps of the normal velocity, tangential velocity and pressure from J
    const float du = (J[1] - uL1 * J[0]) * irR, dv = (J[2] - vL1 * J[0]) * irR;
    const float dp = gm1 * (J[3] - 0.5f * (UL[1] * du + J[1] * uR1 + UL[2] * dv + J[2] * vR1));
    const float sL = sqrtf(rL), sR = sqrtf(rR), isum = 1.0f / (sL + sR);
    const float um = (sL * uL1 + sR * uR1) * isum;
    const float eta2 = 0.5f * (sL * sR) * isum * isum;
    const float dsqr = (gamma * pL * irL * sL + gamma * pR * irR * sR) * isum + eta2 * du * du;
    const float sq = sqrtf(dsqr), SL = um - sq, SR = um + sq;
    if (0.f <= SL) {
      for (int v = 0; v < 4; v++) G[v] -= 0.5f * dF[v];
    } else if (SR <= 0.f) {
      for (int v = 0; v < 4; v++) G[v] += 0.5f * dF[v];
    } else {
      const float div = rL * (SL - uL1) - rR * (SR - uR1);
      const float sigL = fabsf(div) > 1e-37f ? (dp - rR * (SR - uR1) * du) / div : -uL1;  // S* = 0 if degenerate
      const float SS = uL1 + sigL;
      if (SS >= 0.f) {
        const float d = SL - SS;
        for (int v = 0; v < 4; v++) G[v] -= 0.5f * dF[v];
        if (fabsf(d) >= 1e-37f) {
          const float a = sigL / d, chi = (SL - uL1) / d;
          const float q1 = chi * sigL * rL, q3 = chi * sigL * (rL * SS + pL / (SL - uL1));
          G[0] += SL * (a * UL[0]);
          G[1] += SL * (a * UL[1] + q1);
          G[2] += SL * (a * UL[2]);
          G[3] += SL * (a * UL[3] + q3);
        }
      } else {
        const float d = SR - SS, sigR = sigL - du;
        for (int v = 0; v < 4; v++) G[v] += 0.5f * dF[v];
        if (fabsf(d) >= 1e-37f) {
          const float a = sigR / d, chi = (SR - uR1) / d;
          const float q1 = chi * sigR * rR, q3 = chi * sigR * (rR * SS + pR / (SR - uR1));
          G[0] += SR * (a * UR[0]);
          G[1] += SR * (a * UR[1] + q1);
          G[2] += SR * (a * UR[2]);
          G[3] += SR * (a * UR[3] + q3);
        }
      }
    }
    from_normal_frame(G, nx, ny);
    const float jw = (float)(0.5 * area * l3_weight(g));
    for (int k = 0; k < 4; k++) acc[k] += G[k] * jw;
  }
  for (int k = 0; k < 4; k++) {
    out[k] = -(area * 0.5 * (FL[k] + FR[k]) + (double)acc[k]);
    if (!(out[k] == out[k])) bad = true;
  }
  return nred;
}

// EvaluateDt face part (DNDS_FV_EulerEvaluator.cpp:25-137): lambda_f * area, deltaLambdaFace
template <class T>
DG_HD void dt_face(int64_t f, const HotView<T>& h) {
  int32_t L = h.faceL[f], R = h.faceR[f];
  double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1], area = h.faceArea[f];
  double UL[4];
  load4<T>(&h.u[(int64_t)L * 4], UL);
  double pL, aL2, HL, pR, aR2, HR;
  double uL = UL[1] / UL[0], vL = UL[2] / UL[0], uR = uL, vR = vL;
  thermal(UL[3], UL[0], uL * uL + vL * vL, h.gamma, pL, aL2, HL);
  pR = pL; aR2 = aL2;
  double rhoMean = UL[0];
  if (R >= 0) {
    double UR[4];
    load4<T>(&h.u[(int64_t)R * 4], UR);
    rhoMean = (UL[0] + UR[0]) * 0.5;
    uR = UR[1] / UR[0]; vR = UR[2] / UR[0];
    thermal(UR[3], UR[0], uR * uR + vR * vR, h.gamma, pR, aR2, HR);
  }
  double vn = 0.5 * ((uL + uR) * nx + (vL + vR) * ny);
  double pMean = (pL + pR) * 0.5;
  double lam = fabs(vn) + sqrt(h.gamma * pMean / rhoMean);
  if (h.mu > 0) {  // viscous part (DNDS_FV_EulerEvaluator.cpp:80-99)
    const double lamVis = sutherland_mu(h, pMean, rhoMean) / rhoMean * dmax(4. / 3., h.gamma / h.pr);
    lam += lamVis * area * (1.0 / h.vol[L] + 1.0 / (R >= 0 ? h.vol[R] : h.vol[L]));
  }
  h.lamA[f] = lam * area;
  h.dLam[f] = fabs((uR - uL) * nx + (vR - vL) * ny) + sqrt(fabs(aR2 - aL2)) * 0.7071;
}

// EvaluateDt cell part: dt_i = min(CFL V / sum lambda_f A_f, MaxDt)
template <class T>
DG_HD double dt_cell(int64_t i, const HotView<T>& h, double cfl, double maxDt) {
  double lam = 0;
  for (int k = 0; k < h.nfmax; k++) {
    int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    int32_t f = sf >= 0 ? sf : ~sf;
    lam += h.lamA[f];
  }
  return dmin(cfl * h.vol[i] / (lam + 1e-100), maxDt);
}

// rhs of cell i: gather of face fluxes plus the flux-balance term
// (DNDS_FV_EulerEvaluator.cpp:501-508): -F(u_i) . sum_f n_f A_f / V_i
template <class T>
DG_HD void cell_rhs(int64_t i, const HotView<T>& h, double r[4]) {
  double s[4] = {0, 0, 0, 0};
  for (int k = 0; k < h.nfmax; k++) {
    int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    int32_t f = sf >= 0 ? sf : ~sf;
    const double* fl = &h.flux[(int64_t)f * 4];
    if (sf >= 0) { for (int v = 0; v < 4; v++) s[v] += fl[v]; }
    else { for (int v = 0; v < 4; v++) s[v] -= fl[v]; }
  }
  double U[4];
  load4<T>(&h.u[i * 4], U);
  double ir = 1.0 / U[0];
  double vx = U[1] * ir, vy = U[2] * ir;
  double p = (h.gamma - 1) * (U[3] - U[0] * 0.5 * (vx * vx + vy * vy));
  double cx = h.closure[2 * i], cy = h.closure[2 * i + 1];
  double Fn[4] = {U[1] * cx + U[2] * cy, (U[1] * vx + p) * cx + U[1] * vy * cy, U[2] * vx * cx + (U[2] * vy + p) * cy,
                  (U[3] + p) * (vx * cx + vy * cy)};
  double iv = 1.0 / h.vol[i];
  for (int v = 0; v < 4; v++) r[v] = (s[v] - Fn[v]) * iv;
}

}  // namespace dg

namespace dg {

// ---------------------------------------------------------------- setup bodies
// face part of initBaseDiffCache (DNDS_FV_VR.cpp:367-890): weights, geometry
// and the value-row basis of both cells at the face gauss points
// gradient rows (d/dx, d/dy) of both cells' basis at the face gauss points, for the viscous flux
template <class T>
DG_HD void setup_face_grad(int64_t f, const MeshView& m, const CellSetup* cells, T* grad) {
  const FaceGeom g = face_geom(f, m);
  const int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
  const double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
  for (int side = 0; side < 2; side++)
    for (int q = 0; q < 3; q++) {
      double D[6][5];
      if (side == 0) p2_diffs(cells[L].fr, g.gx[q], g.gy[q], D);
      else if (R >= 0) p2_diffs(cells[R].fr, g.gx[q] - sx, g.gy[q] - sy, D);
      else for (int r = 0; r < 6; r++) for (int k = 0; k < 5; k++) D[r][k] = 0;
      for (int d = 0; d < 2; d++)
        for (int k = 0; k < 5; k++) grad[aos(f, ((side * 3 + q) * 2 + d) * 5 + k, 60)] = (T)D[1 + d][k];
    }
}

template <class T>
DG_HD void setup_face(int64_t f, const MeshView& m, const SetupParams& p, const CellSetup* cells, double* faceW,
                      double* normal, double* area, double* center, double* w0, T* basis) {
  FaceGeom g = face_geom(f, m);
  double W[6];
  face_weights(f, m, p, g, cells, W);
  for (int k = 0; k < 6; k++) faceW[f * 6 + k] = W[k];
  normal[2 * f] = g.nx; normal[2 * f + 1] = g.ny;
  area[f] = g.area;
  center[2 * f] = g.cx; center[2 * f + 1] = g.cy;
  w0[f] = W[0];
  int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
  double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
  // gauss point 2 minus the face centre (gauss point 1): s_2 (x1 - x0) / 2
  const int32_t a = m.face_nodes[2 * f], b = m.face_nodes[2 * f + 1];
  const double hx = l3_point(2) * 0.5 * (m.node_xy[2 * b] - m.node_xy[2 * a]);
  const double hy = l3_point(2) * 0.5 * (m.node_xy[2 * b + 1] - m.node_xy[2 * a + 1]);
  for (int side = 0; side < 2; side++) {
    double rec[kFaceBasisSide] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (side == 0 || R >= 0) {
      const CellFrame& fr = cells[side ? R : L].fr;
      const double ox = side ? sx : 0.0, oy = side ? sy : 0.0;
      p2_values(fr, g.gx[1] - ox, g.gy[1] - oy, rec);
      p2_frame_coords(fr, g.gx[1] - ox, g.gy[1] - oy, rec[5], rec[6]);
      rec[7] = fr.Pinv[0][0] * hx + fr.Pinv[0][1] * hy;
      rec[8] = fr.Pinv[1][0] * hx + fr.Pinv[1][1] * hy;
    }
    for (int k = 0; k < kFaceBasisSide; k++) basis[aos(f, side * kFaceBasisSide + k, kFaceBasisE)] = (T)rec[k];
  }
}

// initReconstructionMatVec (DNDS_FV_VR.cpp:892-1154) for one cell:
// A = sum_faces sum_gp |n| w F(D_i, D_i), B_k = ... F(D_i, D_j), b_k = w0^2 D_i[0];
// stores A^-1 B_k and A^-1 b_k per face slot.  Returns false if A is not SPD.
template <class T>
DG_HD bool setup_cell_matrices(int64_t i, const MeshView& m, const SetupParams& p, const CellSetup* cells,
                               const double* faceW, const int32_t* cellFace, int nfmax, T* vrOp, double* vrOpD,
                               int32_t* vrNbr, int32_t* vrMode, int32_t* vrFace, double* Ainv) {
  const int E = nfmax * 30;
  double A[5][5];
  double B[4][5][5], bv[4][5];
  int mode[4], nbr[4], face[4];
  for (int r = 0; r < 5; r++) for (int q = 0; q < 5; q++) A[r][q] = 0;
  for (int k = 0; k < nfmax; k++) {
    mode[k] = VR_EMPTY; nbr[k] = -1; face[k] = -1;
    for (int r = 0; r < 5; r++) { bv[k][r] = 0; for (int q = 0; q < 5; q++) B[k][r][q] = 0; }
    int32_t sf = cellFace[aos(i, k, nfmax)];
    if (sf == kEmptySlot) continue;
    int32_t f = sf >= 0 ? sf : ~sf;
    int side = sf >= 0 ? 0 : 1;
    int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
    int32_t j = side == 0 ? R : L;
    int bc = m.face_bc[f];
    FaceGeom g = face_geom(f, m);
    const double* W = &faceW[f * 6];
    double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
    // own points: the cell on the right of a periodic face sees the face shifted back
    double ox = side == 1 ? -sx : 0.0, oy = side == 1 ? -sy : 0.0;
    double jx = side == 0 ? -sx : 0.0, jy = side == 0 ? -sy : 0.0;
    double tm = tang_modifier(p, cells[L].vol, cells[R >= 0 ? R : L].vol, g.area);
    FaceFunctional Fn = make_functional(W, g.nx, g.ny, p.tang_weight, tm, p.tang_weight_mod_loc);
    bool far = R < 0 && is_far_type(bc);
    for (int q = 0; q < 3; q++) {
      double jw = 0.5 * g.area * l3_weight(q);
      double D[6][5], P[6][5];
      p2_diffs(cells[i].fr, g.gx[q] + ox, g.gy[q] + oy, D);
      functional_proj(Fn, D, P);
      for (int r = 0; r < 5; r++)
        for (int c = 0; c < 5; c++) {
          double s = 0;
          for (int a = 0; a < 6; a++) s += P[a][r] * P[a][c];
          A[r][c] += s * jw;
          if (far) B[k][r][c] += s * jw;
        }
      if (j >= 0) {
        double Dj[6][5], Pj[6][5];
        p2_diffs(cells[j].fr, g.gx[q] + jx, g.gy[q] + jy, Dj);
        functional_proj(Fn, Dj, Pj);
        for (int r = 0; r < 5; r++)
          for (int c = 0; c < 5; c++) {
            double s = 0;
            for (int a = 0; a < 6; a++) s += P[a][r] * Pj[a][c];
            B[k][r][c] += s * jw;
          }
      }
      for (int r = 0; r < 5; r++) bv[k][r] += W[0] * W[0] * D[0][r] * jw;
    }
    face[k] = f;
    if (j >= 0) { mode[k] = VR_INNER; nbr[k] = j; }
    else if (far) { mode[k] = VR_FAR; nbr[k] = (int32_t)i; }
    else if (bc == BC_WALL) { mode[k] = VR_WALL; nbr[k] = -1; }
    else if (bc == BC_WALL_EULER || bc == BC_WALL_NOSLIP) { mode[k] = VR_WALLCORR; nbr[k] = -1; }
    else { mode[k] = VR_EMPTY; }
  }
  double Lc[5][5];
  for (int r = 0; r < 5; r++) for (int q = 0; q < 5; q++) Lc[r][q] = A[r][q];
  if (!chol5(Lc)) return false;
  double Ai[5][5];
  for (int c = 0; c < 5; c++) {
    double col[5];
    for (int r = 0; r < 5; r++) col[r] = r == c ? 1.0 : 0.0;
    chol5_solve_vec(Lc, col);
    for (int r = 0; r < 5; r++) Ai[r][c] = col[r];
  }
  if (Ainv)
    for (int r = 0; r < 5; r++) for (int q = 0; q < 5; q++) Ainv[i * 25 + r * 5 + q] = Ai[r][q];
  for (int k = 0; k < nfmax; k++) {
    vrNbr[aos(i, k, nfmax)] = nbr[k];
    vrMode[aos(i, k, nfmax)] = mode[k];
    vrFace[aos(i, k, nfmax)] = face[k];
    for (int r = 0; r < 5; r++) {
      for (int c = 0; c < 5; c++) {
        double s = 0;
        for (int t = 0; t < 5; t++) s += Ai[r][t] * B[k][t][c];
        vrOp[aos(i, k * 30 + r * 5 + c, E)] = (T)s;
        if (vrOpD) vrOpD[aos(i, k * 30 + r * 5 + c, E)] = s;
      }
      double s = 0;
      for (int t = 0; t < 5; t++) s += Ai[r][t] * bv[k][t];
      vrOp[aos(i, k * 30 + 25 + r, E)] = (T)s;
      if (vrOpD) vrOpD[aos(i, k * 30 + 25 + r, E)] = s;
    }
  }
  return true;
}

}  // namespace dg

namespace dg {

// ---------------------------------------------------------------- thread-per-(item, sub-item) bodies
// VR sweep of one variable v of cell i, relax = 1, split in two phases so a
// kernel can issue every neighbour gather before it waits for its operator tile:
//   vr_var_prefetch: slot modes, the neighbours' coefficients of variable v and
//                    the mean differences du (NF = faces per cell, compile time);
//   vr_var_compute:  acc[r] = sum_k (A^-1B_k urec_j(k))[r][v] + (A^-1b_k)[r] du_k[v].
// Four threads (v = 0..3) cooperate on a cell.  Wall_Euler / Wall_NoSlip slots
// are skipped here and added by vr_wall_fixup.
template <class T, int NF>
struct VrPre {
  int mode[NF];
  T rv[NF][5];
  T du[NF];
};
template <class T, int NF>
DG_HD void vr_var_prefetch(int64_t i, int v, const HotView<T>& h, VrPre<T, NF>& p) {
  const double uiv = h.u[i * 4 + v];
  for (int k = 0; k < NF; k++) {
    const int mode = h.vrMode[aos(i, k, NF)];
    const int32_t j = h.vrNbr[aos(i, k, NF)];
    p.mode[k] = mode;
    const bool rec = mode == VR_INNER || mode == VR_FAR;
    const T* rj = &h.urec[(int64_t)(rec ? j : i) * 20 + v];
    for (int q = 0; q < 5; q++) p.rv[k][q] = rec ? rj[4 * q] : T(0);
    const double uj = mode == VR_INNER ? h.u[(int64_t)j * 4 + v] : 0.0;
    p.du[k] = (mode == VR_INNER || mode == VR_WALL) ? T(uj - uiv) : T(0);
  }
}
template <class T, int NF, class Op>
DG_HD void vr_var_compute(int64_t i, int v, const HotView<T>& h, const VrPre<T, NF>& p, const Op& opk) {
  T acc[5] = {T(0), T(0), T(0), T(0), T(0)};
  for (int k = 0; k < NF; k++) {
    const int mode = p.mode[k];
    if (mode == VR_EMPTY || mode == VR_WALLCORR) continue;
    for (int r = 0; r < 5; r++) {
      T s = acc[r] + opk(k, 25 + r) * p.du[k];
      for (int q = 0; q < 5; q++) s += opk(k, r * 5 + q) * p.rv[k][q];
      acc[r] = s;
    }
  }
  T* out = &h.urecNew[i * 20 + v];
  for (int q = 0; q < 5; q++) out[4 * q] = acc[q];
}
template <class T, class Op>
DG_HD void vr_cell_var(int64_t i, int v, const HotView<T>& h, const Op& opk) {
  if (h.nfmax == 3) {
    VrPre<T, 3> p;
    vr_var_prefetch<T, 3>(i, v, h, p);
    vr_var_compute<T, 3>(i, v, h, p, opk);
  } else {
    VrPre<T, 4> p;
    vr_var_prefetch<T, 4>(i, v, h, p);
    vr_var_compute<T, 4>(i, v, h, p, opk);
  }
}

// Wall_Euler / Wall_NoSlip slots of cell i (DNDS_FV_VR.hpp:1577-1665): adds relax * A^-1 * (integral of
// the weighted jump to the wall state) to urecNew, for conservative component c only (the wall state of
// an Euler wall couples the momentum components, so every component's face value is formed, but the
// jump, its integral and the A^-1 product of component c are independent of the others)
template <class T>
DG_HD void vr_wall_fixup(int64_t i, int c, const HotView<T>& h) {
  double ui[4];
  for (int v = 0; v < 4; v++) ui[v] = h.u[i * 4 + v];
  double add[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < h.nfmax; k++) {
    if (h.vrMode[aos(i, k, h.nfmax)] != VR_WALLCORR) continue;
    int32_t f = h.vrFace[aos(i, k, h.nfmax)];
    double nx = h.faceNormal[2 * f], ny = h.faceNormal[2 * f + 1];
    double w0 = h.faceW0[f], area = h.faceArea[f];
    int bc = h.faceBC[f];
    double corr[5] = {0, 0, 0, 0, 0};
    const FaceBasisSide<T> fb(h.faceBasis, f, 0);
    for (int g = 0; g < 3; g++) {
      double phi[5], uBL[4];
      T pg[5];
      fb.at(g, pg);
      for (int q = 0; q < 5; q++) phi[q] = (double)pg[q];
      for (int v = 0; v < 4; v++) {
        double s = 0;
        for (int q = 0; q < 5; q++) s += phi[q] * (double)h.urec[i * 20 + q * 4 + v];
        uBL[v] = s + ui[v];
      }
      double uBVc;
      if (bc == BC_WALL_EULER) {
        const double d = nx * uBL[1] + ny * uBL[2];
        uBVc = c == 1 ? uBL[1] - nx * d : (c == 2 ? uBL[2] - ny * d : uBL[c]);
      } else {
        uBVc = (c == 1 || c == 2) ? -uBL[c] : uBL[c];
      }
      double jw = 0.5 * area * l3_weight(g);
      for (int q = 0; q < 5; q++) corr[q] += phi[q] * w0 * w0 * (uBVc - ui[c]) * jw;
    }
    const double* Ai = &h.Ainv[i * 25];
    for (int r = 0; r < 5; r++) {
      double s = 0;
      for (int q = 0; q < 5; q++) s += Ai[r * 5 + q] * corr[q];
      add[r] += s;
    }
  }
  for (int r = 0; r < 5; r++) h.urecNew[i * 20 + r * 4 + c] += T(h.relax * add[r]);
}

}  // namespace dg
