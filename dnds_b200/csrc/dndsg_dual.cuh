// Dual time stepping of the reference's implicit driver, included at the end of dndsg.cu:
//   ImplicitBDFDualTimeStep (order 1-4)      DNDS_ODE.hpp:392-497, BDFCoefs :500-505
//   ImplicitSDIRK4DualTimeStep (3 stages)    DNDS_ODE.hpp:269-390
// with the EulerSolver lambdas fdtau / frhs / fsolve / fstop (DNDS_FV_EulerSolver.hpp:713-1061), and
// fsolve's Krylov option: GMRES_LeftPreconditioned (DNDS_Linear.hpp:12-107) over LUSGSMatrixVec
// (DNDS_FV_EulerEvaluator.cpp:1062-1143), the LU-SGS forward + backward sweeps being the left
// preconditioner.  Contexts with 4 variables, and SA contexts (the U5 part of every vector after
// the [N][4] flow part; its rhs and increment pass through CompressInc as in fsolve).
//
// Vectors are the [N][4] increments / states in device memory.  The Arnoldi loop keeps the
// Hessenberg matrix on the device (dot products by a two-pass reduction whose summation order
// is fixed, so repeated runs give the same bits); the host reads it once per restart cycle for the
// (k+1) x k least-squares problem, and reads beta (the break test) once per cycle.

namespace {

// BDFCoefs: row k-1 = {alphaDiag, coefficient of xLast, of the step before, ...}
constexpr double kBdfCoef[4][5] = {{1.0, 1.0, 0.0, 0.0, 0.0},
                                   {2. / 3., 4. / 3., -1. / 3., 0.0, 0.0},
                                   {6. / 11., 18. / 11., -9. / 11., 2. / 11., 0.0},
                                   {12. / 25., 48. / 25., -36. / 25., 16. / 25., -3. / 25.}};

// the 3-stage, 4th-order SDIRK tableau with zeta = 0.128886400515 (butcherA / butcherB / butcherC)
struct Sdirk4 {
  double A[3][3], b[3], c[3];
};
inline Sdirk4 sdirk4_tableau() {
  const double z = 0.128886400515, d = (2 * z - 1) * (2 * z - 1);
  Sdirk4 t{};
  t.A[0][0] = z;
  t.A[1][0] = 0.5 - z;
  t.A[1][1] = z;
  t.A[2][0] = 2 * z;
  t.A[2][1] = 1 - 4 * z;
  t.A[2][2] = z;
  t.b[0] = 1. / (6 * d);
  t.b[1] = (4 * z * z - 4 * z + 2. / 3.) / d;
  t.b[2] = 1. / (6 * d);
  t.c[0] = z;
  t.c[1] = 0.5;
  t.c[2] = 1 - z;
  return t;
}

constexpr int kMaxKrylov = 32;
struct VecList {
  const double* p[kMaxKrylov + 1];
  double a[kMaxKrylov + 1];
};

// BDF right-hand side, in place on rhs = R(x) (DNDS_ODE.hpp:454-466):
// rhs *= a0; rhs += x * (-1/dt); rhs += X_m * (c_m / dt) for xLast and the stored earlier steps
__global__ void __launch_bounds__(kBlock) k_dual_bdf_rhs(int64_t n, const double* x, double a0, double negInvDt,
                                                         VecList X, int m, double* rhs) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  double r = rhs[e] * a0;
  r += x[e] * negInvDt;
  for (int k = 0; k < m; k++) r += X.p[k][e] * X.a[k];
  rhs[e] = r;
}

// SDIRK stage right-hand side (DNDS_ODE.hpp:330-336): rhs = (xLast - x) * (1/dt) + sum_j R_j a_j
__global__ void __launch_bounds__(kBlock) k_dual_sdirk_rhs(int64_t n, const double* xLast, const double* x,
                                                           double invDt, VecList R, int m, double* rhs) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  double r = xLast[e];
  r -= x[e];
  r *= invDt;
  for (int k = 0; k < m; k++) r += R.p[k][e] * R.a[k];
  rhs[e] = r;
}

// x = base + sum_k V_k a_k (base may alias x; base NULL keeps x)
__global__ void __launch_bounds__(kBlock) k_vec_combine(int64_t n, const double* base, VecList V, int m, double* x) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  double r = base ? base[e] : x[e];
  for (int k = 0; k < m; k++) r += V.p[k][e] * V.a[k];
  x[e] = r;
}

// x *= a, or x *= 1 / s[0] with s on the device
__global__ void __launch_bounds__(kBlock) k_vec_scale(int64_t n, double* x, double a, const double* s) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  x[e] *= s ? 1.0 / s[0] : a;
}

// classical Gram-Schmidt subtraction with the projections on the device:
// w += V_i * (-h_i) for i = 0..m-1 in that order
__global__ void __launch_bounds__(kBlock) k_gs_subtract(int64_t n, double* w, VecList V, int m, const double* h) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  double r = w[e];
  for (int k = 0; k < m; k++) r += V.p[k][e] * (-h[k]);
  w[e] = r;
}

// dot products of w with V_0..V_{m-1}: per-block partial sums (fixed grid, fixed tree), then one
// block per product sums the partials in a fixed order; sqrt of the result on request (norm2)
constexpr int kDotBlocks = 296;
__device__ __forceinline__ double block_sum_fixed(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}
__global__ void __launch_bounds__(kBlock) k_dots_partial(int64_t n, const double* w, VecList V, int m,
                                                         double* partial) {
  __shared__ double sh[32];
  for (int k = 0; k < m; k++) {
    double a = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
      a += w[e] * V.p[k][e];
    a = block_sum_fixed(a, sh);
    if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = a;
  }
}
__global__ void __launch_bounds__(kBlock) k_dots_final(const double* partial, int nb, double* out, int root) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  double a = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) a += partial[k * nb + b];
  a = block_sum_fixed(a, sh);
  if (threadIdx.x == 0) out[k] = root ? sqrt(a) : a;
}

// LUSGSMatrixVec: Ax_i = D_i x_i + sum over every neighbour j of (alpha/2) A_f / V_i
// dF(u_j; n_out, x_j, lambda_f), i.e. D x - uIncNewBuf with uIncNewBuf -= (alpha/2) A/V fInc
template <class T>
__global__ void __launch_bounds__(kBlock) k_lusgs_matvec(HotView<T> h, double alpha, const double* D,
                                                         const double* x, double* Ax) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= h.N) return;
  double buf[4] = {0, 0, 0, 0};
  for (int k = 0; k < h.nfmax; k++) {
    const int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    const int32_t f = sf >= 0 ? sf : ~sf;
    const int32_t j = sf >= 0 ? h.faceR[f] : h.faceL[f];
    if (j < 0) continue;
    const double sg = sf >= 0 ? 1.0 : -1.0;
    const double area = h.faceArea[f];
    double U[4], dU[4], dF[4];
    load4<T>(&h.u[(int64_t)j * 4], U);
    load4<double>(&x[(int64_t)j * 4], dU);
    flux_jac_times_du(U, sg * h.faceNormal[2 * f], sg * h.faceNormal[2 * f + 1], dU, h.lamA[f] / area, h.gamma, dF);
    const double w = (0.5 * alpha) * area / h.vol[i];
    for (int v = 0; v < 4; v++) buf[v] -= w * dF[v];
  }
  const double d = D[i];
  for (int v = 0; v < 4; v++) Ax[i * 4 + v] = d * x[i * 4 + v] - buf[v];
}

// the U5 row of LUSGSMatrixVec: Ax5_i = D5_i x5_i + sum_j (alpha/2) A_f / V_i dF5 with
// dF5 = x5_j vn + u5_j dvn - lambda_f x5_j (the U5 entry of fluxJacobian0_Right_Times_du)
template <class T>
__global__ void __launch_bounds__(kBlock) k_lusgs_matvec_sa5(HotView<T> h, const double* u5, double alpha,
                                                             const double* D5, const double* x4, const double* x5,
                                                             double* Ax5) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= h.N) return;
  double buf = 0;
  for (int k = 0; k < h.nfmax; k++) {
    const int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    const int32_t f = sf >= 0 ? sf : ~sf;
    const int32_t j = sf >= 0 ? h.faceR[f] : h.faceL[f];
    if (j < 0) continue;
    const double sg = sf >= 0 ? 1.0 : -1.0, area = h.faceArea[f];
    const double nx = sg * h.faceNormal[2 * f], ny = sg * h.faceNormal[2 * f + 1], lam = h.lamA[f] / area;
    double U[4], dU[4];
    load4<T>(&h.u[(int64_t)j * 4], U);
    load4<double>(&x4[(int64_t)j * 4], dU);
    const double ir = 1.0 / U[0];
    const double vn = (U[1] * nx + U[2] * ny) * ir;
    const double dvn = ((dU[1] - U[1] * ir * dU[0]) * nx + (dU[2] - U[2] * ir * dU[0]) * ny) * ir;
    const double dS = x5[j];
    const double dF = dS * vn + u5[j] * dvn - dS * lam;
    buf -= (0.5 * alpha) * area / h.vol[i] * dF;
  }
  Ax5[i] = D5[i] * x5[i] - buf;
}

// CompressInc of the U5 right-hand side as fsolve applies it: rhs = CompressInc(u, rhs dTau) / dTau
__global__ void k_sa_compress_rhs(int64_t N, const double* u, const double* dt, double alpha, double* rhs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double dTau = dt[i] / alpha;
  rhs[i] = sa_compress_inc(u[i], rhs[i] * dTau) / dTau;
}
// CompressInc of the U5 increment in place
__global__ void k_sa_compress_inc(int64_t N, const double* u, double* inc) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < N) inc[i] = sa_compress_inc(u[i], inc[i]);
}

inline unsigned vgrid(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

struct DualOpts {
  int scheme, order;
  double cfl;
  int maxIter;
  double threshold;
  int nRec, volWise, gmresCode, nSpace, nRestart;
};

int ensure_dual(dndsg_ctx* c, const DualOpts& o) {
  int rc;
  if ((rc = ensure_lusgs(c))) return rc;
  const size_t bytes = sizeof(double) * (c->sa ? 5 : 4) * c->N;  // [N][4] flow, then [N] U5
  const size_t nOde = o.scheme == DNDSG_DUAL_SDIRK4 ? 3 : (size_t)(o.order - 1);
  while (c->odeVec.size() < nOde) {
    double* p = nullptr;
    if ((rc = dalloc(c, p, bytes))) return rc;
    c->odeVec.push_back(p);
  }
  if (c->sa && !c->saDmat && (rc = dalloc(c, c->saDmat, sizeof(double) * c->N))) return rc;
  if (o.gmresCode != 0) {
    while (c->gmV.size() < (size_t)o.nSpace + 1) {
      double* p = nullptr;
      if ((rc = dalloc(c, p, bytes))) return rc;
      c->gmV.push_back(p);
    }
    if (!c->gmTmp)
      if ((rc = dalloc(c, c->gmTmp, bytes)) || (rc = dalloc(c, c->gmMLb, bytes)) ||
          (rc = dalloc(c, c->gmB, bytes)) || (rc = dalloc(c, c->gmX, bytes)) ||
          (rc = dalloc(c, c->gmH, sizeof(double) * (kMaxKrylov + 1) * (kMaxKrylov + 1))) ||
          (rc = dalloc(c, c->gmPartial, sizeof(double) * (kMaxKrylov + 1) * kDotBlocks)))
        return rc;
  }
  return 0;
}

// out[k] = dot(w, V_k) (or its square root), k < m, on the device
inline int64_t dual_len(const dndsg_ctx* c) { return (c->sa ? 5 : 4) * c->N; }

void launch_dots(dndsg_ctx* c, const double* w, const VecList& V, int m, double* out, bool root, cudaStream_t s) {
  const int64_t n = dual_len(c);
  k_dots_partial<<<kDotBlocks, kBlock, 0, s>>>(n, w, V, m, c->gmPartial);
  k_dots_final<<<m, kBlock, 0, s>>>(c->gmPartial, kDotBlocks, out, root ? 1 : 0);
}

// the preconditioner FML: LU-SGS forward + backward with rhs x into MLx
template <class T>
void gmres_fml(dndsg_ctx* c, double alpha, const double* x, double* MLx, cudaStream_t s) {
  if (c->sa) {
    const int64_t n4 = 4 * c->N;
    launch_lusgs_sweep_sa<T>(c, true, alpha, x, MLx, x + n4, MLx + n4, s);
    launch_lusgs_sweep_sa<T>(c, false, alpha, x, MLx, x + n4, MLx + n4, s);
    return;
  }
  launch_lusgs_sweep<T>(c, true, alpha, x, MLx, s);
  launch_lusgs_sweep<T>(c, false, alpha, x, MLx, s);
}
// the matrix FA: LUSGSMatrixVec (the U5 row as well for SA contexts)
template <class T>
void gmres_fa(dndsg_ctx* c, double alpha, const double* x, double* Ax, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  k_lusgs_matvec<T><<<grid_for(c->N), kBlock, 0, s>>>(h, alpha, c->Dmat, x, Ax);
  if (c->sa) {
    const int64_t n4 = 4 * c->N;
    k_lusgs_matvec_sa5<T><<<grid_for(c->N), kBlock, 0, s>>>(h, c->saU, alpha, c->saDmat, x, x + n4, Ax + n4);
  }
}

// least squares min |h y - beta e1| for the (k+1) x k upper Hessenberg h (column j at h + j (K+1)),
// by Givens rotations and back substitution
void hessenberg_lsq(const double* hcols, int K, int k, double beta, double* y) {
  std::vector<double> R((size_t)(k + 1) * k), g(k + 1, 0.0);
  for (int j = 0; j < k; j++)
    for (int i = 0; i <= k; i++) R[(size_t)i * k + j] = hcols[(size_t)j * (K + 1) + i];
  g[0] = beta;
  for (int j = 0; j < k; j++) {
    const double a = R[(size_t)j * k + j], b = R[(size_t)(j + 1) * k + j];
    const double r = std::hypot(a, b);
    const double cs = r == 0.0 ? 1.0 : a / r, sn = r == 0.0 ? 0.0 : b / r;
    for (int q = j; q < k; q++) {
      const double x0 = R[(size_t)j * k + q], x1 = R[(size_t)(j + 1) * k + q];
      R[(size_t)j * k + q] = cs * x0 + sn * x1;
      R[(size_t)(j + 1) * k + q] = -sn * x0 + cs * x1;
    }
    const double g0 = g[j], g1 = g[j + 1];
    g[j] = cs * g0 + sn * g1;
    g[j + 1] = -sn * g0 + cs * g1;
  }
  for (int j = k - 1; j >= 0; j--) {
    double v = g[j];
    for (int q = j + 1; q < k; q++) v -= R[(size_t)j * k + q] * y[q];
    y[j] = v / R[(size_t)j * k + j];
  }
}

// GMRES_LeftPreconditioned::solve with FStop always false (the EulerSolver's), x in place
template <class T>
int gmres_solve(dndsg_ctx* c, int K, int nRestart, double alpha, const double* b, double* x, cudaStream_t s) {
  const int64_t n = dual_len(c);
  double* const H = c->gmH;
  gmres_fml<T>(c, alpha, b, c->gmMLb, s);
  std::vector<double> hHost((size_t)(K + 1) * K), y(K);
  for (int iRestart = 0; iRestart <= nRestart; iRestart++) {
    double* V0 = c->gmV[0];
    gmres_fa<T>(c, alpha, x, c->gmTmp, s);
    gmres_fml<T>(c, alpha, c->gmTmp, V0, s);
    VecList m1{};
    m1.p[0] = c->gmMLb;
    m1.a[0] = -1.0;
    k_vec_combine<<<vgrid(n), kBlock, 0, s>>>(n, nullptr, m1, 1, V0);
    VecList self{};
    self.p[0] = V0;
    launch_dots(c, V0, self, 1, H + (size_t)K * (K + 1), true, s);  // beta in the spare last column
    double beta = 0.0;
    DG_CUDA(c, cudaMemcpyAsync(&beta, H + (size_t)K * (K + 1), sizeof(double), cudaMemcpyDeviceToHost, s));
    DG_CUDA(c, cudaStreamSynchronize(s));
    if (std::abs(beta) < 1e-200 || iRestart == nRestart) break;
    k_vec_scale<<<vgrid(n), kBlock, 0, s>>>(n, V0, -1.0 / beta, nullptr);
    for (int j = 0; j < K; j++) {
      double* w = c->gmV[j + 1];
      gmres_fa<T>(c, alpha, c->gmV[j], c->gmTmp, s);
      gmres_fml<T>(c, alpha, c->gmTmp, w, s);
      VecList V{};
      for (int i = 0; i <= j; i++) V.p[i] = c->gmV[i];
      double* hcol = H + (size_t)j * (K + 1);
      launch_dots(c, w, V, j + 1, hcol, false, s);
      k_gs_subtract<<<vgrid(n), kBlock, 0, s>>>(n, w, V, j + 1, hcol);
      VecList ws{};
      ws.p[0] = w;
      launch_dots(c, w, ws, 1, hcol + j + 1, true, s);
      k_vec_scale<<<vgrid(n), kBlock, 0, s>>>(n, w, 0.0, hcol + j + 1);
    }
    DG_CUDA(c, cudaMemcpyAsync(hHost.data(), H, sizeof(double) * (K + 1) * K, cudaMemcpyDeviceToHost, s));
    DG_CUDA(c, cudaStreamSynchronize(s));
    hessenberg_lsq(hHost.data(), K, K, beta, y.data());
    VecList V{};
    for (int j = 0; j < K; j++) {
      V.p[j] = c->gmV[j];
      V.a[j] = y[j];
    }
    k_vec_combine<<<vgrid(n), kBlock, 0, s>>>(n, nullptr, V, K, x);
  }
  return check_launch(c);
}

// fdtau + frhs: local EvaluateDt at cfl (dTau = dt / alphaDiag is folded into the diagonal),
// nInternalRecStep Jacobi sweeps, [limiter], EvaluateRHS at tEval into c->rhs
template <class T>
void dual_frhs(dndsg_ctx* c, const DualOpts& o, double tEval, cudaStream_t s) {
  if (c->sa) {
    run_dt_sa<T>(c, o.cfl, 1e100, s);
    for (int k = 0; k < o.nRec; k++) run_vr_sa<T>(c, s);
    run_rhs_sa<T>(c, s);
    return;
  }
  run_dt<T>(c, o.cfl, 1e100, false, s);
  for (int k = 0; k < o.nRec; k++) run_vr<T>(c, false, s);
  if (c->s.limiter) run_limiter<T>(c, 0, s);
  run_rhs<T>(c, tEval, s);
}

// fsolve on rhs = c->rhs into c->inc (CompressInc is the identity for 4 variables)
template <class T>
int dual_fsolve(dndsg_ctx* c, const DualOpts& o, double dt, double alpha, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  const int64_t N = c->N, n4 = 4 * N;
  k_lusgs_init<T><<<grid_for(N), kBlock, 0, s>>>(h, 1.0 / dt, alpha, c->Dinv, c->Dmat);
  if (c->sa) {
    k_sa_diag<<<grid_for(N), kBlock, 0, s>>>(N, c->Dmat, c->saSrcJac, alpha, c->saDinv, c->saDmat);
    k_sa_compress_rhs<<<grid_for(N), kBlock, 0, s>>>(N, c->saU, c->dt, alpha, c->saRhs);
  }
  if (o.gmresCode == 0 || o.gmresCode == 2) {
    if (c->sa) {
      launch_lusgs_sweep_sa<T>(c, true, alpha, c->rhs, c->inc, c->saRhs, c->saInc, s);
      launch_lusgs_sweep_sa<T>(c, false, alpha, c->rhs, c->inc, c->saRhs, c->saInc, s);
      k_sa_compress_inc<<<grid_for(N), kBlock, 0, s>>>(N, c->saU, c->saInc);
    } else {
      launch_lusgs_sweep<T>(c, true, alpha, c->rhs, c->inc, s);
      launch_lusgs_sweep<T>(c, false, alpha, c->rhs, c->inc, s);
    }
  }
  if (o.gmresCode != 0) {
    if (o.gmresCode == 1) {
      DG_CUDA(c, cudaMemsetAsync(c->inc, 0, sizeof(double) * n4, s));
      if (c->sa) DG_CUDA(c, cudaMemsetAsync(c->saInc, 0, sizeof(double) * N, s));
    }
    if (!c->sa) return gmres_solve<T>(c, o.nSpace, o.nRestart, alpha, c->rhs, c->inc, s);
    // SA: the flow and U5 parts side by side in one vector for the Krylov solve
    DG_CUDA(c, cudaMemcpyAsync(c->gmB, c->rhs, sizeof(double) * n4, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(c, cudaMemcpyAsync(c->gmB + n4, c->saRhs, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(c, cudaMemcpyAsync(c->gmX, c->inc, sizeof(double) * n4, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(c, cudaMemcpyAsync(c->gmX + n4, c->saInc, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    int rc;
    if ((rc = gmres_solve<T>(c, o.nSpace, o.nRestart, alpha, c->gmB, c->gmX, s))) return rc;
    DG_CUDA(c, cudaMemcpyAsync(c->inc, c->gmX, sizeof(double) * n4, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(c, cudaMemcpyAsync(c->saInc, c->gmX + n4, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  }
  return 0;
}

// x += inc and fstop: the L1 increment norm (volume-weighted on request) against its running
// maximum over the iterations; true when the density entry drops below the threshold
struct Fstop {
  double base[5] = {0, 0, 0, 0, 0}, rel[5] = {0, 0, 0, 0, 0};
};
template <class T>
int dual_add_and_test(dndsg_ctx* c, const DualOpts& o, int iter, Fstop& f, bool& stop, cudaStream_t s) {
  DG_CUDA(c, cudaMemsetAsync(c->resAcc, 0, sizeof(double) * 16, s));
  k_add_inc<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->u, c->inc, c->vol, o.volWise, c->resAcc);
  if (c->sa)  // CompressInc of the U5 increment (after the Krylov solve too), u5 += inc
    k_sa_add_inc<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->saU, c->saInc, c->vol, o.volWise, c->resAcc + 8);
  double acc[16];
  DG_CUDA(c, cudaMemcpyAsync(acc, c->resAcc, sizeof(acc), cudaMemcpyDeviceToHost, s));
  DG_CUDA(c, cudaStreamSynchronize(s));
  const int nv = c->sa ? 5 : 4;
  double res[5] = {acc[0], acc[1], acc[2], acc[3], acc[8]};
  for (int v = 0; v < nv; v++) {
    f.base[v] = iter == 1 ? res[v] : std::max(f.base[v], res[v]);
    f.rel[v] = res[v] / f.base[v];
  }
  stop = f.rel[0] < o.threshold;
  return check_launch(c);
}

template <class T>
int dual_step(dndsg_ctx* c, const DualOpts& o, double dt, double t, int* itersOut, double* resOut, cudaStream_t s) {
  int rc;
  if ((rc = ensure_dual(c, o))) return rc;
  // a dual-time vector is [N][4] flow then, for SA contexts, [N] U5: the state, xLast and the rhs
  // live in separate arrays, so each vector operation runs once per part
  const int64_t N = c->N, n = 4 * N;
  const bool sa = c->sa;
  auto copy = [&](double* dst4, double* dst5, const double* src4, const double* src5) -> int {
    DG_CUDA(c, cudaMemcpyAsync(dst4, src4, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    if (sa) DG_CUDA(c, cudaMemcpyAsync(dst5, src5, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    return 0;
  };
  auto part5 = [&](VecList L, int m) {  // the same list, pointing at the U5 parts of the vectors
    for (int k = 0; k < m; k++) L.p[k] += n;
    return L;
  };
  if ((rc = copy(c->uLast, c->saULast, c->u, c->saU))) return rc;
  Fstop f;
  if (o.scheme == DNDSG_DUAL_BDF) {
    const int prevSiz = o.order - 1, kCur = c->odeCnPrev + 1;
    if (c->odeCnPrev > 0 && !(std::abs(c->odeDtPrev - dt) < dt * 1e-8))
      return fail(c, DNDSG_BAD_ARGUMENT, "BDF history holds steps of another dt: dndsg_dual_reset first");
    const double* coef = kBdfCoef[kCur - 1];
    int iter = 1;
    for (; iter <= o.maxIter; iter++) {
      dual_frhs<T>(c, o, t + 1.0 * dt, s);
      VecList X{};
      X.p[0] = c->uLast;
      X.a[0] = coef[1] / dt;
      for (int k = 0; k < c->odeCnPrev; k++) {
        X.p[1 + k] = c->odeVec[(size_t)((k + c->odePrevStart) % prevSiz)];
        X.a[1 + k] = coef[2 + k] / dt;
      }
      const int m = 1 + c->odeCnPrev;
      k_dual_bdf_rhs<<<vgrid(n), kBlock, 0, s>>>(n, c->u, coef[0], -1. / dt, X, m, c->rhs);
      if (sa) {
        VecList X5 = part5(X, m);
        X5.p[0] = c->saULast;
        k_dual_bdf_rhs<<<vgrid(N), kBlock, 0, s>>>(N, c->saU, coef[0], -1. / dt, X5, m, c->saRhs);
      }
      if ((rc = dual_fsolve<T>(c, o, dt, coef[0], s))) return rc;
      bool stop = false;
      if ((rc = dual_add_and_test<T>(c, o, iter, f, stop, s))) return rc;
      if (stop) break;
    }
    if (itersOut) itersOut[0] = std::min(iter, o.maxIter);
    if (prevSiz) {
      c->odePrevStart = ((c->odePrevStart - 1) % prevSiz + prevSiz) % prevSiz;
      double* h = c->odeVec[(size_t)c->odePrevStart];
      if ((rc = copy(h, h + n, c->uLast, c->saULast))) return rc;
      c->odeDtPrev = dt;
      c->odeCnPrev = std::min(c->odeCnPrev + 1, prevSiz);
    }
  } else {
    const Sdirk4 tb = sdirk4_tableau();
    for (int iB = 0; iB < 3; iB++) {
      if ((rc = copy(c->u, c->saU, c->uLast, c->saULast))) return rc;
      int iter = 1;
      for (; iter <= o.maxIter; iter++) {
        dual_frhs<T>(c, o, t + tb.c[iB] * dt, s);
        if ((rc = copy(c->odeVec[iB], c->odeVec[iB] + n, c->rhs, c->saRhs))) return rc;
        VecList R{};
        for (int j = 0; j <= iB; j++) {
          R.p[j] = c->odeVec[j];
          R.a[j] = tb.A[iB][j];
        }
        k_dual_sdirk_rhs<<<vgrid(n), kBlock, 0, s>>>(n, c->uLast, c->u, 1.0 / dt, R, iB + 1, c->rhs);
        if (sa)
          k_dual_sdirk_rhs<<<vgrid(N), kBlock, 0, s>>>(N, c->saULast, c->saU, 1.0 / dt, part5(R, iB + 1), iB + 1,
                                                       c->saRhs);
        if ((rc = dual_fsolve<T>(c, o, dt, tb.A[iB][iB], s))) return rc;
        bool stop = false;
        if ((rc = dual_add_and_test<T>(c, o, iter, f, stop, s))) return rc;
        if (stop) break;
      }
      if (itersOut) itersOut[iB] = std::min(iter, o.maxIter);
    }
    VecList R{};
    for (int j = 0; j < 3; j++) {
      R.p[j] = c->odeVec[j];
      R.a[j] = tb.b[j] * dt;
    }
    k_vec_combine<<<vgrid(n), kBlock, 0, s>>>(n, c->uLast, R, 3, c->u);
    if (sa) k_vec_combine<<<vgrid(N), kBlock, 0, s>>>(N, c->saULast, part5(R, 3), 3, c->saU);
  }
  if (resOut)
    for (int v = 0; v < (sa ? 5 : 4); v++) resOut[v] = f.rel[v];
  return check_launch(c);
}

// The steady internal loop of EulerSolver with ifSteadyQuit: first-order BDF pseudo-time
// iterations (DNDS_ODE.hpp:444-486) with the fstop lambda's CFL ramp (DNDS_FV_EulerSolver.hpp:
// 1047-1052), until the density fstop ratio drops below the threshold
template <class T>
int steady_solve(dndsg_ctx* c, const dndsg_steady_settings* st, int* itersOut, double* resOut, double* wallOut,
                 double* hist, cudaStream_t s) {
  DualOpts o{DNDSG_DUAL_BDF, 1, st->cfl, st->max_iter, st->threshold, st->n_rec, st->vol_wise,
             st->gmres_code, st->n_gmres_space, st->n_gmres_iter};
  int rc;
  if ((rc = ensure_dual(c, o))) return rc;
  const int64_t N = c->N, n = 4 * N;
  const bool sa = c->sa;
  const double dt = st->dt;
  DG_CUDA(c, cudaMemcpyAsync(c->uLast, c->u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  if (sa) DG_CUDA(c, cudaMemcpyAsync(c->saULast, c->saU, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  Fstop f;
  double cflNow = st->cfl, acc[16] = {0};
  int iter = 1;
  for (; iter <= st->max_iter; iter++) {
    o.cfl = cflNow;
    dual_frhs<T>(c, o, 0.0, s);
    VecList X{};
    X.p[0] = c->uLast;
    X.a[0] = 1.0 / dt;
    k_dual_bdf_rhs<<<vgrid(n), kBlock, 0, s>>>(n, c->u, 1.0, -1. / dt, X, 1, c->rhs);
    if (sa) {
      VecList X5{};
      X5.p[0] = c->saULast;
      X5.a[0] = 1.0 / dt;
      k_dual_bdf_rhs<<<vgrid(N), kBlock, 0, s>>>(N, c->saU, 1.0, -1. / dt, X5, 1, c->saRhs);
    }
    if ((rc = dual_fsolve<T>(c, o, dt, 1.0, s))) return rc;
    // x += inc with the increment norms, and the wall force of this iteration's residual
    DG_CUDA(c, cudaMemsetAsync(c->resAcc, 0, sizeof(double) * 16, s));
    k_add_inc<<<grid_for(N), kBlock, 0, s>>>(N, c->u, c->inc, c->vol, o.volWise, c->resAcc);
    if (sa) k_sa_add_inc<<<grid_for(N), kBlock, 0, s>>>(N, c->saU, c->saInc, c->vol, o.volWise, c->resAcc + 8);
    if (c->F > c->Fi) {
      k_wall_flux<<<grid_for(c->F - c->Fi), kBlock, 0, s>>>(c->Fi, c->F, c->faceBC, c->flux, c->resAcc + 4);
      if (sa) k_sa_wall_flux<<<grid_for(c->F - c->Fi), kBlock, 0, s>>>(c->Fi, c->F, c->faceBC, c->saFlux, c->resAcc + 9);
    }
    DG_CUDA(c, cudaMemcpyAsync(acc, c->resAcc, sizeof(acc), cudaMemcpyDeviceToHost, s));
    DG_CUDA(c, cudaStreamSynchronize(s));
    if ((rc = check_launch(c))) return rc;
    const double res[5] = {acc[0], acc[1], acc[2], acc[3], acc[8]};
    for (int v = 0; v < (sa ? 5 : 4); v++) {
      f.base[v] = iter == 1 ? res[v] : std::max(f.base[v], res[v]);
      f.rel[v] = res[v] / f.base[v];
    }
    if (hist) hist[iter - 1] = f.rel[0];
    if (!(res[0] == res[0])) return fail(c, DNDSG_NUMERIC_ERROR, "steady solve: NaN increment");
    if (f.rel[0] < st->threshold) break;
    if (iter >= st->cfl_ramp_start && iter <= st->cfl_ramp_start + st->cfl_ramp_length && st->cfl_ramp_length > 0) {
      const double inter = double(iter - st->cfl_ramp_start) / st->cfl_ramp_length;
      cflNow = std::exp(std::log(st->cfl) + std::log(st->cfl_ramp_end / st->cfl) * inter);
    }
  }
  if (itersOut) *itersOut = std::min(iter, st->max_iter);
  if (resOut)
    for (int v = 0; v < (sa ? 5 : 4); v++) resOut[v] = f.rel[v];
  if (wallOut) {
    for (int v = 0; v < 4; v++) wallOut[v] = acc[4 + v];
    if (sa) wallOut[4] = acc[9];
  }
  return 0;
}

int dual_opts(dndsg_ctx* c, const dndsg_dual_settings* d, DualOpts& o) {
  if (!d) return DNDSG_BAD_ARGUMENT;
  o = DualOpts{d->scheme, d->bdf_order, d->cfl, d->max_iter, d->threshold, d->n_rec, d->vol_wise,
               d->gmres_code, d->n_gmres_space, d->n_gmres_iter};
  if (o.scheme != DNDSG_DUAL_BDF && o.scheme != DNDSG_DUAL_SDIRK4)
    return fail(c, DNDSG_BAD_ARGUMENT, "scheme must be DNDSG_DUAL_BDF or DNDSG_DUAL_SDIRK4");
  if (o.scheme == DNDSG_DUAL_BDF && (o.order < 1 || o.order > 4))
    return fail(c, DNDSG_BAD_ARGUMENT, "bdf_order must be 1..4");
  if (!(o.cfl > 0) || o.maxIter < 1 || o.nRec < 0 || o.gmresCode < 0 || o.gmresCode > 2)
    return fail(c, DNDSG_BAD_ARGUMENT, "cfl > 0, max_iter >= 1, n_rec >= 0, gmres_code 0..2");
  if (o.gmresCode != 0 && (o.nSpace < 1 || o.nSpace > kMaxKrylov || o.nRestart < 0))
    return fail(c, DNDSG_BAD_ARGUMENT, "n_gmres_space must be 1..32 and n_gmres_iter >= 0");
  return 0;
}

}  // namespace

extern "C" {

int dndsg_dual_reset(dndsg_ctx* c) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  c->odeCnPrev = 0;
  c->odePrevStart = 0;
  c->odeOrder = 0;
  c->odeDtPrev = 0.0;
  return 0;
}

int dndsg_dual_step(dndsg_ctx* c, const dndsg_dual_settings* d, double dt, double t, int* iters_out, double* res_out,
                    void* s) {
  if (!c || !(dt > 0)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  DualOpts o;
  int rc;
  if ((rc = dual_opts(c, d, o)) || (rc = set_device(c))) return rc;
  if (o.scheme == DNDSG_DUAL_BDF && c->odeOrder != o.order) {  // a new ImplicitBDFDualTimeStep(k)
    c->odeCnPrev = 0;
    c->odePrevStart = o.order - 2 > 0 ? o.order - 2 : 0;
    c->odeOrder = o.order;
  }
  rc = c->fp32 ? dual_step<float>(c, o, dt, t, iters_out, res_out, st(s))
              : dual_step<double>(c, o, dt, t, iters_out, res_out, st(s));
  return rc ? rc : observe_timeout(c, st(s));
}

int dndsg_steady_solve(dndsg_ctx* c, const dndsg_steady_settings* ss, int* iters_out, double* res_out,
                       double* wall_flux_out, double* history, void* s) {
  if (!c || !ss) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (!(ss->cfl > 0) || !(ss->cfl_ramp_end > 0) || ss->max_iter < 1 || !(ss->dt > 0) || ss->n_rec < 0 ||
      ss->gmres_code < 0 || ss->gmres_code > 2 || ss->cfl_ramp_length < 0 ||
      (ss->gmres_code != 0 && (ss->n_gmres_space < 1 || ss->n_gmres_space > kMaxKrylov || ss->n_gmres_iter < 0)))
    return fail(c, DNDSG_BAD_ARGUMENT, "steady settings: cfl, cfl_ramp_end, dt > 0; max_iter >= 1; n_rec >= 0; "
                                       "gmres_code 0..2 with n_gmres_space 1..32");
  int rc;
  if ((rc = set_device(c))) return rc;
  rc = c->fp32 ? steady_solve<float>(c, ss, iters_out, res_out, wall_flux_out, history, st(s))
               : steady_solve<double>(c, ss, iters_out, res_out, wall_flux_out, history, st(s));
  return rc ? rc : observe_timeout(c, st(s));
}

int dndsg_gmres_lusgs(dndsg_ctx* c, double alpha, int n_space, int n_restart, const double* b, double* x, void* s) {
  if (!c || !b || !x || n_space < 1 || n_space > kMaxKrylov || n_restart < 0) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "4-variable contexts");
  if (!c->rankOf) return fail(c, DNDSG_BAD_ARGUMENT, "dndsg_lusgs_matrix_init first");
  DualOpts o{DNDSG_DUAL_BDF, 1, 1.0, 1, 0.0, 0, 0, 1, n_space, n_restart};
  int rc;
  if ((rc = set_device(c)) || (rc = ensure_dual(c, o))) return rc;
  return c->fp32 ? gmres_solve<float>(c, n_space, n_restart, alpha, b, x, st(s))
                 : gmres_solve<double>(c, n_space, n_restart, alpha, b, x, st(s));
}

int dndsg_lusgs_matvec(dndsg_ctx* c, double alpha, const double* x, double* ax, void* s) {
  if (!c || !x || !ax) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "4-variable contexts");
  if (!c->rankOf) return fail(c, DNDSG_BAD_ARGUMENT, "dndsg_lusgs_matrix_init first");
  int rc;
  if ((rc = set_device(c))) return rc;
  if (c->fp32) k_lusgs_matvec<float><<<grid_for(c->N), kBlock, 0, st(s)>>>(view<float>(c), alpha, c->Dmat, x, ax);
  else k_lusgs_matvec<double><<<grid_for(c->N), kBlock, 0, st(s)>>>(view<double>(c), alpha, c->Dmat, x, ax);
  return check_launch(c);
}

}  // extern "C"
