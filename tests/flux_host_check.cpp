// Host check of the FP32-bulk interior face fluxes (dndsg_bodies.cuh compiled as plain C++):
// face_flux_roe_delta32 and face_flux_hllc_delta32 (flux-difference form, FP64 means and central flux,
// FP32 increments, jumps and wave terms) against the FP64 face_flux on the same face data.  One face per
// sample, its own two cells; the FP64 view holds the FP32 view's coefficients and basis record exactly,
// so the two differ only by the arithmetic.  Built as a shared library by tests/test_flux_host.py.
#include <algorithm>
#include <cmath>
#include <vector>

#include "dndsg_bodies.cuh"

using namespace dg;

// n faces; u: 2n x 4 cell means (cell 2f left of face f, 2f + 1 right), urec: 2n x 20 coefficients,
// basis: n x 18 record values (side 0 then side 1), normal: n x 2, area, dlam: n.  riemann 1 Roe,
// 2 HLLC.  err[f] = max_k |F32_k - F64_k|, scale[f] = max_k |F64_k|, reduced[f] = the Gauss points
// each path sent to the positivity fallback (FP32 + 8 x FP64; at most 6 each).  Returns the number of
// faces either path flagged.
extern "C" int flux_check(int64_t n, int riemann, const double* u, const float* urec, const float* basis,
                          const double* normal, const double* area, const double* dlam, double gamma, double* err,
                          double* scale, int32_t* reduced) {
  std::vector<int32_t> faceL(n), faceR(n);
  for (int64_t f = 0; f < n; f++) { faceL[f] = (int32_t)(2 * f); faceR[f] = (int32_t)(2 * f + 1); }
  std::vector<float> fb32(aos_size(n, kFaceBasisE));
  std::vector<double> fb64(aos_size(n, kFaceBasisE)), urec64(40 * n);
  for (int64_t f = 0; f < n; f++)
    for (int e = 0; e < kFaceBasisE; e++) {
      fb32[aos(f, e, kFaceBasisE)] = basis[f * kFaceBasisE + e];
      fb64[aos(f, e, kFaceBasisE)] = (double)basis[f * kFaceBasisE + e];
    }
  for (int64_t k = 0; k < 40 * n; k++) urec64[k] = (double)urec[k];
  HotView<float> h32{};
  HotView<double> h64{};
  h32.N = h64.N = 2 * n;
  h32.F = h64.F = n;
  h32.faceL = h64.faceL = faceL.data();
  h32.faceR = h64.faceR = faceR.data();
  h32.faceNormal = h64.faceNormal = normal;
  h32.faceArea = h64.faceArea = area;
  h32.dLam = h64.dLam = const_cast<double*>(dlam);
  h32.u = h64.u = const_cast<double*>(u);
  h32.urec = const_cast<float*>(urec);
  h64.urec = urec64.data();
  h32.faceBasis = fb32.data();
  h64.faceBasis = fb64.data();
  h32.gamma = h64.gamma = gamma;
  int flagged = 0;
  for (int64_t f = 0; f < n; f++) {
    double o32[4], o64[4];
    bool b32 = false, b64 = false;
    int r32, r64;
    if (riemann == 2) {
      r32 = face_flux_hllc_delta32(f, h32, o32, b32);
      r64 = face_flux<double, 2, false>(f, h64, 0.0, o64, b64);
    } else {
      r32 = face_flux_roe_delta32(f, h32, o32, b32);
      r64 = face_flux<double, 1, false>(f, h64, 0.0, o64, b64);
    }
    reduced[f] = r32 + 8 * r64;
    flagged += (b32 || b64) ? 1 : 0;
    err[f] = scale[f] = 0;
    for (int k = 0; k < 4; k++) {
      err[f] = std::max(err[f], std::fabs(o32[k] - o64[k]));
      scale[f] = std::max(scale[f], std::fabs(o64[k]));
    }
  }
  return flagged;
}
