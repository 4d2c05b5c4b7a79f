// Host checks of the limiter's building blocks (dndsg_limiter.cuh compiled as plain C++; the
// device-only limiting pass is never instantiated here).  Built as a shared library by
// tests/test_limiter_host.py.
//
// char_rows: the rows of the left (L) and right (R) characteristic matrices at the face mean state,
// in FP64 and in the FP32 branch (reciprocals of rho, a^2 and gamma - 1).  R L must be the identity,
// and the FP32 rows must agree with the FP64 ones to FP32 resolution.
// wbap_biway: the FP32 version (hardware-style quotients, the 1e9 cap on the ratio) against FP64.
#define __device__
#define __forceinline__ inline
#include <algorithm>
#include <cmath>

#include "dndsg_limiter.cuh"

using namespace dg;

template <class C>
static double identity_error(const double* UL, const double* UR, double gamma, double nx, double ny, double Lout[4][4]) {
  C L[4][4], R[4][4];
  for (int a = 0; a < 4; a++) char_rows<C>(a, (C)gamma, UL, UR, (C)nx, (C)ny, L[a], R[a]);
  double err = 0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += (double)R[i][k] * (double)L[k][j];
      err = std::max(err, std::fabs(s - (i == j ? 1.0 : 0.0)));
      Lout[i][j] = (double)L[i][j];
    }
  return err;
}

// states: n x 8 (UL then UR, conservative), normals: n x 2 (unit).  Outputs: max |R L - I| in FP64
// and FP32, and the largest difference of an FP32 row entry from the FP64 one relative to that row's
// largest FP64 entry.
extern "C" void char_rows_check(int n, const double* states, const double* normals, double gamma, double* err64,
                                double* err32, double* diff32) {
  *err64 = *err32 = *diff32 = 0;
  for (int s = 0; s < n; s++) {
    const double* UL = states + 8 * s;
    const double* UR = UL + 4;
    const double nx = normals[2 * s], ny = normals[2 * s + 1];
    double L64[4][4], L32[4][4];
    *err64 = std::max(*err64, identity_error<double>(UL, UR, gamma, nx, ny, L64));
    *err32 = std::max(*err32, identity_error<float>(UL, UR, gamma, nx, ny, L32));
    for (int i = 0; i < 4; i++) {
      double rowMax = 0;
      for (int j = 0; j < 4; j++) rowMax = std::max(rowMax, std::fabs(L64[i][j]));
      for (int j = 0; j < 4; j++) *diff32 = std::max(*diff32, std::fabs(L32[i][j] - L64[i][j]) / rowMax);
    }
  }
}

// the largest |biway32 - biway64| relative to |u1| (u1 != 0) over n pairs
extern "C" double biway_check(int n, const double* u1, const double* u2, double nn) {
  double worst = 0;
  for (int s = 0; s < n; s++) {
    const double r64 = wbap_biway(u1[s], u2[s], nn);
    const double r32 = (double)wbap_biway((float)u1[s], (float)u2[s], (float)nn);
    worst = std::max(worst, std::fabs(r32 - r64) / std::fabs(u1[s]));
  }
  return worst;
}
