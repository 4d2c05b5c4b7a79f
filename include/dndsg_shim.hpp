// dndsg_shim.hpp -- header-only C++ shim over the dndsg C ABI with the call
// surface of the DNDS classes it replaces on the GPU:
//
//   VRFiniteVolume2DGPU::ReconstructionJacobiStep      VRFiniteVolume2D, DNDS_FV_VR.hpp:1474-1479
//   VRFiniteVolume2DGPU::ReconstructionWBAPLimitFacialV3  DNDS_FV_VR.hpp:2055-2061
//   EulerEvaluatorGPU::EvaluateDt                       EulerEvaluator, DNDS_FV_EulerEvaluator.hpp:1408-1411
//   EulerEvaluatorGPU::EvaluateRHS                      DNDS_FV_EulerEvaluator.hpp:1412-1418
//   EulerEvaluatorGPU::EvaluateResidual                 DNDS_FV_EulerEvaluator.hpp:1455-1461
//
// The reference's ArrayDOFV / ArrayRecV live in host memory and are passed to
// every call; here the state is resident on the GPU, and the shim moves it
// only when asked (PullState / PushState), i.e. at run start and end.
// Errors raise dndsg::Error (the reference aborts through DNDS_assert).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "dndsg.h"

namespace dndsg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error("dndsg error " + std::to_string(c) + ": " + m), code(c) {}
};

// Owns the context: mesh, VR setup and device state (one GPU)
class Context {
 public:
  Context(const dndsg_mesh_desc& mesh, const dndsg_settings& settings, int device = 0) {
    int rc = dndsg_create(&mesh, &settings, device, &ctx_);
    if (rc != DNDSG_OK) {
      std::string msg = ctx_ ? dndsg_last_error(ctx_) : "no context";
      if (ctx_) dndsg_destroy(ctx_);
      ctx_ = nullptr;
      throw Error(rc, msg);
    }
  }
  ~Context() {
    if (ctx_) dndsg_destroy(ctx_);
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;

  dndsg_ctx* get() const { return ctx_; }
  int64_t nCells() const { return dndsg_n_cells(ctx_); }
  void check(int rc) const {
    if (rc != DNDSG_OK) throw Error(rc, dndsg_last_error(ctx_));
  }
  // u: [nCells][nVars] cell means (ArrayDOFV order); uRec: [nCells][5][nVars]
  void PushState(const std::vector<double>& u, const std::vector<double>* uRec = nullptr, void* stream = nullptr) {
    check(dndsg_set_u(ctx_, u.data(), stream));
    if (uRec) check(dndsg_set_urec(ctx_, uRec->data(), stream));
  }
  void PullState(std::vector<double>& u, std::vector<double>* uRec = nullptr, void* stream = nullptr) const {
    u.resize(nCells() * 4);
    check(dndsg_get_u(ctx_, u.data(), stream));
    if (uRec) {
      uRec->resize(nCells() * 20);
      check(dndsg_get_urec(ctx_, uRec->data(), stream));
    }
  }

 private:
  dndsg_ctx* ctx_ = nullptr;
};

class VRFiniteVolume2DGPU {
 public:
  explicit VRFiniteVolume2DGPU(Context& c) : c_(c) {}
  // one Jacobi sweep of the resident uRec from the resident u (u/uRec/uRecNewBuf roles of the reference)
  void ReconstructionJacobiStep(int nSweeps = 1, void* stream = nullptr) {
    c_.check(dndsg_vr_jacobi_step(c_.get(), nSweeps, nullptr, stream));
  }
  // CWBAP limiting in place; ifUseLimiter (nullable) receives the smoothness indicator
  void ReconstructionWBAPLimitFacialV3(bool ifAll, std::vector<double>* ifUseLimiter = nullptr, void* stream = nullptr) {
    if (ifUseLimiter) ifUseLimiter->resize(c_.nCells());
    c_.check(dndsg_limiter_wbap(c_.get(), ifAll ? 1 : 0, ifUseLimiter ? ifUseLimiter->data() : nullptr, stream));
  }

 private:
  Context& c_;
};

class EulerEvaluatorGPU {
 public:
  explicit EulerEvaluatorGPU(Context& c) : c_(c) {}
  // dt: per-cell time steps (host copy), dtMinall: global minimum
  void EvaluateDt(std::vector<double>& dt, double CFL, double& dtMinall, double MaxDt = 1, bool UseLocaldt = false,
                  void* stream = nullptr) {
    c_.check(dndsg_eval_dt(c_.get(), CFL, MaxDt, UseLocaldt ? 1 : 0, &dtMinall, stream));
    dt.resize(c_.nCells());
    c_.check(dndsg_get_dt(c_.get(), dt.data(), stream));
  }
  // rhs is overwritten, as in the reference
  void EvaluateRHS(std::vector<double>& rhs, double t, void* stream = nullptr) {
    rhs.resize(c_.nCells() * 4);
    c_.check(dndsg_eval_rhs(c_.get(), t, rhs.data(), stream));
  }
  // res[nVars] of the last EvaluateRHS
  void EvaluateResidual(std::vector<double>& res, int P = 1, bool volWise = false, void* stream = nullptr) {
    res.resize(4);
    c_.check(dndsg_residual(c_.get(), P, volWise ? 1 : 0, res.data(), stream));
  }

 private:
  Context& c_;
};

}  // namespace dndsg
