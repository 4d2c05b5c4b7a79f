// dndsg_shim.hpp -- header-only C++ shim over the dndsg C ABI with the call
// surface of the DNDS classes it replaces on the GPU:
//
//   VRFiniteVolume2DGPU::ReconstructionJacobiStep      VRFiniteVolume2D, DNDS_FV_VR.hpp:1474-1479
//   VRFiniteVolume2DGPU::ReconstructionWBAPLimitFacialV3  DNDS_FV_VR.hpp:2055-2061
//   VRFiniteVolume2DGPU::ReconstructionWBAPLimitFacialV2  DNDS_FV_VR.hpp:1751-1757
//   EulerEvaluatorGPU::EvaluateDt                       EulerEvaluator, DNDS_FV_EulerEvaluator.hpp:1408-1411
//   EulerEvaluatorGPU::EvaluateRHS                      DNDS_FV_EulerEvaluator.hpp:1412-1418
//   EulerEvaluatorGPU::EvaluateResidual                 DNDS_FV_EulerEvaluator.hpp:1455-1461
//   EulerEvaluatorGPU::LUSGSMatrixInit                  DNDS_FV_EulerEvaluator.cpp:995-1047
//   EulerEvaluatorGPU::UpdateLUSGSForward / Backward    DNDS_FV_EulerEvaluator.cpp:1149-1357
//   ImplicitSteadyGPU::Step                             ImplicitBDFDualTimeStep::Step (order 1) with the
//                                                       EulerSolver lambdas, DNDS_ODE.hpp:444-486 and
//                                                       DNDS_FV_EulerSolver.hpp:713-994
//   ImplicitSteadyGPU::Run                              the same internal loop in one call, with the fstop
//                                                       CFL ramp and fsolve per gmresCode (:984-1061)
//   ImplicitDualTimeStepGPU::Step                       ImplicitSDIRK4DualTimeStep / ImplicitBDFDualTimeStep
//                                                       ::Step, DNDS_ODE.hpp:269-497, with the EulerSolver
//                                                       lambdas (odeCode, gmresCode), :594-1226
//   EulerEvaluatorGPU::LUSGSMatrixVec                   DNDS_FV_EulerEvaluator.cpp:1062-1143
//   GMRES_LeftPreconditionedGPU::solve                  GMRES_LeftPreconditioned, DNDS_Linear.hpp:47-105
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
  // 3WBAP limiting (limiterProcedure 0) in place
  void ReconstructionWBAPLimitFacialV2(bool ifAll, std::vector<double>* ifUseLimiter = nullptr, void* stream = nullptr) {
    if (ifUseLimiter) ifUseLimiter->resize(c_.nCells());
    c_.check(dndsg_limiter_wbap_v2(c_.get(), ifAll ? 1 : 0, ifUseLimiter ? ifUseLimiter->data() : nullptr, stream));
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
  // the diagonal from the dTau of the last EvaluateDt (called with UseLocaldt) divided by alphaDiag
  void LUSGSMatrixInit(double dt, double alphaDiag, void* stream = nullptr) {
    c_.check(dndsg_lusgs_matrix_init(c_.get(), dt, alphaDiag, stream));
  }
  // rhs / uInc are device arrays [nCells][nVars]; uInc is updated in place (uInc == uIncNew in the reference)
  void UpdateLUSGSForward(double alphaDiag, const double* rhs, double* uInc, void* stream = nullptr) {
    c_.check(dndsg_lusgs_forward(c_.get(), alphaDiag, rhs, uInc, stream));
  }
  void UpdateLUSGSBackward(double alphaDiag, const double* rhs, double* uInc, void* stream = nullptr) {
    c_.check(dndsg_lusgs_backward(c_.get(), alphaDiag, rhs, uInc, stream));
  }
  void LUSGSMatrixVec(double alphaDiag, const double* x, double* Ax, void* stream = nullptr) {
    c_.check(dndsg_lusgs_matvec(c_.get(), alphaDiag, x, Ax, stream));
  }
  // sweep order: mode 0 colour batches, 1 the sequential order scan2cell (nullptr: natural), level-scheduled
  int SetLUSGSOrder(int mode, const int64_t* scan2cell = nullptr) {
    int nb = 0;
    c_.check(dndsg_lusgs_set_order(c_.get(), mode, scan2cell, &nb));
    return nb;
  }
  // the mode-1 sweep partitioned as on nParts ranks (part of every cell; nullptr: one part)
  int SetLUSGSParts(const int32_t* part, int nParts) {
    int nb = 0;
    c_.check(dndsg_lusgs_set_parts(c_.get(), part, nParts, &nb));
    return nb;
  }

 private:
  Context& c_;
};

// the explicit driver: ExplicitSSPRK3LocalDt::Step with the frhs body (DNDS_ODE.hpp:131-177,
// DNDS_FV_EulerSolver.hpp:713-837), one step or n of them (pairs replayed from a CUDA graph)
class ExplicitSSPRK3GPU {
 public:
  explicit ExplicitSSPRK3GPU(Context& c) : c_(c) {}
  void Step(double CFL, double tEnd = 1e300, void* stream = nullptr) {
    c_.check(dndsg_ssprk3_step(c_.get(), CFL, tEnd, stream));
  }
  void Steps(double CFL, int64_t n, double tEnd = 1e300, void* stream = nullptr) {
    c_.check(dndsg_ssprk3_steps(c_.get(), CFL, tEnd, n, stream));
  }

 private:
  Context& c_;
};

// the steady path: pseudo-time iterations of a first-order BDF step until the density increment,
// relative to its largest value so far, drops below rhsThresholdInternal (fstop)
class ImplicitSteadyGPU {
 public:
  explicit ImplicitSteadyGPU(Context& c) : c_(c) {}
  // returns the iterations taken; wallFlux (may be null) receives fluxWallSum of the last iteration
  int Step(double CFL, double rhsThresholdInternal, int nTimeStepInternal, double dtImplicit = 1e100,
           int nInternalRecStep = 1, bool useVolWiseResidual = false, std::vector<double>* wallFlux = nullptr,
           void* stream = nullptr) {
    c_.check(dndsg_bdf_begin(c_.get(), stream));
    double base = 0, res[4], wf[4];
    int iter = 1;
    for (; iter <= nTimeStepInternal; iter++) {
      c_.check(dndsg_implicit_iteration(c_.get(), CFL, dtImplicit, 1.0, nInternalRecStep, useVolWiseResidual ? 1 : 0,
                                        0.0, res, wf, stream));
      base = iter == 1 ? res[0] : (res[0] > base ? res[0] : base);
      if (res[0] < rhsThresholdInternal * base) break;
    }
    if (wallFlux) wallFlux->assign(wf, wf + 4);
    return iter > nTimeStepInternal ? nTimeStepInternal : iter;
  }
  // the whole steady internal loop in one call (dndsg_steady_solve); returns the iterations taken
  int Run(const dndsg_steady_settings& settings, std::vector<double>* wallFlux = nullptr,
          std::vector<double>* history = nullptr, void* stream = nullptr) {
    int it = 0;
    double res[5], wf[5];
    if (history) history->assign(settings.max_iter, 0.0);
    c_.check(dndsg_steady_solve(c_.get(), &settings, &it, res, wf, history ? history->data() : nullptr, stream));
    if (wallFlux) wallFlux->assign(wf, wf + 4);
    if (history) history->resize(it);
    return it;
  }

 private:
  Context& c_;
};

// the reference's implicit driver: one physical step of SDIRK4 (odeCode 0) or BDF of order k
// (odeCode 1) in dual time, fsolve by LU-SGS / GMRES per gmresCode; the ODE object's history (BDF)
// lives in the context, Reset() where the reference's solver would construct a new ODE object
class ImplicitDualTimeStepGPU {
 public:
  ImplicitDualTimeStepGPU(Context& c, int odeCode, int bdfOrder = 2) : c_(c) {
    d_.scheme = odeCode == 0 ? DNDSG_DUAL_SDIRK4 : DNDSG_DUAL_BDF;
    d_.bdf_order = bdfOrder;
    c_.check(dndsg_dual_reset(c_.get()));
  }
  // returns the internal iterations of the last stage
  int Step(double dt, double tSimu, double CFL, int nTimeStepInternal, double rhsThresholdInternal,
           int nInternalRecStep = 1, bool useVolWiseResidual = false, int gmresCode = 0, int nGmresSpace = 10,
           int nGmresIter = 2, void* stream = nullptr) {
    d_.cfl = CFL;
    d_.max_iter = nTimeStepInternal;
    d_.threshold = rhsThresholdInternal;
    d_.n_rec = nInternalRecStep;
    d_.vol_wise = useVolWiseResidual ? 1 : 0;
    d_.gmres_code = gmresCode;
    d_.n_gmres_space = nGmresSpace;
    d_.n_gmres_iter = nGmresIter;
    int its[3] = {0, 0, 0};
    double res[5];
    c_.check(dndsg_dual_step(c_.get(), &d_, dt, tSimu, its, res, stream));
    return d_.scheme == DNDSG_DUAL_SDIRK4 ? its[2] : its[0];
  }
  void Reset() { c_.check(dndsg_dual_reset(c_.get())); }

 private:
  Context& c_;
  dndsg_dual_settings d_{};
};

// GMRES over LUSGSMatrixVec with the LU-SGS sweeps as left preconditioner (the EulerSolver's
// FA / FML pair), on device arrays; x holds the initial guess and receives the result
class GMRES_LeftPreconditionedGPU {
 public:
  GMRES_LeftPreconditionedGPU(Context& c, int kSubspace) : c_(c), k_(kSubspace) {}
  void solve(double alphaDiag, const double* b, double* x, int nRestart, void* stream = nullptr) {
    c_.check(dndsg_gmres_lusgs(c_.get(), alphaDiag, k_, nRestart, b, x, stream));
  }

 private:
  Context& c_;
  int k_;
};

}  // namespace dndsg
