/*
 * dnds_oracle.h -- FP64 CPU restatement of the DNDS residual-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs
 * may load it; the product (dnds_b200, libdndsg) never does.
 *
 * It restates, function by function, the reference's algorithms:
 *   - VRFiniteVolume2D setup        DNDS_FV_VR.cpp:22-1154, DNDS_FV_VR.hpp:300-1293
 *   - ReconstructionJacobiStep      DNDS_FV_VR.hpp:1474-1713
 *   - ReconstructionWBAPLimitFacialV3  DNDS_FV_VR.hpp:2053-2329, DNDS_FV_Limiters.hpp:341-449
 *   - EulerEvaluator::EvaluateDt    DNDS_FV_EulerEvaluator.cpp:14-183
 *   - EulerEvaluator::EvaluateRHS   DNDS_FV_EulerEvaluator.cpp:198-640
 *   - Roe / HLLC fluxes             DNDS_Gas.hpp:312-654
 *   - ExplicitSSPRK3LocalDt::Step   DNDS_ODE.hpp:131-177
 *   - LU-SGS (LUSGSMatrixInit, UpdateLUSGSForward/Backward,
 *     fluxJacobian0_Right_Times_du)  DNDS_FV_EulerEvaluator.cpp:995-1357,
 *                                   DNDS_FV_EulerEvaluator.hpp:928-956
 *   - ImplicitBDFDualTimeStep::Step DNDS_ODE.hpp:392-497 (orders 1-4)
 *   - ImplicitSDIRK4DualTimeStep    DNDS_ODE.hpp:269-390
 *   - GMRES_LeftPreconditioned      DNDS_Linear.hpp:12-107, over
 *     LUSGSMatrixVec                DNDS_FV_EulerEvaluator.cpp:1062-1143
 *   - EvaluateResidual              DNDS_FV_EulerEvaluator.cpp:1557-1592
 * Deviations (documented where they occur): no Eigen (the 5x5 inverse is a
 * pivoted Gauss-Jordan instead of JacobiSVD; A_ii is SPD so both give A^-1),
 * a closed-form 2x2 eigen-frame instead of Eigen::computeDirect (the VR
 * polynomial does not depend on the basis orientation), periodic faces
 * (absent from the reference), and SSP-RK3 stage times 0, 1, 1/2 for
 * time-dependent boundary data.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Unstructured 2-D mesh of straight-sided triangles / quadrilaterals.
 * cell_nodes: 4 per cell, counter-clockwise, -1 in slot 3 for triangles.
 * face_nodes: 2 per face, ordered so that the right-hand normal points out of
 *             face_cells[2f] (the left cell).
 * face_cells: left, right (-1 on a boundary face).
 * face_bc:    DNDS BoundaryType code (-1 inner, 1 Wall, 2 Farfield, 3 Wall_Euler,
 *             4 Wall_NoSlip, -4 Special_IVFar, -5 Special_2DRiemannFar).
 * face_shift: per face (dx, dy) that moves the right cell next to the face
 *             (periodic faces); may be NULL. */
typedef struct {
  int64_t n_nodes, n_cells, n_faces;
  const double* node_xy;
  const int32_t* cell_nodes;
  const int32_t* face_nodes;
  const int32_t* face_cells;
  const int32_t* face_bc;
  const double* face_shift;
} orc_mesh;

/* Same field order and meaning as dndsg_settings in include/dndsg.h. */
typedef struct {
  int32_t nvars;              /* 4: NS_2D */
  int32_t rec_order;          /* 2 (P2) */
  int32_t riemann;            /* 1 Roe, 2 HLLC */
  int32_t sor_instead;        /* oracle only: 1 = in-place Gauss-Seidel sweep */
  double jacobi_relax;
  double tang_weight;
  double tang_weight_mod_min;
  double tang_weight_mod_power;
  int32_t tang_weight_mod_loc;
  int32_t tang_weight_direction; /* 0 Norm, 1 Bary */
  int32_t base_center_type;      /* 0 Bary, 1 Param */
  int32_t use_local_coord;
  int32_t anisotropic_lengths;
  int32_t weight_scheme_geom;    /* 0 None, 1 D, 2 S, 3 SDHQM */
  int32_t weight_scheme_dir;     /* 0 None, 1 optHQM */
  int32_t limiter;               /* 0 none, 1 CWBAP (V3, limiterProcedure 1), 2 3WBAP (V2, limiterProcedure 0) */
  double weight_len_scale;
  double wall_weight;
  double far_weight;
  double wbap_smooth_indicator_scale;
  double wbap_n_std;
  double gamma;
  double far_field[6];
  int32_t n_threads;             /* 0 = hardware concurrency */
  int32_t pad0;
  /* idealGasProperty (DNDS_FV_EulerEvaluator.hpp:150-160): mu_gas = 0 is the
   * inviscid Euler model (the reference's Euler runs use 1e-200); mu_gas > 0
   * adds the Navier-Stokes viscous flux with Sutherland's law */
  double mu_gas;
  double cp_gas;                 /* Rgas * gamma / (gamma - 1) */
  double pr_gas;
  double t_ref;
  double c_sutherland;
} orc_settings;

typedef struct orc_ctx orc_ctx;

int orc_create(const orc_mesh* mesh, const orc_settings* s, orc_ctx** out);
void orc_destroy(orc_ctx* c);
const char* orc_last_error(orc_ctx* c);

/* state I/O: u is [n_cells][nvars], urec is [n_cells][5][nvars] */
int orc_set_u(orc_ctx* c, const double* u);
int orc_get_u(orc_ctx* c, double* u);
int orc_set_urec(orc_ctx* c, const double* urec);
int orc_get_urec(orc_ctx* c, double* urec);
int orc_get_geometry(orc_ctx* c, double* vol, double* bary /*[n][2]*/, double* face_area);

/* isentropic-vortex cell averages (DNDS_FV_EulerSolver.hpp:536-582) */
int orc_init_isentropic_vortex(orc_ctx* c);
/* cell-average of the exact advected vortex at time t, into out [n][nvars] */
int orc_exact_isentropic_vortex(orc_ctx* c, double t, double* out);
/* piecewise-constant states by cell barycentre: 4 quadrant states split at (xs, ys):
 * q[0]=NE (x>xs,y>ys), q[1]=NW, q[2]=SW, q[3]=SE; each (rho,u,v,p) */
int orc_init_quadrants(orc_ctx* c, double xs, double ys, const double* q);

/* one ReconstructionJacobiStep per sweep, on the internal u / urec */
int orc_vr_step(orc_ctx* c, int nsweeps);
/* increment norm: sum over cells of ||uRecNew-uRec||^2 / N for the last sweep */
double orc_vr_last_increment(orc_ctx* c);
/* ReconstructionWBAPLimitFacialV3 on the internal urec (in place) */
int orc_limiter_wbap(orc_ctx* c, int if_all, double* indicator_out /*[n] or NULL*/);
/* ReconstructionWBAPLimitFacialV2 (3WBAP, limiterProcedure 0), in place on urec */
int orc_limiter_wbap_v2(orc_ctx* c, int if_all, double* indicator_out /*[n] or NULL*/);
/* EvaluateDt */
int orc_eval_dt(orc_ctx* c, double cfl, double max_dt, int use_local_dt, double* dt_out, double* dt_min);
/* EvaluateRHS on the internal u/urec; rhs_out [n][nvars]; wall_flux [nvars] may be NULL */
int orc_eval_rhs(orc_ctx* c, double t, double* rhs_out, double* wall_flux);
/* reconstructed and positivity-compressed values at every face Gauss point:
 * out[f][g][side][nvars], side 1 of a boundary face holds the boundary state */
int orc_face_values(orc_ctx* c, double t, double* out);
/* one SSP-RK3 step (fdt + 3 stages of VR sweep, limiter, RHS) of size dt */
int orc_ssprk3_step(orc_ctx* c, double dt, double t);
/* EvaluateResidual */
int orc_residual(orc_ctx* c, const double* rhs, int p, int vol_wise, double* out);

/* LUSGSMatrixInit (DNDS_FV_EulerEvaluator.cpp:995-1047): dtau [n] (NULL: the
 * dt of the last orc_eval_dt divided by alpha), physical dt, alphaDiag */
int orc_lusgs_matrix_init(orc_ctx* c, const double* dtau, double dt, double alpha);
/* UpdateLUSGSForward / Backward (DNDS_FV_EulerEvaluator.cpp:1149-1357) in place
 * on inc [n][nvars]; scan2cell [n] is the sweep order (NULL: natural order) */
int orc_lusgs_forward(orc_ctx* c, double alpha, const double* rhs, double* inc, const int64_t* scan2cell);
int orc_lusgs_backward(orc_ctx* c, double alpha, const double* rhs, double* inc, const int64_t* scan2cell);
/* partitioned sweeps, the reference run on several ranks: part [n] of every cell (NULL: one part);
 * a neighbour in another part enters only the backward sweep, with its post-forward increment */
int orc_set_lusgs_parts(orc_ctx* c, const int32_t* part);
/* one BDF pseudo-time iteration (ImplicitBDFDualTimeStep::Step, DNDS_ODE.hpp:444-486,
 * first order) with the EulerSolver fdtau/frhs/fsolve lambdas; x_last [n][nvars]
 * is the state at the start of the physical step; inc_out [n][nvars] may be NULL */
int orc_implicit_iteration(orc_ctx* c, double cfl, double dt, double alpha, const double* x_last,
                           const int64_t* scan2cell, double t, int n_rec, double* inc_out);

/* LUSGSMatrixVec (DNDS_FV_EulerEvaluator.cpp:1062-1143) with the diagonal of the
 * last orc_lusgs_matrix_init; x, ax [n][nvars] */
int orc_lusgs_matvec(orc_ctx* c, double alpha, const double* x, double* ax);
/* GMRES_LeftPreconditioned::solve (DNDS_Linear.hpp:47-105) of LUSGSMatrixVec x = b
 * with the LU-SGS sweeps as left preconditioner, x [n][nvars] in place (initial guess) */
int orc_gmres_lusgs(orc_ctx* c, double alpha, int n_space, int n_restart, const double* b, double* x,
                    const int64_t* scan2cell);
/* dual time stepping: ImplicitBDFDualTimeStep (scheme 1, order 1..4) or
 * ImplicitSDIRK4DualTimeStep (scheme 0), DNDS_ODE.hpp:269-497, with fsolve by
 * LU-SGS (gmres_code 0), GMRES_LeftPreconditioned (1, DNDS_Linear.hpp:12-107)
 * or both (2) */
typedef struct orc_dual_settings {
  int scheme, bdf_order;
  double cfl;
  int max_iter;
  double threshold;
  int n_rec, vol_wise, gmres_code, n_gmres_space, n_gmres_iter;
} orc_dual_settings;
int orc_dual_reset(orc_ctx* c);
/* one physical step of size dt from t on the internal u; iters_out [3], res_out [nvars] may be NULL */
int orc_dual_step(orc_ctx* c, const orc_dual_settings* d, double dt, double t, const int64_t* scan2cell,
                  int* iters_out, double* res_out);

/* setup products, for cross-checks: [n][5][5], [n][4][5][5], [n][4][5] */
int orc_get_vr_blocks(orc_ctx* c, double* ainv, double* ainvb, double* ainv_b);
/* basis values/derivatives at a face gauss point: [f][g][side][6][6] */
int orc_get_face_dibj(orc_ctx* c, double* out);

/* Roe / HLLC flux in the face-normal x direction (DNDS_Gas.hpp) for 2-D, 4 vars */
void orc_riemann_flux(int riemann, const double* ul, const double* ur, double gamma,
                      double dlambda, double* f);

#ifdef __cplusplus
}
#endif
