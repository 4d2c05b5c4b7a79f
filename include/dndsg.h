/*
 * dndsg.h -- C ABI of the B200 (sm_100a) implementation of the DNDS
 * residual-evaluation hot path: the variational-reconstruction (VR) Jacobi
 * sweep, the WBAP limiters (CWBAP and 3WBAP) and the face Gauss-point Riemann
 * flux with scatter to cells, the SSP-RK3 stage composition that drives them,
 * and the implicit path (EvaluateDt, LU-SGS, BDF / SDIRK4 dual time, GMRES).
 *
 * Every entry point returns 0 on success and a non-zero dndsg_status code on
 * failure; nothing throws or aborts.  dndsg_last_error() gives the message.
 * Arrays passed as host pointers are plain C arrays in the layouts stated
 * below; the state itself stays resident on the GPU inside the context.
 *
 * The reference exposes this path as C++ templates, not a plugin ABI; each
 * function below names the reference member function it replaces
 * (file:line inside the DNDS repository).
 */
#ifndef DNDSG_H
#define DNDSG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum dndsg_status {
  DNDSG_OK = 0,
  DNDSG_BAD_ARGUMENT = 1,
  DNDSG_CUDA_ERROR = 2,
  DNDSG_UNSUPPORTED = 3,
  DNDSG_NUMERIC_ERROR = 4, /* NaN / non-positive state seen by a kernel */
  DNDSG_SETUP_ERROR = 5,   /* degenerate mesh or singular VR matrix */
  DNDSG_TIMEOUT = 6        /* a bounded wait inside a kernel ran out: the kernel skipped its work,
                              and the context refuses every later call (destroy it) */
};

/* Mesh topology and geometry.  Replaces CompactFacedMeshSerialRW
 * (DNDS_Mesh.hpp:634-1906) as the input of the solver.
 *   node_xy    [n_nodes][2]
 *   cell_nodes [n_cells][4]  counter-clockwise, slot 3 = -1 for a triangle
 *   face_nodes [n_faces][2]  right-hand normal of node0->node1 points out of the left cell
 *   face_cells [n_faces][2]  (left, right), right = -1 on a boundary face
 *   face_bc    [n_faces]     BoundaryType (DNDS_Mesh.hpp:21-35): -1 inner, 1 Wall,
 *                            2 Farfield, 3 Wall_Euler, 4 Wall_NoSlip,
 *                            -4 Special_IVFar, -5 Special_2DRiemannFar
 *   face_shift [n_faces][2]  translation that brings the right cell next to a
 *                            periodic face (NULL: no periodic faces)
 * Indices are int32 (meshes up to 2^31-1 cells / faces). */
typedef struct {
  int64_t n_nodes, n_cells, n_faces;
  const double* node_xy;
  const int32_t* cell_nodes;
  const int32_t* face_nodes;
  const int32_t* face_cells;
  const int32_t* face_bc;
  const double* face_shift;
} dndsg_mesh_desc;

/* The subset of the reference's JSON settings the path reads:
 * VRFiniteVolume2D::Setting (DNDS_FV_VR.hpp:170-230) and
 * EulerEvaluator::Setting (DNDS_FV_EulerEvaluator.hpp:138-194). */
typedef struct {
  int32_t nvars;                 /* 4 = NS_2D */
  int32_t rec_order;             /* 2 = P2 (5 coefficients per variable) */
  int32_t riemann;               /* 1 Roe (Harten-Yee), 2 HLLC */
  int32_t sor_instead;           /* must be 0: the GPU sweep is a Jacobi sweep */
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
  int32_t limiter;               /* limiter in every stage: 0 none, 1 CWBAP (V3, limiterProcedure 1),
                                    2 3WBAP (V2, limiterProcedure 0) */
  double weight_len_scale;
  double wall_weight;
  double far_weight;
  double wbap_smooth_indicator_scale;
  double wbap_n_std;
  double gamma;
  double far_field[6];           /* farFieldStaticValue (conservative) */
  int32_t n_threads;             /* unused by the GPU path */
  int32_t precision;             /* 0 FP64 throughout, 1 FP32 bulk (FP64 means/norms) */
  /* idealGasProperty (DNDS_FV_EulerEvaluator.hpp:150-160): mu_gas = 0 is the
   * inviscid Euler model (the reference's Euler runs use 1e-200); mu_gas > 0
   * adds the Navier-Stokes viscous flux with Sutherland's law */
  double mu_gas;
  double cp_gas;                 /* Rgas * gamma / (gamma - 1) */
  double pr_gas;
  double t_ref;
  double c_sutherland;
} dndsg_settings;

typedef struct dndsg_ctx dndsg_ctx;

/* device buffers reachable through dndsg_device_buffer */
enum dndsg_buffer {
  DNDSG_BUF_U = 0,    /* double [n_cells][4] cell means (the flow part in SA contexts) */
  DNDSG_BUF_UREC = 1, /* double or float [n_cells][5][4] VR coefficients (flow part) */
  DNDSG_BUF_RHS = 2,  /* double [n_cells][4] */
  DNDSG_BUF_DT = 3,   /* double [n_cells] */
  DNDSG_BUF_SA_U = 4,   /* SA contexts: double [n_cells], the fifth variable's means */
  DNDSG_BUF_SA_UREC = 5 /* SA contexts: double or float [n_cells][5], its VR coefficients */
};

/* Build the context on CUDA device `device`: uploads the mesh and runs the
 * FP64 VR setup on the GPU.  Replaces ImplicitFiniteVolume2D's constructor
 * (DNDS_FV_VR.hpp:29-102), VRFiniteVolume2D::Initialization
 * (DNDS_FV_VR.cpp:3-13) and the EulerEvaluator constructor
 * (DNDS_FV_EulerEvaluator.hpp:196-365).  On failure *out may still hold a
 * context that carries the error message; destroy it. */
int dndsg_create(const dndsg_mesh_desc* mesh, const dndsg_settings* settings, int device, dndsg_ctx** out);
void dndsg_destroy(dndsg_ctx* ctx);
const char* dndsg_last_error(dndsg_ctx* ctx);
int64_t dndsg_n_cells(dndsg_ctx* ctx);
int64_t dndsg_n_faces(dndsg_ctx* ctx);

/* State transfer between host arrays and the resident device state.  `stream`
 * is a cudaStream_t (NULL = legacy default stream); the call returns after the
 * copy has completed.  u is [n_cells][nvars] (ArrayDOFV order); urec is
 * [n_cells][5][nvars] (coefficient-major per cell), in the context's basis. */
int dndsg_set_u(dndsg_ctx* ctx, const double* u, void* stream);
int dndsg_get_u(dndsg_ctx* ctx, double* u, void* stream);
int dndsg_set_urec(dndsg_ctx* ctx, const double* urec, void* stream);
int dndsg_get_urec(dndsg_ctx* ctx, double* urec, void* stream);
int dndsg_get_dt(dndsg_ctx* ctx, double* dt, void* stream);
int dndsg_device_buffer(dndsg_ctx* ctx, int which, void** ptr, int64_t* bytes);
int dndsg_get_time(dndsg_ctx* ctx, double* t, void* stream);
int dndsg_set_time(dndsg_ctx* ctx, double t, void* stream);

/* VRFiniteVolume2D::ReconstructionJacobiStep (DNDS_FV_VR.hpp:1474-1713):
 * nsweeps Jacobi sweeps on the resident u / urec.  If inc_out is not NULL it
 * receives sum ||urec_new - urec||^2 / n_cells of the last sweep (FP64). */
int dndsg_vr_jacobi_step(dndsg_ctx* ctx, int nsweeps, double* inc_out, void* stream);

/* VRFiniteVolume2D::ReconstructionWBAPLimitFacialV3 (DNDS_FV_VR.hpp:2053-2329):
 * CWBAP limiting of the resident urec in place.  indicator_out (nullable) gets
 * the smoothness indicator per cell [n_cells]. */
int dndsg_limiter_wbap(dndsg_ctx* ctx, int if_all, double* indicator_out, void* stream);

/* VRFiniteVolume2D::ReconstructionWBAPLimitFacialV2 (DNDS_FV_VR.hpp:1749-2047,
 * "3WBAP", limiterProcedure 0): the same indicator; then the P2 rows of every
 * listed cell, then its P1 rows against the neighbours' P2-limited
 * coefficients; biway WBAP with n = WBAP_nStd, multiway with n = 1 centred on
 * the first neighbour (faces in element-local order).  In place, as above.
 * The stage compositions run this one when settings.limiter = 2. */
int dndsg_limiter_wbap_v2(dndsg_ctx* ctx, int if_all, double* indicator_out, void* stream);

/* EulerEvaluator::EvaluateDt (DNDS_FV_EulerEvaluator.cpp:14-183): per-cell dt
 * into DNDSG_BUF_DT and the face spectral data used by the Roe entropy fix.
 * dt_min_out (nullable) receives the global minimum. */
int dndsg_eval_dt(dndsg_ctx* ctx, double cfl, double max_dt, int use_local_dt, double* dt_min_out, void* stream);

/* EulerEvaluator::EvaluateRHS (DNDS_FV_EulerEvaluator.cpp:198-640) on the
 * resident u / urec at time t, into DNDSG_BUF_RHS; rhs_out (nullable) gets a
 * host copy [n_cells][nvars]. */
int dndsg_eval_rhs(dndsg_ctx* ctx, double t, double* rhs_out, void* stream);

/* One explicit SSP-RK3 step: ExplicitSSPRK3LocalDt::Step (DNDS_ODE.hpp:131-177)
 * with the EulerSolver stage body frhs (DNDS_FV_EulerSolver.hpp:713-837):
 * EvaluateDt (global dt, clipped so that t does not pass t_end), then per
 * stage one VR Jacobi sweep, the limiter when enabled, EvaluateRHS and the
 * stage update.  In inviscid contexts EvaluateDt's face terms are written by
 * the first stage's face-flux launch (from the same means; the first sweep and
 * limiter do not depend on dt), and its cell pass runs before the first
 * update.  Time lives on the device and advances by the step's dt, so the
 * call is asynchronous and can be captured in a CUDA graph. */
int dndsg_ssprk3_step(dndsg_ctx* ctx, double cfl, double t_end, void* stream);

/* n calls of dndsg_ssprk3_step, with the same results: pairs of steps are
 * replayed from a CUDA graph captured on first use for this cfl / t_end (one
 * graph launch instead of 26 kernel launches, 28 with a viscous flux; small
 * meshes are launch-bound).
 * Same arguments as dndsg_ssprk3_step plus the step count n >= 0. */
int dndsg_ssprk3_steps(dndsg_ctx* ctx, double cfl, double t_end, int64_t n, void* stream);

/* EulerEvaluator::EvaluateResidual (DNDS_FV_EulerEvaluator.cpp:1557-1592) of
 * DNDSG_BUF_RHS: p < 3 gives the p-norm (volume-weighted when vol_wise), else
 * the max norm; out [nvars] (host), FP64. */
int dndsg_residual(dndsg_ctx* ctx, int p, int vol_wise, double* out, void* stream);

/* Diagnostic: reconstructed, positivity-compressed states at every face Gauss
 * point, out [n_faces][3][2][nvars] (side 1 of a boundary face = boundary
 * state), evaluated as in EvaluateRHS (DNDS_FV_EulerEvaluator.cpp:250-360). */
int dndsg_face_values(dndsg_ctx* ctx, double t, double* out, void* stream);

/* Allocation-free EvaluateRHS.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory when they need a residual -- a
 * real-time loop that cannot afford cudaMalloc's implicit device
 * synchronisation, a host framework that owns all device memory and forbids
 * allocations after start-up, or code running inside another library's
 * callback where allocating is not allowed.  It computes what dndsg_eval_rhs computes, but
 * from caller-owned device arrays -- u [n_cells][4] double, urec
 * [n_cells][5][4] in the context's precision (double, or float when
 * precision = 1), rhs [n_cells][4] double (output) -- and it allocates
 * nothing: its face-flux scratch is a fixed array inside the library of
 * DNDSG_NOALLOC_MAX_FACES faces (8 MiB per GPU, held until exit); larger
 * meshes are rejected with DNDSG_BAD_ARGUMENT.  The first call on a device
 * looks up the scratch address (cudaGetSymbolAddress), so make that first call
 * before any stream capture.  All calls share the one scratch array: calls
 * that overlap on the GPU (different streams or contexts at the same time)
 * race and must be serialised by the caller.  The Roe entropy fix uses the
 * face data of the context's last dndsg_eval_dt, as dndsg_eval_rhs does.
 * u, urec and rhs must be 16-byte aligned (the kernels move them in 16-byte
 * vectors; cudaMalloc'd arrays are); other pointers are rejected with
 * DNDSG_BAD_ARGUMENT before anything is launched. */
#define DNDSG_NOALLOC_MAX_FACES 262144
int dndsg_eval_rhs_noalloc(dndsg_ctx* ctx, const double* u, const void* urec, double* rhs, double t, void* stream);

/* Error flags raised by kernels since the last call (bit 0: NaN or
 * non-positive density/pressure in a flux; bit 1: reduced-order face point;
 * bit 2: a bounded wait inside a kernel ran out).  Bit 2 makes this call, and
 * every later call on the context, return DNDSG_TIMEOUT; so do the calls that
 * read results back from the device (dndsg_get_u, dndsg_get_time,
 * dndsg_implicit_iteration, dndsg_dual_step, dndsg_vr_to_tolerance,
 * dndsg_ssprk3_step_tol) when they see it. */
int dndsg_get_status(dndsg_ctx* ctx, uint32_t* flags, uint64_t* n_reduced, void* stream);

/* ---------------------------------------------------------------------------
 * Implicit steady path: LU-SGS and first-order BDF pseudo time.
 * The reference sweeps cells one at a time in a scan order
 * (UpdateLUSGSForward / Backward, DNDS_FV_EulerEvaluator.cpp:1149-1357).  By
 * default the cells get a greedy distance-1 colouring and each colour is one
 * parallel step; that is exactly the reference's sweep in the colour-sorted
 * scan order (a neighbour is "before" a cell when its colour is smaller).
 * dndsg_lusgs_set_order runs a given scan order (the reference's natural order
 * by default) as dependency levels, and dndsg_lusgs_set_parts that sweep as on
 * several ranks.  The diagonal is one scalar per cell, as in the reference
 * without source terms (the SA variable adds its source Jacobian).
 * ------------------------------------------------------------------------ */
/* the colouring: colour_out [n_cells] (host, may be NULL), n_colours */
int dndsg_lusgs_colours(dndsg_ctx* ctx, int32_t* colour_out, int* n_colours);
/* the sweep schedule.  mode 0 (default): colour batches, the reference's sweep
 * in the colour-sorted order (few batches; on meshes with strongly coupled
 * cell lines, such as stretched boundary-layer cells, it converges more slowly
 * than a line-following order).  mode 1: the reference's sequential sweep in
 * the scan order scan2cell [n_cells] (host; NULL = natural cell order, the
 * reference's SOR_iScan2iCell default), run as dependency levels (one batch
 * per level) so that it computes what the sequential sweep computes.
 * n_batches (may be NULL): forward plus backward batches per iteration (mode 1
 * with parts: the most levels of one part, forward plus backward). */
int dndsg_lusgs_set_order(dndsg_ctx* ctx, int mode, const int64_t* scan2cell, int* n_batches);
/* partitioned sweeps: the mode-1 sweep as the reference runs it on n_parts MPI
 * ranks (DNDS_FV_EulerEvaluator.cpp:1177-1181, 1313-1317; replaces the ranks'
 * UpdateLUSGSForward / pull / UpdateLUSGSBackward sequence).  Every part sweeps
 * its own cells in the scan order; a neighbour in another part is a ghost that
 * enters only the backward sweep, with its increment as it stood after the
 * forward sweep (the pull between the two).  part [n_cells] (host) in
 * [0, n_parts); NULL or n_parts == 1: one part.  Rebuilds the mode-1 schedule
 * with the scan order last given to dndsg_lusgs_set_order (natural order if
 * none) and switches to it; each sweep then runs the parts' level walks
 * concurrently, one thread block per part.  Parts apply to mode 1 only; a later
 * dndsg_lusgs_set_order(mode 1) keeps them.  DNDSG_UNSUPPORTED (nothing
 * changed) when a cell has more than 4 faces or a part more than 4095 levels.
 * n_batches (may be NULL): the most levels of one part, forward plus backward. */
int dndsg_lusgs_set_parts(dndsg_ctx* ctx, const int32_t* part, int n_parts, int* n_batches);
/* LUSGSMatrixInit (DNDS_FV_EulerEvaluator.cpp:995-1047): D_i = 1/dTau_i + 1/dt
 * + sum_f (alpha/2) lambda_f A_f / V_i with dTau = (the DNDSG_BUF_DT of the last
 * dndsg_eval_dt) / alpha, and lambda_f from that same call */
int dndsg_lusgs_matrix_init(dndsg_ctx* ctx, double dt_phys, double alpha, void* stream);
/* UpdateLUSGSForward / UpdateLUSGSBackward (DNDS_FV_EulerEvaluator.cpp:1149-1357)
 * in place on inc [n_cells][nvars] (device) with rhs [n_cells][nvars] (device),
 * about the context's u; forward expects inc zero where the reference does */
int dndsg_lusgs_forward(dndsg_ctx* ctx, double alpha, const double* rhs, double* inc, void* stream);
int dndsg_lusgs_backward(dndsg_ctx* ctx, double alpha, const double* rhs, double* inc, void* stream);
/* start of a physical BDF step: xLast = u */
int dndsg_bdf_begin(dndsg_ctx* ctx, void* stream);
/* one pseudo-time iteration of ImplicitBDFDualTimeStep::Step at order 1
 * (DNDS_ODE.hpp:444-486) with the EulerSolver fdtau / frhs / fsolve lambdas
 * (DNDS_FV_EulerSolver.hpp:713-925): local EvaluateDt at cfl, n_rec Jacobi
 * sweeps, [limiter], EvaluateRHS at t, rhs = alpha R - (u - xLast)/dt_phys,
 * LU-SGS forward + backward from zero, u += inc.  inc_res_out [nvars] (host,
 * may be NULL): the L1 norm of inc (volume-weighted when vol_wise), the
 * quantity the reference's fstop tests; wall_flux_out [nvars] (host, may be
 * NULL): fluxWallSum of this iteration's RHS. */
int dndsg_implicit_iteration(dndsg_ctx* ctx, double cfl, double dt_phys, double alpha, int n_rec, int vol_wise,
                             double t, double* inc_res_out, double* wall_flux_out, void* stream);

/* ---------------------------------------------------------------------------
 * Partitioned runs (the reference's MPI domain decomposition, one partition per
 * context): a context built on a partition's cells plus one layer of ghost cells
 * (every cell across a face of an owned cell; a ghost's faces to cells outside
 * the partition closed as far-field faces) computes the owned cells
 * exactly as the whole mesh would, given the ghosts' values after every VR
 * sweep (and limiter) and every stage update.  dndsg_set_owned marks the owned
 * cells (host [n_cells] 0/1; NULL: all owned): the dt minimum and
 * dndsg_residual run over owned cells only.  It first waits for all work on
 * the device (cudaDeviceSynchronize), so steps queued before it on any stream
 * see the old mask and steps after it the new one.  One SSP-RK3 step by stage
 * (ExplicitSSPRK3LocalDt::Step, DNDS_ODE.hpp:131-177):
 *   dndsg_rk_dt (local minimum; the caller reduces it over all partitions and
 *   clips it to the end time) -> dndsg_rk_set_dt -> 3 x [dndsg_rk_vr ->
 *   exchange urec -> dndsg_rk_limit -> exchange urec -> dndsg_rk_stage(k) ->
 *   exchange u] -> dndsg_rk_finish.
 * dndsg_halo_pack / unpack gather / scatter whole cells of u ([n][4] double) or
 * urec ([n][5][4] of the context's precision) at device cell indices, to or
 * from a device buffer (the caller moves buffers between partitions: a device
 * copy on one GPU, NCCL send / receive across GPUs).
 * ------------------------------------------------------------------------ */
#define DNDSG_HALO_U 0
#define DNDSG_HALO_UREC 1
int dndsg_set_owned(dndsg_ctx* ctx, const uint8_t* owned);
int dndsg_rk_dt(dndsg_ctx* ctx, double cfl, double* dt_min_out, void* stream);
int dndsg_rk_set_dt(dndsg_ctx* ctx, double dt, void* stream);
int dndsg_rk_vr(dndsg_ctx* ctx, void* stream);
int dndsg_rk_limit(dndsg_ctx* ctx, void* stream);
int dndsg_rk_stage(dndsg_ctx* ctx, int stage, void* stream);
int dndsg_rk_finish(dndsg_ctx* ctx, void* stream);
int dndsg_halo_pack(dndsg_ctx* ctx, int what, const int32_t* cells, int64_t n, void* buf, void* stream);
int dndsg_halo_unpack(dndsg_ctx* ctx, int what, const int32_t* cells, int64_t n, const void* buf, void* stream);

/* ---------------------------------------------------------------------------
 * Dual time stepping, the reference's implicit driver: one physical step of
 * ImplicitBDFDualTimeStep (order k; DNDS_ODE.hpp:392-497) or of the 3-stage
 * ImplicitSDIRK4DualTimeStep (DNDS_ODE.hpp:269-390), each internal iteration
 * being the EulerSolver's fdtau / frhs / fsolve / fstop
 * (DNDS_FV_EulerSolver.hpp:713-1061).  fsolve per gmres_code (gmresCode):
 * 0 the LU-SGS forward + backward sweeps; 1 GMRES_LeftPreconditioned
 * (DNDS_Linear.hpp:12-107) from a zero start, n_gmres_space Krylov vectors
 * (nGmresSpace) and n_gmres_iter restarts (nGmresIter), over LUSGSMatrixVec
 * with the LU-SGS sweeps as left preconditioner; 2 the sweeps, then GMRES from
 * their result.  fstop: the L1 norm of the increment (volume-weighted when
 * vol_wise) over its running maximum in the stage; an internal loop ends when
 * the density entry drops below threshold (rhsThresholdInternal) or after
 * max_iter (nTimeStepInternal) iterations.  The sweep order is the one of
 * dndsg_lusgs_set_order.  4-variable and SA contexts (SA: the U5 rhs and
 * increment pass through CompressInc as in fsolve).
 * ------------------------------------------------------------------------ */
#define DNDSG_DUAL_SDIRK4 0 /* odeCode 0 */
#define DNDSG_DUAL_BDF 1    /* odeCode 1 (the reference's driver uses bdf_order 2) */
typedef struct dndsg_dual_settings {
  int scheme;       /* DNDSG_DUAL_SDIRK4 or DNDSG_DUAL_BDF */
  int bdf_order;    /* 1..4 (BDF only) */
  double cfl;       /* CFL of the local pseudo time step */
  int max_iter;     /* nTimeStepInternal */
  double threshold; /* rhsThresholdInternal */
  int n_rec;        /* nInternalRecStep */
  int vol_wise;     /* useVolWiseResidual */
  int gmres_code;   /* 0, 1, 2 */
  int n_gmres_space;
  int n_gmres_iter;
} dndsg_dual_settings;
/* a fresh integrator: forgets the BDF history (also implied by a change of
 * bdf_order between calls) */
int dndsg_dual_reset(dndsg_ctx* ctx);
/* one physical step of size dt from time t, in place on the context's u;
 * iters_out [3] (host, may be NULL): internal iterations per stage (BDF: [0]);
 * res_out [nvars] (host, may be NULL): the last fstop ratios.  A BDF history built
 * with another dt is an error (the reference asserts a constant dt). */
int dndsg_dual_step(dndsg_ctx* ctx, const dndsg_dual_settings* settings, double dt, double t, int* iters_out,
                    double* res_out, void* stream);

/* Steady solve: the internal loop of one implicit step of the reference's
 * EulerSolver run with ifSteadyQuit (DNDS_FV_EulerSolver.hpp:609-615,
 * 713-1061; ImplicitBDFDualTimeStep::Step of order 1, DNDS_ODE.hpp:444-486)
 * until fstop: each iteration is fdtau (EvaluateDt at the current CFL, local
 * dt), frhs (n_rec VR sweeps, [limiter], EvaluateRHS), the first-order BDF
 * right-hand side with physical step dt (1e100: steady), fsolve per
 * gmres_code as in dndsg_dual_step, and u += inc.  fstop: the L1 increment
 * norm (volume-weighted when vol_wise) over its running maximum; the loop ends
 * when the density entry drops below threshold or after max_iter iterations.
 * The CFL ramp of fstop: between iterations cfl_ramp_start and
 * cfl_ramp_start + cfl_ramp_length the CFL moves log-linearly from cfl to
 * cfl_ramp_end and then stays there (nCFLRampStart, nCFLRampLength,
 * CFLRampEnd).  Outputs (host, each may be NULL): iters_out; res_out [nvars]
 * the last fstop ratios; wall_flux_out [nvars] fluxWallSum of the last
 * residual; history [max_iter] the density fstop ratio of every iteration. */
typedef struct dndsg_steady_settings {
  double cfl;          /* CFL */
  double cfl_ramp_end; /* CFLRampEnd */
  int cfl_ramp_start;  /* nCFLRampStart (a large value: no ramp) */
  int cfl_ramp_length; /* nCFLRampLength */
  int max_iter;        /* nTimeStepInternal */
  double threshold;    /* rhsThresholdInternal */
  double dt;           /* dtImplicit (1e100: steady) */
  int n_rec;           /* nInternalRecStep */
  int vol_wise;        /* useVolWiseResidual */
  int gmres_code;      /* 0, 1, 2 */
  int n_gmres_space;   /* nGmresSpace */
  int n_gmres_iter;    /* nGmresIter */
} dndsg_steady_settings;
int dndsg_steady_solve(dndsg_ctx* ctx, const dndsg_steady_settings* settings, int* iters_out, double* res_out,
                       double* wall_flux_out, double* history, void* stream);
/* GMRES_LeftPreconditioned::solve (DNDS_Linear.hpp:47-105) of LUSGSMatrixVec x = b,
 * the LU-SGS forward + backward sweeps as left preconditioner, n_space Krylov
 * vectors (1..32), n_restart restarts; x [n_cells][4] (device) holds the
 * initial guess and receives the result; b [n_cells][4] (device).  Uses the
 * diagonal and spectral radii of the last dndsg_lusgs_matrix_init. */
int dndsg_gmres_lusgs(dndsg_ctx* ctx, double alpha, int n_space, int n_restart, const double* b, double* x,
                      void* stream);
/* LUSGSMatrixVec (DNDS_FV_EulerEvaluator.cpp:1062-1143): ax = D x + sum over all
 * neighbours of (alpha/2) A_f / V_i dF(u_j; n, x_j), with D from the last
 * dndsg_lusgs_matrix_init; x, ax [n_cells][4] (device) */
int dndsg_lusgs_matvec(dndsg_ctx* ctx, double alpha, const double* x, double* ax, void* stream);

/* ---------------------------------------------------------------------------
 * Learned warm start for the VR coefficients.  No counterpart in the
 * reference: a per-cell network 64 -> 64 -> 64 -> 64 -> 20 (SiLU), BF16
 * weights and activations with FP32 accumulation on the tensor cores, trained
 * on pairs the solver itself produces.  From the starting coefficients x0 and
 * two plain Jacobi sweeps x1, x2 (ReconstructionJacobiStep,
 * DNDS_FV_VR.hpp:1474-1479) it proposes the converged coefficients.  Its output
 * is only a starting point: the plain sweep still iterates to the same
 * tolerance, and per cell the learned start is kept only where the Jacobi
 * increment from it is smaller than from x2.
 * Features per cell [DNDSG_MLP_IN] (float): neighbour mean differences (16)
 * divided per variable by their largest magnitude; the two sweep increments
 * x1 - x0 and x2 - x1 (20 + 20) divided per variable by r_v, the largest
 * |x1 - x0| of that variable; the slot face centres in the cell's own
 * polynomial frame (8).  Targets [20]: (converged - x2) / r_v.
 * ------------------------------------------------------------------------ */
#define DNDSG_MLP_IN 64
#define DNDSG_MLP_OUT 20
#define DNDSG_MLP_NPARAM 14560 /* FP32 parameters, W1[64][64] b1 W2[64][64] b2 W3[64][64] b3 W4[32][64] b4[32] */
typedef struct dndsg_mlp dndsg_mlp;

/* new network on a device: Glorot-uniform weights from seed, zero biases */
int dndsg_mlp_create(int device, uint64_t seed, dndsg_mlp** out);
void dndsg_mlp_destroy(dndsg_mlp* mlp);
const char* dndsg_mlp_last_error(dndsg_mlp* mlp);
/* host FP32 parameters [DNDSG_MLP_NPARAM] (padded rows/columns are zero);
 * set_params also resets the Adam moments */
int dndsg_mlp_set_params(dndsg_mlp* mlp, const float* params);
int dndsg_mlp_get_params(dndsg_mlp* mlp, float* params);
/* Y [n][20] = network(X [n][64]), device arrays.  Runs on the 5th-generation
 * tensor cores (tcgen05.mma, 128 rows per tile, FP32 accumulator in tensor
 * memory); returns when the forward is complete, DNDSG_CUDA_ERROR if a
 * tensor-core completion wait ran out (bounded wait) */
int dndsg_mlp_forward(dndsg_mlp* mlp, const float* X, int64_t n, float* Y, void* stream);
/* mean-square loss over n rows x 20 outputs against targets T [n][20] (device)
 * and its gradient (host [DNDSG_MLP_NPARAM], may be NULL); synchronous */
int dndsg_mlp_gradient(dndsg_mlp* mlp, const float* X, const float* T, int64_t n, double* loss, float* grad,
                       void* stream);
/* one Adam step (b1 0.9, b2 0.999, eps 1e-8) on the batch X, T (device);
 * loss (host, may be NULL) is the batch loss before the step */
int dndsg_mlp_train_step(dndsg_mlp* mlp, const float* X, const float* T, int64_t n, float lr, double* loss,
                         void* stream);
/* The warm start's input design, per context (for harvesting and use) and per
 * network (the design it is trained for; a mismatch is an error):
 *   0  Jacobi extrapolation (default): the neighbour mean differences, the
 *      increments of two plain sweeps from the start x0 and the slot geometry;
 *      output (x* - x2) / r, the learned start x2 + y r, gated against J(x2)
 *   1  the previous-step coefficients: the neighbour mean differences to up to
 *      4 neighbours and x0 itself (the coefficients the previous stage or step
 *      left), before any sweep; output (x* - x0) / s with s the per-variable
 *      mean-difference scale, the learned start x0 + y s gated against J(x0)
 *      (the two gate sweeps count), needs max_sweeps >= 2 */
int dndsg_mlp_set_features(dndsg_mlp* mlp, int mode);
int dndsg_set_warm_start_features(dndsg_ctx* ctx, int mode);
/* features of the context's current coefficients, X [n_cells][64], and the
 * output scales r [n_cells][4] (device); design 0 runs two sweeps into work
 * buffers; the context's coefficients are left unchanged */
int dndsg_mlp_features(dndsg_ctx* ctx, float* X, float* scales, void* stream);
/* Jacobi sweeps on the context's coefficients until the rms increment
 * sqrt(sum |dx|^2 / n_cells) <= tol or max_sweeps.  With mlp (may be NULL;
 * design 0 needs max_sweeps >= 4): sweeps x0 -> x1 -> x2, the learned start
 * xm, then J(x2) and J(xm) gated per cell (accepted_out: cells that kept the
 * learned start); the four count as sweeps (design 1: see above).  harvest_x
 * [n_cells][64], harvest_t [n_cells][20] (device, may be NULL; only without
 * mlp) receive the features and the training targets of the context's
 * design. */
int dndsg_vr_to_tolerance(dndsg_ctx* ctx, const dndsg_mlp* mlp, double tol, int max_sweeps, int* sweeps_out,
                          int64_t* accepted_out, float* harvest_x, float* harvest_t, void* stream);
/* dndsg_ssprk3_step with the reconstruction of every stage iterated to tol
 * (above); harvest arrays, when given, hold 3 stages back to back */
int dndsg_ssprk3_step_tol(dndsg_ctx* ctx, const dndsg_mlp* mlp, double cfl, double t_end, double tol,
                          int max_sweeps, int* sweeps_out, float* harvest_x, float* harvest_t, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DNDSG_H */
