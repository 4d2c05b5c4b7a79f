// dndsg.cu -- context, kernels and C ABI of the B200 DNDS hot path.
//
// Build: nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -shared
// (see dnds_b200/build.py).  One thread per cell / face around the bodies of
// dndsg_bodies.cuh; block-level reductions use warp shuffles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/dndsg.h"
#include "dndsg_bodies.cuh"
#include "dndsg_limiter.cuh"
#include "dndsg_async.cuh"
#include "dndsg_mlp.cuh"
#include "dndsg_sa.cuh"

using namespace dg;

namespace {
constexpr int kBlock = 256;
inline unsigned grid_for(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// device scalar slots
enum { S_T = 0, S_DT = 1, S_DTMIN = 2, S_TEVAL = 3, S_ZERO = 4, S_INC = 5, S_NSLOT = 8 };
}  // namespace

struct dndsg_ctx {
  int device = 0;
  dndsg_settings s{};
  int64_t N = 0, F = 0;
  int64_t Fi = 0;                // faces [0, Fi) are interior, [Fi, F) boundary (internal order)
  std::vector<int64_t> facePerm; // internal face id -> caller's face id
  int nfmax = 3;
  bool fp32 = false;
  bool hasWallCorr = false;
  std::string err;
  // mesh / geometry
  int32_t *faceL = nullptr, *faceR = nullptr, *faceBC = nullptr;
  double *vol = nullptr, *closure = nullptr, *faceNormal = nullptr, *faceArea = nullptr, *faceCenter = nullptr,
         *faceW0 = nullptr;
  int32_t *cellFace = nullptr, *vrNbr = nullptr, *vrMode = nullptr, *vrFace = nullptr;
  void* vrOp = nullptr;       // T
  void* faceBasis = nullptr;  // T
  void* faceGrad = nullptr;   // T, viscous contexts only
  // SA contexts (nvars 5): the fifth variable in its own arrays
  bool sa = false;
  double* saDmat = nullptr;  // the U5 LU-SGS diagonal itself (GMRES matrix-vector product)
  double *saU = nullptr, *saULast = nullptr, *saRhs = nullptr, *saFlux = nullptr, *saInc = nullptr, *saDinv = nullptr,
         *saSrcJac = nullptr, *saDWall = nullptr, *saCellGp = nullptr;
  void *saUrec = nullptr, *saUrecNew = nullptr;  // T [N][5]
  double* Ainv = nullptr;
  void* limFace = nullptr;                                 // T: the limiting pass's per-face matrices
  void* faceInd = nullptr;                                  // the indicator's face integrals (precision T)
  double* indicator = nullptr;                              // the indicator's values
  int32_t *limList = nullptr, *limCount = nullptr;  // cells the limiter pass limits, and their number
  void *limG = nullptr, *limCell = nullptr;         // the indicator's compact face and cell data (T)
  int sms = 0;                                      // multiprocessors of the device
  // dndsg_ssprk3_steps: CUDA graphs of two SSP-RK3 steps, one per coefficient buffer holding urec at
  // the start (a step swaps the buffers three times), for the cfl / t_end they were captured with
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    double cfl = 0, tEnd = 0;
    void* urec = nullptr;
  } stepGraph[2];
  cudaStream_t capStream = nullptr;
  int32_t* wallCells = nullptr;  // cells with a Wall_Euler / Wall_NoSlip face
  float* mlpGeom = nullptr;  // [N][8] slot face centres in each cell's polynomial frame
  void *mlpM = nullptr, *mlpA = nullptr, *mlpB = nullptr, *mlpH = nullptr;  // learned warm start work (T)
  float* mlpSc = nullptr;                                                     // [N][4] output scales
  int mlpFeatureMode = 0;  // warm-start features: 0 Jacobi extrapolation, 1 previous coefficients
  unsigned long long* accCount = nullptr;
  int64_t nWallCells = 0;
  // implicit path: the sweep order as a rank per cell (a neighbour of lower rank is "before"),
  // the forward / backward schedules (batches of independent cells), LU-SGS diagonal,
  // increment, residual accumulator
  int32_t *rankOf = nullptr, *fwdCells = nullptr, *bwdCells = nullptr;
  std::vector<int64_t> fwdOff, bwdOff;
  int64_t *fwdOffDev = nullptr, *bwdOffDev = nullptr;  // level offsets on the device (scan-order mode)
  int32_t *fwdNbF = nullptr, *fwdNbJ = nullptr, *bwdNbF = nullptr, *bwdNbJ = nullptr;  // [pos][4] records
  void* lusgsMat = nullptr;  // per-position neighbour-matrix records of one sweep (scan-order mode)
  int32_t *fwdNbP = nullptr, *bwdNbP = nullptr;  // [pos][4] neighbour schedule positions (-1: not in the ring)
  int64_t maxLevelWidth = 0;
  std::vector<int32_t> colourHost;  // greedy colouring, kept for dndsg_lusgs_colours
  int lusgsOrder = 0;               // 0 colour batches, 1 level-scheduled scan order
  // partitioned scan-order sweeps (the reference on several ranks): the part of every cell (empty:
  // one part), and per sweep the index of every part's first level in fwdOff / bwdOff ([parts + 1],
  // device) with the most levels of one part
  std::vector<int32_t> lusgsPart;
  int lusgsParts = 1;
  int32_t *fwdPartLev = nullptr, *bwdPartLev = nullptr;
  int fwdPartMax = 0, bwdPartMax = 0;
  std::vector<int64_t> scanHost;  // the scan order last set (empty: natural cell order)
  double *Dinv = nullptr, *inc = nullptr, *resAcc = nullptr;
  double* Dmat = nullptr;  // the LU-SGS diagonal itself (GMRES matrix-vector product)
  // dual time stepping: BDF history (earlier steps' states) or the SDIRK stage right-hand sides,
  // the GMRES Krylov basis, Hessenberg matrix and reduction scratch
  std::vector<double*> odeVec, gmV;
  int odeOrder = 0, odeCnPrev = 0, odePrevStart = 0;
  double odeDtPrev = 0.0;
  double *gmTmp = nullptr, *gmMLb = nullptr, *gmH = nullptr, *gmPartial = nullptr, *gmB = nullptr, *gmX = nullptr;
  // state
  double *u = nullptr, *uLast = nullptr, *rhs = nullptr, *dt = nullptr, *flux = nullptr, *lamA = nullptr,
         *dLam = nullptr, *scal = nullptr, *partial = nullptr;
  void *urec = nullptr, *urecNew = nullptr;  // T
  unsigned* flags = nullptr;
  unsigned long long* nreduced = nullptr;
  bool dead = false;  // a kernel's bounded wait ran out: the context refuses further work
  uint8_t* owned = nullptr;  // [N] owned-cell mask of a partitioned run (null: every cell owned)
  uint8_t* ownedBuf = nullptr;
  std::vector<void*> allocs;

  size_t tsize() const { return fp32 ? sizeof(float) : sizeof(double); }
};

namespace {

int fail(dndsg_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
#define DG_CUDA(ctx, call)                                                                          \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return fail(ctx, DNDSG_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

template <class P>
int dalloc(dndsg_ctx* c, P*& p, size_t bytes) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes > 0 ? bytes : 16);
  if (e != cudaSuccess) return fail(c, DNDSG_CUDA_ERROR, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  c->allocs.push_back(q);
  p = (P*)q;
  return 0;
}

// ------------------------------------------------------------------ warp/block reductions
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// the sum of v over a block of kBlock threads (all of them call this) added to *acc by one thread:
// one atomic per block instead of one per warp (many warps adding to one address serialise in L2)
__device__ __forceinline__ void block_add(double v, double* acc) {
  __shared__ double part[kBlock / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kBlock / 32 ? part[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0 && t != 0.0) atomicAdd(acc, t);
  }
  __syncthreads();  // part is reused by the next call
}

// ------------------------------------------------------------------ setup kernels
__global__ void k_setup_cell(MeshView m, SetupParams p, CellSetup* cells, double* vol, double* bary, int* bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m.N) return;
  CellSetup c;
  if (!setup_cell(i, m, p, c)) atomicOr(bad, 1);
  cells[i] = c;
  vol[i] = c.vol;
  bary[2 * i] = c.bary[0];
  bary[2 * i + 1] = c.bary[1];
}

template <class T>
__global__ void k_setup_face(MeshView m, SetupParams p, const CellSetup* cells, double* faceW, double* normal,
                             double* area, double* center, double* w0, T* basis) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f >= m.F) return;
  setup_face<T>(f, m, p, cells, faceW, normal, area, center, w0, basis);
}

__global__ void k_setup_sa_cells(int64_t N, const CellSetup* cells, const double* seg, int64_t nw, double* gp,
                                 double* dWall) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  setup_sa_cell_gp(i, cells, gp);
  dWall[i] = sa_wall_distance(cells[i].bary[0], cells[i].bary[1], seg, nw);
}

template <class T>
__global__ void k_setup_face_grad(MeshView m, const CellSetup* cells, T* grad) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f < m.F) setup_face_grad<T>(f, m, cells, grad);
}

template <class T>
__global__ void k_setup_matrices(MeshView m, SetupParams p, const CellSetup* cells, const double* faceW,
                                 const int32_t* cellFace, int nfmax, T* vrOp, int32_t* vrNbr, int32_t* vrMode,
                                 int32_t* vrFace, double* Ainv, int* bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m.N) return;
  if (!setup_cell_matrices<T>(i, m, p, cells, faceW, cellFace, nfmax, vrOp, nullptr, vrNbr, vrMode, vrFace, Ainv))
    atomicOr(bad, 2);
}

// slot face centres in the cell's polynomial frame, the geometric inputs of the learned warm start
__global__ void k_setup_mlp_geom(MeshView m, const CellSetup* cells, const int32_t* cellFace, int nfmax,
                                 const double* faceCenter, float* geom) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m.N) return;
  const CellFrame& fr = cells[i].fr;
  for (int k = 0; k < 4; k++) {
    double g0 = 0, g1 = 0;
    if (k < nfmax) {
      int32_t sf = cellFace[aos(i, k, nfmax)];
      if (sf != kEmptySlot) {
        const int64_t f = sf >= 0 ? sf : ~sf;
        double x = faceCenter[2 * f], y = faceCenter[2 * f + 1];
        if (sf < 0 && m.face_shift) { x -= m.face_shift[2 * f]; y -= m.face_shift[2 * f + 1]; }
        const double dx = x - fr.c[0], dy = y - fr.c[1];
        g0 = fr.Pinv[0][0] * dx + fr.Pinv[0][1] * dy;
        g1 = fr.Pinv[1][0] * dx + fr.Pinv[1][1] * dy;
      }
    }
    geom[i * 8 + 2 * k] = (float)g0;
    geom[i * 8 + 2 * k + 1] = (float)g1;
  }
}

// ------------------------------------------------------------------ hot kernels
template <class T, bool RELAX1, bool INC>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? 2 : 1) k_vr(HotView<T> h, double* incAcc) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double d2 = 0;
  if (i < h.N) {
    vr_cell<T, RELAX1>(i, h);
    if (INC) {
      for (int k = 0; k < 20; k++) {
        double d = (double)h.urecNew[i * 20 + k] - (double)h.urec[i * 20 + k];
        d2 += d * d;
      }
    }
  }
  if (INC) {
    d2 = warp_sum(d2);
    if ((threadIdx.x & 31) == 0 && d2 != 0.0) atomicAdd(incAcc, d2);
  }
}

// VR operator of the CTA's tile in shared memory, same AoSoA order as in global memory
template <class T>
struct VrOpSmem {
  const T* p;  // &tile[(sub * E) * 32 + lane]
  __device__ __forceinline__ T operator()(int k, int e) const { return p[(k * 30 + e) * 32]; }
};

// cells per CTA of the VR sweep: one 32-cell AoSoA block (the smallest contiguous operator tile).
// Small tiles keep many CTAs resident per SM, so tile loads and gathers of different CTAs overlap
// (measured on 2,097,152 triangles, FP32: 128 cells 0.233 ms = 77% of HBM peak, 64: 0.226, 32:
// 0.212 = 85%; FP64: 64 cells 0.367 ms, 32: 0.358)
template <class T>
constexpr int vr_tile() { return 32; }

// VR Jacobi sweep, 4 threads per cell (one per conserved variable).  One
// elected thread bulk-copies the CTA's TILE-cell operator tile (contiguous in the
// AoSoA layout) into shared memory on an mbarrier; meanwhile every thread issues
// its neighbour gathers; then the 4 threads of a cell read the same shared words
// (broadcast) and keep only 5 accumulators each.
template <class T, int TILE, int NF>
__global__ void __launch_bounds__(TILE * 4) k_vr_tma4(HotView<T> h, unsigned* flags) {
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) unsigned long long bar;
  constexpr int E = NF * 30;
  const int tid = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * TILE;
  constexpr uint32_t bytes = (uint32_t)(TILE * E * sizeof(T));
  const uint32_t b = smem_u32(&bar);
  if (tid == 0) {
    mbar_init(b, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(b, bytes);
    bulk_g2s(smem_u32(dsm), h.vrOp + c0 * E, bytes, b);
  }
  const int cl = tid >> 2, v = tid & 3;
  const int64_t i = c0 + cl;
  VrPre<T, NF> pre;
  if (i < h.N) vr_var_prefetch<T, NF>(i, v, h, pre);
  const bool ok = mbar_wait(b, 0, kWaitLimit);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicOr(flags, kFlagTimeout);
      mbar_wait(b, 0, kWaitLimit);
    }
    return;
  }
  if (i < h.N) {
    const T* sm = reinterpret_cast<const T*>(dsm);
    vr_var_compute<T, NF>(i, v, h, pre, VrOpSmem<T>{sm + (cl >> 5) * E * 32 + (cl & 31)});
  }
}

template <class T>
__global__ void k_vr_wall_fixup(HotView<T> h, const int32_t* cells, int64_t n) {  // 4 threads per wall cell
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < 4 * n) vr_wall_fixup<T>(cells[k >> 2], (int)(k & 3), h);
}
// ---- CWBAP limiter: face indicator integrals, cell indicator, limiting pass
template <class T>
__global__ void k_setup_limiter(MeshView m, SetupParams p, const CellSetup* cells, const double* faceW, T* lim,
                                int* bad) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f < m.F && !setup_limiter_face(f, m, p, cells, faceW, lim)) atomicOr(bad, 4);
}
template <class T>
__global__ void k_setup_lim_compact(MeshView m, const CellSetup* cells, const double* faceW, T* g, T* cellFr) {
  const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  setup_limiter_compact<T>(f, m, cells, faceW, g, cellFr);
}
// FP64: 2 blocks per SM.  FP32: 4 blocks per SM (64 registers; the pass waits on its gathers, and the
// fourth block took the 8,388,608-triangle Riemann step from 8.61 to 8.44 ms against three)
template <class T>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? 4 : 2) k_lim_face(LimView v, const T* urec, int32_t* count) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f == 0) *count = 0;  // the list of cells to limit, filled by the next launch
  if (f < v.F) limiter_face_indicator<T>(f, v, urec);
}
// the indicator of every cell; a cell with si >= scale (or every cell, ifAll) is appended to the
// list (order of the list is immaterial: each cell's result depends on the unlimited data only)
template <class T>
__global__ void __launch_bounds__(kBlock) k_lim_cell_indicator(LimView v, int32_t* list, int32_t* count) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool lim = false;
  if (i < v.N) {
    const double ind = limiter_cell_indicator<T>(i, v);
    v.indicator[i] = ind;
    lim = !(ind < v.scale) || v.ifAll;
  }
  const unsigned b = __ballot_sync(0xffffffffu, lim);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && b) base = atomicAdd(count, __popc(b));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (lim) list[base + __popc(b & ((1u << lane) - 1))] = (int32_t)i;
}
// the limiting pass over the listed cells, four lanes per cell (limiter_cell4), into buf[t] for list
// entry t: V3 = true both orders of ReconstructionWBAPLimitFacialV3; V3 = false the order PASS of
// ReconstructionWBAPLimitFacialV2.  A grid-stride loop whose trip count is the same for all lanes of a
// warp (eight cells per warp per trip), so the width-4 shuffles always have all 32 lanes
template <class T, bool V3, int PASS, int NF>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? 4 : 2) k_lim_apply4(LimView v, const T* urec, T* buf, const int32_t* list,
                                                       const int32_t* count) {
  const int64_t n = *count;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp * 8; base < n; base += nwarps * 8) {
    const int64_t t = base + (lane >> 2);
    const bool valid = t < n;
    const int64_t i = valid ? list[t] : 0;
    limiter_cell4<T, V3, PASS, NF>(valid, i, lane & 3, v, urec, buf + (valid ? t : 0) * 20);
  }
}
// the limited coefficients back over the listed cells' ones, 16 bytes per thread
template <class T>
__global__ void __launch_bounds__(kBlock) k_lim_scatter(T* urec, const T* buf, const int32_t* list,
                                                        const int32_t* count) {
  constexpr int W = 16 / sizeof(T), V = 20 / W;  // elements per vector, vectors per cell
  const int64_t n = (int64_t)*count * V;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = e / V, k = e - t * V;
    reinterpret_cast<int4*>(urec + (int64_t)list[t] * 20)[k] = reinterpret_cast<const int4*>(buf + t * 20)[k];
  }
}

__device__ __forceinline__ double stage_time(const double* scal, int useDev, double tHost, double c) {
  return useDev ? (c == 0.0 ? scal[S_T] : scal[S_T] + c * scal[S_DT]) : tHost;
}

// faces [f0, f1): interior faces first (BND = false), then boundary faces.  The FP32 Roe interior
// kernel runs 4 blocks per SM (64 registers, a few spilled words): the gathers want the occupancy
// more than the registers (measured: 2 blocks 0.296 ms, 3: 0.283, 4: 0.243, 5: 0.318 per RHS on
// 2,097,152 triangles).  The FP32 HLLC interior kernel (flux-difference form) runs 3 (measured per
// SSP-RK3 step of the 8,388,608-triangle Riemann problem: 3 blocks 7.79-7.81 ms, 4 blocks with 64
// registers and 172 B spilled 8.02-8.04 ms)
// DT = true (the first stage of an SSP-RK3 step): each thread first writes its face's EvaluateDt terms
// (dt_face: lambda A and the entropy-fix dLambda, from the same means this stage reads), which the
// flux then reads back, so the step needs no separate face pass for dt
template <class T, int RIEMANN, bool BND, bool DT = false>
__global__ void __launch_bounds__(kBlock, (sizeof(T) == 4 && RIEMANN == 1 && !BND) ? 4 : ((sizeof(T) == 4 && !BND) ? 3 : 2)) k_face_flux(HotView<T> h, int64_t f0, int64_t f1, const double* scal,
                                                         int useDev, double tHost, double c, unsigned* flags,
                                                         unsigned long long* nred) {
  int64_t f = f0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int r = 0;
  bool bad = false;
  if (f < f1) {
    if constexpr (DT) dt_face<T>(f, h);
    double out[4];
    double t = stage_time(scal, useDev, tHost, c);
    if constexpr (sizeof(T) == 4 && RIEMANN == 1 && !BND)
      r = face_flux_roe_delta32(f, h, out, bad);
    else if constexpr (sizeof(T) == 4 && RIEMANN == 2 && !BND)
      r = face_flux_hllc_delta32(f, h, out, bad);
    else
      r = face_flux<T, RIEMANN, BND>(f, h, t, out, bad);
    double* o = &h.flux[f * 4];
    *reinterpret_cast<double2*>(o) = make_double2(out[0], out[1]);
    *reinterpret_cast<double2*>(o + 2) = make_double2(out[2], out[3]);
  }
  unsigned anyBad = __ballot_sync(0xffffffffu, bad);
  int rs = __reduce_add_sync(0xffffffffu, r);
  if ((threadIdx.x & 31) == 0) {
    if (anyBad) atomicOr(flags, 1u);
    if (rs) atomicAdd(nred, (unsigned long long)rs);
  }
}

// the same with the Navier-Stokes viscous term (contexts with mu_gas > 0)
template <class T, int RIEMANN, bool BND>
__global__ void __launch_bounds__(kBlock) k_face_flux_vis(HotView<T> h, int64_t f0, int64_t f1, const double* scal,
                                                          int useDev, double tHost, double c, unsigned* flags,
                                                          unsigned long long* nred) {
  int64_t f = f0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int r = 0;
  bool bad = false;
  if (f < f1) {
    double out[4];
    r = face_flux_vis<T, RIEMANN, BND>(f, h, stage_time(scal, useDev, tHost, c), out, bad);
    double* o = &h.flux[f * 4];
    *reinterpret_cast<double2*>(o) = make_double2(out[0], out[1]);
    *reinterpret_cast<double2*>(o + 2) = make_double2(out[2], out[3]);
  }
  unsigned anyBad = __ballot_sync(0xffffffffu, bad);
  int rs = __reduce_add_sync(0xffffffffu, r);
  if ((threadIdx.x & 31) == 0) {
    if (anyBad) atomicOr(flags, 1u);
    if (rs) atomicAdd(nred, (unsigned long long)rs);
  }
}

template <class T>
__global__ void k_face_values(HotView<T> h, double t, double* out) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f >= h.F) return;
  double UL[3][4], UR[3][4], nx, ny, area;
  face_states(f, h, t, UL, UR, nx, ny, area);
  for (int g = 0; g < 3; g++)
    for (int v = 0; v < 4; v++) {
      out[((f * 3 + g) * 2 + 0) * 4 + v] = UL[g][v];
      out[((f * 3 + g) * 2 + 1) * 4 + v] = UR[g][v];
    }
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_dt_face(HotView<T> h) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f < h.F) dt_face<T>(f, h);
}

__global__ void k_init_dtmin(double* scal) {
  unsigned long long inf = 0x7ff0000000000000ull;
  reinterpret_cast<unsigned long long*>(scal)[S_DTMIN] = inf;
  scal[S_INC] = 0.0;
}

// per-cell dt, global min, and (for a step) the copy u -> uLast
template <class T, bool COPY_LAST>
__global__ void __launch_bounds__(kBlock) k_dt_cell(HotView<T> h, double cfl, double maxDt, double* scal) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double d = 1e300;
  if (i < h.N) {
    d = dt_cell<T>(i, h, cfl, maxDt);
    h.dt[i] = d;
    if (h.owned && !h.owned[i]) d = 1e300;  // a ghost cell's faces are incomplete: not in the minimum
    if (COPY_LAST) {
      const double2* s = reinterpret_cast<const double2*>(&h.u[i * 4]);
      double2* o = reinterpret_cast<double2*>(&h.uLast[i * 4]);
      o[0] = s[0];
      o[1] = s[1];
    }
  }
  d = warp_min(d);
  __shared__ double sm[kBlock / 32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kBlock / 32 ? sm[threadIdx.x] : 1e300;
    v = warp_min(v);
    if (threadIdx.x == 0 && v >= 0)
      atomicMin(reinterpret_cast<unsigned long long*>(scal) + S_DTMIN, (unsigned long long)__double_as_longlong(v));
  }
}

// step dt = min(dt_min, t_end - t)
__global__ void k_dt_finalize(double* scal, double tEnd) {
  double dmin = __longlong_as_double((long long)reinterpret_cast<unsigned long long*>(scal)[S_DTMIN]);
  double rem = tEnd - scal[S_T];
  scal[S_DT] = fmax(0.0, fmin(dmin, rem));
}
__global__ void k_advance_time(double* scal) { scal[S_T] += scal[S_DT]; }

__global__ void k_fill_dt(double* dt, int64_t n, const double* scal) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dt[i] = __longlong_as_double((long long)reinterpret_cast<const unsigned long long*>(scal)[S_DTMIN]);
}

// rhs gather + (optionally) SSP-RK3 stage update (ExplicitSSPRK3LocalDt::Step, DNDS_ODE.hpp:140-163)
template <class T, int STAGE>
__global__ void __launch_bounds__(kBlock) k_cell_update(HotView<T> h, const double* scal) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= h.N) return;
  double r[4];
  cell_rhs<T>(i, h, r);
  if (STAGE < 0) {
    double2* o = reinterpret_cast<double2*>(&h.rhs[i * 4]);
    o[0] = make_double2(r[0], r[1]);
    o[1] = make_double2(r[2], r[3]);
    return;
  }
  const double dt = scal[S_DT];
  double x[4];
  load4<T>(&h.u[i * 4], x);
  for (int v = 0; v < 4; v++) x[v] += r[v] * dt;
  if (STAGE > 0) {
    const double cf = STAGE == 1 ? 0.25 : 2.0 / 3.0;
    double xl[4];
    load4<T>(&h.uLast[i * 4], xl);
    for (int v = 0; v < 4; v++) {
      double a = x[v] * (cf / (1 - cf));
      a += xl[v];
      x[v] = a * (1 - cf);
    }
  }
  double2* o = reinterpret_cast<double2*>(&h.u[i * 4]);
  o[0] = make_double2(x[0], x[1]);
  o[1] = make_double2(x[2], x[3]);
}

// per-block partial sums / maxima of |rhs|^p (EvaluateResidual)
__global__ void k_residual(const double* rhs, const double* vol, int64_t n, int p, int volWise, double* partial,
                           const uint8_t* owned) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double a[4] = {0, 0, 0, 0};
  if (i < n && (!owned || owned[i]))
    for (int v = 0; v < 4; v++) {
      double x = fabs(rhs[i * 4 + v]);
      if (p < 3) {
        x = p == 1 ? x : (p == 2 ? x * x : pow(x, (double)p));
        if (volWise) x *= vol[i];
      }
      a[v] = x;
    }
  __shared__ double sm[4][kBlock / 32];
  for (int v = 0; v < 4; v++) {
    double w = p < 3 ? warp_sum(a[v]) : warp_max(a[v]);
    if ((threadIdx.x & 31) == 0) sm[v][threadIdx.x >> 5] = w;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double acc = 0;
    for (int k = 0; k < kBlock / 32; k++) acc = p < 3 ? acc + sm[threadIdx.x][k] : fmax(acc, sm[threadIdx.x][k]);
    partial[blockIdx.x * 4 + threadIdx.x] = acc;
  }
}

template <class T>
__global__ void k_cvt_to(const double* src, T* dst, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (T)src[i];
}
template <class T>
__global__ void k_cvt_from(const T* src, double* dst, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}

template <class T>
HotView<T> view(dndsg_ctx* c) {
  HotView<T> h;
  h.N = c->N; h.F = c->F; h.nfmax = c->nfmax;
  h.vol = c->vol; h.closure = c->closure; h.cellFace = c->cellFace;
  h.vrOp = (const T*)c->vrOp; h.vrNbr = c->vrNbr; h.vrMode = c->vrMode; h.vrFace = c->vrFace; h.Ainv = c->Ainv;
  h.faceL = c->faceL; h.faceR = c->faceR; h.faceBC = c->faceBC;
  h.faceBasis = (const T*)c->faceBasis; h.faceNormal = c->faceNormal; h.faceArea = c->faceArea;
  h.faceCenter = c->faceCenter; h.faceW0 = c->faceW0;
  h.u = c->u; h.uLast = c->uLast; h.rhs = c->rhs; h.dt = c->dt;
  h.urec = (const T*)c->urec; h.urecNew = (T*)c->urecNew;
  h.flux = c->flux; h.lamA = c->lamA; h.dLam = c->dLam; h.owned = c->owned;
  h.gamma = c->s.gamma;
  for (int k = 0; k < 4; k++) h.farU[k] = c->s.far_field[k];
  h.relax = c->s.jacobi_relax;
  h.faceGrad = (const T*)c->faceGrad;
  h.mu = c->s.mu_gas; h.cp = c->s.cp_gas; h.pr = c->s.pr_gas; h.tRef = c->s.t_ref; h.cSuth = c->s.c_sutherland;
  return h;
}

template <class T>
SaView<T> sa_view(dndsg_ctx* c) {
  SaView<T> v;
  v.u = c->saU; v.uLast = c->saULast; v.urec = (const T*)c->saUrec; v.urecNew = (T*)c->saUrecNew;
  v.rhs = c->saRhs; v.flux = c->saFlux; v.inc = c->saInc; v.Dinv = c->saDinv; v.srcJac = c->saSrcJac;
  v.dWall = c->saDWall; v.cellGp = c->saCellGp; v.far5 = c->s.far_field[4];
  return v;
}

inline cudaStream_t st(void* s) { return (cudaStream_t)s; }

// ------------------------------------------------------------------ hot-path drivers (templated on T)
template <class T>
int run_vr(dndsg_ctx* c, bool inc, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  bool r1 = c->s.jacobi_relax == 1.0;
  if (inc) {
    if (r1) k_vr<T, true, true><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal + S_INC);
    else k_vr<T, false, true><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal + S_INC);
  } else if (r1) {
    constexpr int TILE = vr_tile<T>();
    const size_t smem = (size_t)TILE * c->nfmax * 30 * sizeof(T);
    if (c->nfmax == 3)
      k_vr_tma4<T, TILE, 3><<<(unsigned)((c->N + TILE - 1) / TILE), TILE * 4, smem, s>>>(h, c->flags);
    else
      k_vr_tma4<T, TILE, 4><<<(unsigned)((c->N + TILE - 1) / TILE), TILE * 4, smem, s>>>(h, c->flags);
    if (c->nWallCells > 0) k_vr_wall_fixup<T><<<grid_for(4 * c->nWallCells), kBlock, 0, s>>>(h, c->wallCells, c->nWallCells);
  } else {
    k_vr<T, false, false><<<grid_for(c->N), kBlock, 0, s>>>(h, nullptr);
  }
  std::swap(c->urec, c->urecNew);
  return 0;
}

LimView lim_view(dndsg_ctx* c, int ifAll) {
  LimView v;
  v.N = c->N; v.F = c->F; v.Fi = c->Fi; v.nfmax = c->nfmax;
  v.cellFace = c->cellFace; v.faceL = c->faceL; v.faceR = c->faceR;
  v.faceNormal = c->faceNormal; v.faceArea = c->faceArea; v.limFace = c->limFace; v.limG = c->limG; v.limCell = c->limCell;
  v.u = c->u; v.faceInd = c->faceInd; v.indicator = c->indicator;
  v.gamma = c->s.gamma; v.tangWeight = c->s.tang_weight; v.tangModMin = c->s.tang_weight_mod_min;
  v.tangModPower = c->s.tang_weight_mod_power; v.tangModLoc = c->s.tang_weight_mod_loc; v.vol = c->vol;
  v.porder2 = (double)(c->s.rec_order * c->s.rec_order);
  v.scale = c->s.wbap_smooth_indicator_scale; v.nStd = c->s.wbap_n_std; v.ifAll = ifAll;
  return v;
}

// ReconstructionWBAPLimitFacialV3 on the resident urec (result swapped into urec)
template <class T>
void run_limiter_v3(dndsg_ctx* c, int ifAll, cudaStream_t s) {
  LimView v = lim_view(c, ifAll);
  k_lim_face<T><<<grid_for(c->F), kBlock, 0, s>>>(v, (const T*)c->urec, c->limCount);
  k_lim_cell_indicator<T><<<grid_for(c->N), kBlock, 0, s>>>(v, c->limList, c->limCount);
  // urecNew (the previous sweep's coefficients, free until the next sweep) holds the limited ones
  if (!c->sms && cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) c->sms = 148;
  const unsigned g = (unsigned)std::min<int64_t>(grid_for(c->N), 4 * c->sms);
  if (c->nfmax == 3) k_lim_apply4<T, true, 0, 3><<<g, kBlock, 0, s>>>(v, (const T*)c->urec, (T*)c->urecNew, c->limList, c->limCount);
  else k_lim_apply4<T, true, 0, 4><<<g, kBlock, 0, s>>>(v, (const T*)c->urec, (T*)c->urecNew, c->limList, c->limCount);
  k_lim_scatter<T><<<g, kBlock, 0, s>>>((T*)c->urec, (const T*)c->urecNew, c->limList, c->limCount);
}

// ReconstructionWBAPLimitFacialV2 on the resident urec: the same indicator and list, then the P2 pass
// over the listed cells scattered back before the P1 pass reads it, as the reference's order loop
// copies uRecNewBuf1 into uRecNewBuf between the orders
template <class T>
void run_limiter_v2(dndsg_ctx* c, int ifAll, cudaStream_t s) {
  LimView v = lim_view(c, ifAll);
  k_lim_face<T><<<grid_for(c->F), kBlock, 0, s>>>(v, (const T*)c->urec, c->limCount);
  k_lim_cell_indicator<T><<<grid_for(c->N), kBlock, 0, s>>>(v, c->limList, c->limCount);
  if (!c->sms && cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) c->sms = 148;
  const unsigned g = (unsigned)std::min<int64_t>(grid_for(c->N), 4 * c->sms);
  if (c->nfmax == 3) k_lim_apply4<T, false, 0, 3><<<g, kBlock, 0, s>>>(v, (const T*)c->urec, (T*)c->urecNew, c->limList, c->limCount);
  else k_lim_apply4<T, false, 0, 4><<<g, kBlock, 0, s>>>(v, (const T*)c->urec, (T*)c->urecNew, c->limList, c->limCount);
  k_lim_scatter<T><<<g, kBlock, 0, s>>>((T*)c->urec, (const T*)c->urecNew, c->limList, c->limCount);
  if (c->nfmax == 3) k_lim_apply4<T, false, 1, 3><<<g, kBlock, 0, s>>>(v, (const T*)c->urec, (T*)c->urecNew, c->limList, c->limCount);
  else k_lim_apply4<T, false, 1, 4><<<g, kBlock, 0, s>>>(v, (const T*)c->urec, (T*)c->urecNew, c->limList, c->limCount);
  k_lim_scatter<T><<<g, kBlock, 0, s>>>((T*)c->urec, (const T*)c->urecNew, c->limList, c->limCount);
}

// the limiter of the stage compositions: limiterProcedure 1 (CWBAP, V3) or 0 (3WBAP, V2)
template <class T>
void run_limiter(dndsg_ctx* c, int ifAll, cudaStream_t s) {
  if (c->s.limiter == 2) run_limiter_v2<T>(c, ifAll, s);
  else run_limiter_v3<T>(c, ifAll, s);
}

// the inviscid face-flux launches (interior faces, then boundary faces); DT: with the faces' dt terms
template <class T, bool DT>
void launch_flux_inviscid(dndsg_ctx* c, const HotView<T>& h, int useDev, double tHost, double cst, cudaStream_t s) {
  const int64_t Fi = c->Fi, F = c->F;
  if (c->s.riemann == 2) {
    if (Fi > 0)
      k_face_flux<T, 2, false, DT><<<grid_for(Fi), kBlock, 0, s>>>(h, 0, Fi, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
    if (F > Fi)
      k_face_flux<T, 2, true, DT><<<grid_for(F - Fi), kBlock, 0, s>>>(h, Fi, F, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
  } else {
    if (Fi > 0)
      k_face_flux<T, 1, false, DT><<<grid_for(Fi), kBlock, 0, s>>>(h, 0, Fi, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
    if (F > Fi)
      k_face_flux<T, 1, true, DT><<<grid_for(F - Fi), kBlock, 0, s>>>(h, Fi, F, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
  }
}

// the face-flux launches of EvaluateRHS over the arrays of h (interior faces, then boundary faces).
// dt = true (inviscid contexts only, the caller checks): the launches also write the faces' EvaluateDt
// terms (k_face_flux with DT)
template <class T>
void launch_flux_h(dndsg_ctx* c, const HotView<T>& h, int useDev, double tHost, double cst, cudaStream_t s,
                   bool dt = false) {
  const int64_t Fi = c->Fi, F = c->F;
  if (c->s.mu_gas > 0) {
    if (c->s.riemann == 2) {
      if (Fi > 0)
        k_face_flux_vis<T, 2, false><<<grid_for(Fi), kBlock, 0, s>>>(h, 0, Fi, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
      if (F > Fi)
        k_face_flux_vis<T, 2, true><<<grid_for(F - Fi), kBlock, 0, s>>>(h, Fi, F, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
    } else {
      if (Fi > 0)
        k_face_flux_vis<T, 1, false><<<grid_for(Fi), kBlock, 0, s>>>(h, 0, Fi, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
      if (F > Fi)
        k_face_flux_vis<T, 1, true><<<grid_for(F - Fi), kBlock, 0, s>>>(h, Fi, F, c->scal, useDev, tHost, cst, c->flags, c->nreduced);
    }
    return;
  }
  if (dt) {
    launch_flux_inviscid<T, true>(c, h, useDev, tHost, cst, s);
    return;
  }
  launch_flux_inviscid<T, false>(c, h, useDev, tHost, cst, s);
}

template <class T>
void launch_flux(dndsg_ctx* c, int useDev, double tHost, double cst, cudaStream_t s, bool dt = false) {
  launch_flux_h<T>(c, view<T>(c), useDev, tHost, cst, s, dt);
}

template <class T>
int run_dt(dndsg_ctx* c, double cfl, double maxDt, bool copyLast, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  k_init_dtmin<<<1, 1, 0, s>>>(c->scal);
  k_dt_face<T><<<grid_for(c->F), kBlock, 0, s>>>(h);
  if (copyLast) k_dt_cell<T, true><<<grid_for(c->N), kBlock, 0, s>>>(h, cfl, maxDt, c->scal);
  else k_dt_cell<T, false><<<grid_for(c->N), kBlock, 0, s>>>(h, cfl, maxDt, c->scal);
  return 0;
}

// one SSP-RK3 step.  Inviscid contexts take EvaluateDt's face terms from the first stage's face-flux
// launches (the same means, the same dt_face arithmetic): the VR sweep and the limiter of stage 1 do
// not depend on dt, so dt_cell and the minimum follow the first face pass and precede the first update.
// Viscous contexts (whose dt_face adds the viscous term) run the dt pass first.
template <class T>
int run_step(dndsg_ctx* c, double cfl, double tEnd, cudaStream_t s) {
  const bool fuseDt = !(c->s.mu_gas > 0);
  if (fuseDt) {
    k_init_dtmin<<<1, 1, 0, s>>>(c->scal);
  } else {
    run_dt<T>(c, cfl, 1e100, true, s);
    k_dt_finalize<<<1, 1, 0, s>>>(c->scal, tEnd);
  }
  const double cst[3] = {0.0, 1.0, 0.5};
  for (int stg = 0; stg < 3; stg++) {
    run_vr<T>(c, false, s);
    if (c->s.limiter) run_limiter<T>(c, 0, s);
    HotView<T> h = view<T>(c);
    if (stg == 0 && fuseDt) {
      launch_flux<T>(c, 1, 0.0, cst[stg], s, true);
      k_dt_cell<T, true><<<grid_for(c->N), kBlock, 0, s>>>(h, cfl, 1e100, c->scal);
      k_dt_finalize<<<1, 1, 0, s>>>(c->scal, tEnd);
    } else {
      launch_flux<T>(c, 1, 0.0, cst[stg], s);
    }
    if (stg == 0) k_cell_update<T, 0><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
    else if (stg == 1) k_cell_update<T, 1><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
    else k_cell_update<T, 2><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
  }
  k_advance_time<<<1, 1, 0, s>>>(c->scal);
  return 0;
}

// stage k of SSP-RK3 after its VR sweep (and limiter): the face fluxes and the stage update
template <class T>
void run_rk_stage(dndsg_ctx* c, int stg, cudaStream_t s) {
  const double cst[3] = {0.0, 1.0, 0.5};
  launch_flux<T>(c, 1, 0.0, cst[stg], s);
  HotView<T> h = view<T>(c);
  if (stg == 0) k_cell_update<T, 0><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
  else if (stg == 1) k_cell_update<T, 1><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
  else k_cell_update<T, 2><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
}

// halo exchange buffers: PACK buf[k][0..w) = a[cells[k]][0..w), else the reverse
template <class T, bool PACK>
__global__ void k_halo_copy(T* a, const int32_t* cells, int64_t n, int w, T* buf) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n * w) return;
  const int64_t k = e / w, v = e - k * w;
  const int64_t i = cells[k];
  if (PACK) buf[e] = a[i * w + v];
  else a[i * w + v] = buf[e];
}

template <class T>
int run_rhs(dndsg_ctx* c, double t, cudaStream_t s) {
  launch_flux<T>(c, 0, t, 0.0, s);
  HotView<T> h = view<T>(c);
  k_cell_update<T, -1><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
  return 0;
}

int check_launch(dndsg_ctx* c) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, DNDSG_CUDA_ERROR, std::string("kernel launch: ") + cudaGetErrorString(e));
  return 0;
}

int set_device(dndsg_ctx* c) {
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail(c, DNDSG_CUDA_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return 0;
}

// A bounded wait inside a kernel that ran out (kFlagTimeout: an mbarrier phase of a bulk copy or of a
// tensor-core commit, or a level-walk handshake, not complete within its poll limit) leaves the
// context's resident data unreliable: the kernel skipped its work, and a copy may still have been in
// flight when it returned.  Entry points that synchronise with the device read the flag word in that
// synchronisation; once the bit is seen the context is dead and every later call on it returns
// DNDSG_TIMEOUT (dndsg_destroy and dndsg_last_error still work).
int refuse_dead(dndsg_ctx* c) {
  return fail(c, DNDSG_TIMEOUT, "a bounded wait in a kernel ran out earlier; the context refuses further work");
}

int observe_timeout(dndsg_ctx* c, cudaStream_t s) {
  unsigned f = 0;
  DG_CUDA(c, cudaMemcpyAsync(&f, c->flags, sizeof(f), cudaMemcpyDeviceToHost, s));
  DG_CUDA(c, cudaStreamSynchronize(s));
  if (f & kFlagTimeout) {
    c->dead = true;
    return fail(c, DNDSG_TIMEOUT, "a bounded wait in a kernel ran out (timeout flag); the context refuses further work");
  }
  return 0;
}

// A cell's face slots in element-local face order, the order of the reference's cell2face (vol2face is
// filled per local face, DNDS_Mesh.hpp:288-320): slot k holds the face joining nodes k and k+1
// (FaceNodeList of TRI3 / QUAD4, DNDS_Elements.hpp:248-253).  A face is matched by its node pair, or --
// a periodic face seen from its translated side -- by its midpoint against the edge midpoint moved by
// the face shift.  Sums over a cell's faces run in slot order, and V2's multiway WBAP is centred on
// the first slot's neighbour.  slot[k] encodes the face as f (left side) or ~f (right side).
void order_cell_slots(const dndsg_mesh_desc* md, int64_t i, int32_t* slot, int nf) {
  const int nn = md->cell_nodes[4 * i + 3] < 0 ? 3 : 4;
  if (nf != nn) return;
  int32_t out[4] = {0, 0, 0, 0};
  bool got[4] = {false, false, false, false}, used[4] = {false, false, false, false};
  for (int pass = 0; pass < 2; pass++)
    for (int e = 0; e < nn; e++) {
      if (got[e]) continue;
      const int32_t p = md->cell_nodes[4 * i + e], q = md->cell_nodes[4 * i + (e + 1) % nn];
      const double mx = 0.5 * (md->node_xy[2 * p] + md->node_xy[2 * q]);
      const double my = 0.5 * (md->node_xy[2 * p + 1] + md->node_xy[2 * q + 1]);
      const double len = std::hypot(md->node_xy[2 * q] - md->node_xy[2 * p], md->node_xy[2 * q + 1] - md->node_xy[2 * p + 1]);
      for (int k = 0; k < nf && !got[e]; k++) {
        if (used[k]) continue;
        const int32_t f = slot[k] >= 0 ? slot[k] : ~slot[k];
        const int32_t a = md->face_nodes[2 * f], b = md->face_nodes[2 * f + 1];
        bool hit = (a == p && b == q) || (a == q && b == p);
        if (!hit && pass == 1 && md->face_shift) {
          const double fx = 0.5 * (md->node_xy[2 * a] + md->node_xy[2 * b]);
          const double fy = 0.5 * (md->node_xy[2 * a + 1] + md->node_xy[2 * b + 1]);
          const double sx = md->face_shift[2 * f], sy = md->face_shift[2 * f + 1];
          for (int sg = -1; sg <= 1 && !hit; sg += 2)
            hit = std::fabs(mx + sg * sx - fx) + std::fabs(my + sg * sy - fy) < 1e-9 * len;
        }
        if (hit) {
          out[e] = slot[k];
          got[e] = used[k] = true;
        }
      }
    }
  for (int e = 0; e < nn; e++)
    if (!got[e]) return;  // unmatched: keep the given order
  for (int e = 0; e < nn; e++) slot[e] = out[e];
}

template <class T>
int setup_run(dndsg_ctx* c, const dndsg_mesh_desc* md) {
  const int64_t N = c->N, F = c->F;
  // ---- host-side topology: per-cell face slots, closure vectors, checks
  std::vector<int32_t> slots((size_t)aos_size(N, c->nfmax), kEmptySlot);
  std::vector<int> cnt(N, 0);
  std::vector<double> closure(2 * N, 0.0);
  bool hasWallCorr = false;
  for (int64_t f = 0; f < F; f++) {
    int32_t L = md->face_cells[2 * f], R = md->face_cells[2 * f + 1];
    if (L < 0 || L >= N || R >= N || R < -1) return fail(c, DNDSG_BAD_ARGUMENT, "face_cells out of range");
    int32_t a = md->face_nodes[2 * f], b = md->face_nodes[2 * f + 1];
    if (a < 0 || b < 0 || a >= md->n_nodes || b >= md->n_nodes) return fail(c, DNDSG_BAD_ARGUMENT, "face_nodes out of range");
    int bc = md->face_bc[f];
    if (R < 0 && !(bc == BC_WALL || bc == BC_FAR || bc == BC_WALL_EULER || bc == BC_WALL_NOSLIP || bc == BC_IV_FAR ||
                   bc == BC_RIEMANN_FAR))
      return fail(c, DNDSG_UNSUPPORTED, "boundary face with an unsupported BoundaryType");
    if (R >= 0 && bc != BC_INNER) return fail(c, DNDSG_BAD_ARGUMENT, "interior face with a boundary type");
    if (bc == BC_WALL_EULER || bc == BC_WALL_NOSLIP) hasWallCorr = true;
    double dx = md->node_xy[2 * b] - md->node_xy[2 * a], dy = md->node_xy[2 * b + 1] - md->node_xy[2 * a + 1];
    if (cnt[L] >= c->nfmax) return fail(c, DNDSG_BAD_ARGUMENT, "cell with more faces than nodes");
    slots[aos(L, cnt[L]++, c->nfmax)] = (int32_t)f;
    closure[2 * L] += dy; closure[2 * L + 1] += -dx;
    if (R >= 0) {
      if (cnt[R] >= c->nfmax) return fail(c, DNDSG_BAD_ARGUMENT, "cell with more faces than nodes");
      slots[aos(R, cnt[R]++, c->nfmax)] = ~(int32_t)f;
      closure[2 * R] -= dy; closure[2 * R + 1] -= -dx;
    }
  }
  for (int64_t i = 0; i < N; i++) {
    int nn = md->cell_nodes[4 * i + 3] < 0 ? 3 : 4;
    for (int k = 0; k < nn; k++) {
      int32_t nd = md->cell_nodes[4 * i + k];
      if (nd < 0 || nd >= md->n_nodes) return fail(c, DNDSG_BAD_ARGUMENT, "cell_nodes out of range");
    }
    if (cnt[i] != nn) return fail(c, DNDSG_BAD_ARGUMENT, "cell face count differs from its node count");
    int32_t sl[4];
    for (int k = 0; k < nn; k++) sl[k] = slots[aos(i, k, c->nfmax)];
    order_cell_slots(md, i, sl, nn);
    for (int k = 0; k < nn; k++) slots[aos(i, k, c->nfmax)] = sl[k];
  }
  c->hasWallCorr = hasWallCorr;
  // ---- device mesh
  double* dNode; int32_t *dCellNodes, *dFaceNodes, *dFaceCells; double* dShift = nullptr;
  int rc = 0;
  if ((rc = dalloc(c, dNode, sizeof(double) * 2 * md->n_nodes))) return rc;
  if ((rc = dalloc(c, dCellNodes, sizeof(int32_t) * 4 * N))) return rc;
  if ((rc = dalloc(c, dFaceNodes, sizeof(int32_t) * 2 * F))) return rc;
  if ((rc = dalloc(c, dFaceCells, sizeof(int32_t) * 2 * F))) return rc;
  if ((rc = dalloc(c, c->faceBC, sizeof(int32_t) * F))) return rc;
  if ((rc = dalloc(c, c->faceL, sizeof(int32_t) * F))) return rc;
  if ((rc = dalloc(c, c->faceR, sizeof(int32_t) * F))) return rc;
  DG_CUDA(c, cudaMemcpy(dNode, md->node_xy, sizeof(double) * 2 * md->n_nodes, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(dCellNodes, md->cell_nodes, sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(dFaceNodes, md->face_nodes, sizeof(int32_t) * 2 * F, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(dFaceCells, md->face_cells, sizeof(int32_t) * 2 * F, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->faceBC, md->face_bc, sizeof(int32_t) * F, cudaMemcpyHostToDevice));
  {
    std::vector<int32_t> l(F), r(F);
    for (int64_t f = 0; f < F; f++) { l[f] = md->face_cells[2 * f]; r[f] = md->face_cells[2 * f + 1]; }
    DG_CUDA(c, cudaMemcpy(c->faceL, l.data(), sizeof(int32_t) * F, cudaMemcpyHostToDevice));
    DG_CUDA(c, cudaMemcpy(c->faceR, r.data(), sizeof(int32_t) * F, cudaMemcpyHostToDevice));
  }
  if (md->face_shift) {
    if ((rc = dalloc(c, dShift, sizeof(double) * 2 * F))) return rc;
    DG_CUDA(c, cudaMemcpy(dShift, md->face_shift, sizeof(double) * 2 * F, cudaMemcpyHostToDevice));
  }
  MeshView m{N, F, dNode, dCellNodes, dFaceNodes, dFaceCells, c->faceBC, dShift};
  SetupParams p;
  p.use_local_coord = c->s.use_local_coord; p.anisotropic_lengths = c->s.anisotropic_lengths;
  p.base_center_type = c->s.base_center_type; p.weight_scheme_geom = c->s.weight_scheme_geom;
  p.weight_scheme_dir = c->s.weight_scheme_dir; p.tang_weight_direction = c->s.tang_weight_direction;
  p.tang_weight_mod_loc = c->s.tang_weight_mod_loc; p.weight_len_scale = c->s.weight_len_scale;
  p.wall_weight = c->s.wall_weight; p.far_weight = c->s.far_weight; p.tang_weight = c->s.tang_weight;
  p.tang_weight_mod_min = c->s.tang_weight_mod_min; p.tang_weight_mod_power = c->s.tang_weight_mod_power;
  // ---- per-cell geometry
  CellSetup* cells;
  double* bary;
  int* dBad;
  if ((rc = dalloc(c, cells, sizeof(CellSetup) * N))) return rc;
  if ((rc = dalloc(c, c->vol, sizeof(double) * N))) return rc;
  if ((rc = dalloc(c, bary, sizeof(double) * 2 * N))) return rc;
  if ((rc = dalloc(c, dBad, sizeof(int)))) return rc;
  DG_CUDA(c, cudaMemset(dBad, 0, sizeof(int)));
  k_setup_cell<<<grid_for(N), kBlock>>>(m, p, cells, c->vol, bary, dBad);
  if ((rc = check_launch(c))) return rc;
  // ---- faces
  double* faceW;
  if ((rc = dalloc(c, faceW, sizeof(double) * 6 * F))) return rc;
  if ((rc = dalloc(c, c->faceNormal, sizeof(double) * 2 * F))) return rc;
  if ((rc = dalloc(c, c->faceArea, sizeof(double) * F))) return rc;
  if ((rc = dalloc(c, c->faceCenter, sizeof(double) * 2 * F))) return rc;
  if ((rc = dalloc(c, c->faceW0, sizeof(double) * F))) return rc;
  if ((rc = dalloc(c, c->faceBasis, sizeof(T) * aos_size(F, kFaceBasisE)))) return rc;
  k_setup_face<T><<<grid_for(F), kBlock>>>(m, p, cells, faceW, c->faceNormal, c->faceArea, c->faceCenter, c->faceW0,
                                           (T*)c->faceBasis);
  if ((rc = check_launch(c))) return rc;
  if (c->s.mu_gas > 0) {
    if ((rc = dalloc(c, c->faceGrad, sizeof(T) * aos_size(F, 60)))) return rc;
    k_setup_face_grad<T><<<grid_for(F), kBlock>>>(m, cells, (T*)c->faceGrad);
    if ((rc = check_launch(c))) return rc;
  }
  if (c->sa) {
    // wall segments for the first-order wall distance, and the cell quadrature data of the source
    std::vector<double> seg;
    for (int64_t f = 0; f < F; f++)
      if (md->face_bc[f] == BC_WALL_NOSLIP) {
        const int32_t a = md->face_nodes[2 * f], b = md->face_nodes[2 * f + 1];
        seg.insert(seg.end(), {md->node_xy[2 * a], md->node_xy[2 * a + 1], md->node_xy[2 * b], md->node_xy[2 * b + 1]});
      }
    double* dSeg = nullptr;
    const int64_t nw = (int64_t)seg.size() / 4;
    if (nw > 0) {
      if ((rc = dalloc(c, dSeg, sizeof(double) * seg.size()))) return rc;
      DG_CUDA(c, cudaMemcpy(dSeg, seg.data(), sizeof(double) * seg.size(), cudaMemcpyHostToDevice));
    }
    if ((rc = dalloc(c, c->saCellGp, sizeof(double) * N * kSaGp * kSaGpE)) || (rc = dalloc(c, c->saDWall, sizeof(double) * N)))
      return rc;
    k_setup_sa_cells<<<grid_for(N), kBlock>>>(N, cells, dSeg, nw, c->saCellGp, c->saDWall);
    if ((rc = check_launch(c))) return rc;
    DG_CUDA(c, cudaDeviceSynchronize());
    if (dSeg) {
      auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)dSeg);
      if (it != c->allocs.end()) { cudaFree(dSeg); c->allocs.erase(it); }
    }
  }
  // ---- VR matrices
  if ((rc = dalloc(c, c->cellFace, sizeof(int32_t) * slots.size()))) return rc;
  DG_CUDA(c, cudaMemcpy(c->cellFace, slots.data(), sizeof(int32_t) * slots.size(), cudaMemcpyHostToDevice));
  if ((rc = dalloc(c, c->vrNbr, sizeof(int32_t) * slots.size()))) return rc;
  if ((rc = dalloc(c, c->vrMode, sizeof(int32_t) * slots.size()))) return rc;
  if ((rc = dalloc(c, c->vrFace, sizeof(int32_t) * slots.size()))) return rc;
  // padded to whole bulk-copy tiles (128 cells) so every tile copy stays inside the allocation
  if ((rc = dalloc(c, c->vrOp, sizeof(T) * aos_size(((N + 127) / 128) * 128, c->nfmax * 30)))) return rc;
  {
    constexpr int TILE = vr_tile<T>();
    DG_CUDA(c, cudaFuncSetAttribute(k_vr_tma4<T, TILE, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(TILE * 3 * 30 * sizeof(T))));
    DG_CUDA(c, cudaFuncSetAttribute(k_vr_tma4<T, TILE, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(TILE * 4 * 30 * sizeof(T))));
  }
  if (hasWallCorr)
    if ((rc = dalloc(c, c->Ainv, sizeof(double) * 25 * N))) return rc;
  k_setup_matrices<T><<<grid_for(N), kBlock>>>(m, p, cells, faceW, c->cellFace, c->nfmax, (T*)c->vrOp, c->vrNbr,
                                               c->vrMode, c->vrFace, c->Ainv, dBad);
  if ((rc = check_launch(c))) return rc;
  if ((rc = dalloc(c, c->mlpGeom, sizeof(float) * 8 * N))) return rc;
  k_setup_mlp_geom<<<grid_for(N), kBlock>>>(m, cells, c->cellFace, c->nfmax, c->faceCenter, c->mlpGeom);
  if ((rc = check_launch(c))) return rc;
  if (c->s.limiter) {
    if ((rc = dalloc(c, c->limFace, sizeof(T) * kLimStride * F))) return rc;
    if ((rc = dalloc(c, c->faceInd, sizeof(T) * 4 * F))) return rc;
    if ((rc = dalloc(c, c->indicator, sizeof(double) * N))) return rc;
    if ((rc = dalloc(c, c->limList, sizeof(int32_t) * N)) || (rc = dalloc(c, c->limCount, sizeof(int32_t)))) return rc;
    k_setup_limiter<T><<<grid_for(F), kBlock>>>(m, p, cells, faceW, (T*)c->limFace, dBad);
    if ((rc = check_launch(c))) return rc;
    if ((rc = dalloc(c, c->limG, sizeof(T) * aos_size(F, kLimG))) ||
        (rc = dalloc(c, c->limCell, sizeof(T) * kLimCell * N)))
      return rc;
    k_setup_lim_compact<T><<<grid_for(std::max<int64_t>(F, N)), kBlock>>>(m, cells, faceW, (T*)c->limG, (T*)c->limCell);
    if ((rc = check_launch(c))) return rc;
  }
  DG_CUDA(c, cudaDeviceSynchronize());
  int bad = 0;
  DG_CUDA(c, cudaMemcpy(&bad, dBad, sizeof(int), cudaMemcpyDeviceToHost));
  if (bad & 1) return fail(c, DNDSG_SETUP_ERROR, "non-positive cell jacobian (cell not counter-clockwise?)");
  if (bad & 2) return fail(c, DNDSG_SETUP_ERROR, "VR matrix A_ii is not positive definite");
  if (bad & 4) return fail(c, DNDSG_SETUP_ERROR, "singular secondary-reconstruction matrix at a face");
  {
    std::vector<char> isWall(N, 0);
    for (int64_t f = 0; f < F; f++) {
      int bc = md->face_bc[f];
      if (md->face_cells[2 * f + 1] < 0 && (bc == BC_WALL_EULER || bc == BC_WALL_NOSLIP)) isWall[md->face_cells[2 * f]] = 1;
    }
    std::vector<int32_t> wc;
    for (int64_t i = 0; i < N; i++) if (isWall[i]) wc.push_back((int32_t)i);
    c->nWallCells = (int64_t)wc.size();
    if (!wc.empty()) {
      if ((rc = dalloc(c, c->wallCells, sizeof(int32_t) * wc.size()))) return rc;
      DG_CUDA(c, cudaMemcpy(c->wallCells, wc.data(), sizeof(int32_t) * wc.size(), cudaMemcpyHostToDevice));
    }
  }
  if ((rc = dalloc(c, c->closure, sizeof(double) * 2 * N))) return rc;
  DG_CUDA(c, cudaMemcpy(c->closure, closure.data(), sizeof(double) * 2 * N, cudaMemcpyHostToDevice));
  // setup-only buffers are released here
  for (void* q : {(void*)dNode, (void*)dCellNodes, (void*)dFaceNodes, (void*)dFaceCells, (void*)dShift, (void*)cells,
                  (void*)bary, (void*)faceW, (void*)dBad}) {
    if (!q) continue;
    auto it = std::find(c->allocs.begin(), c->allocs.end(), q);
    if (it != c->allocs.end()) { cudaFree(q); c->allocs.erase(it); }
  }
  // ---- state
  if ((rc = dalloc(c, c->u, sizeof(double) * 4 * N))) return rc;
  if ((rc = dalloc(c, c->uLast, sizeof(double) * 4 * N))) return rc;
  if ((rc = dalloc(c, c->rhs, sizeof(double) * 4 * N))) return rc;
  if ((rc = dalloc(c, c->dt, sizeof(double) * N))) return rc;
  if ((rc = dalloc(c, c->urec, sizeof(T) * 20 * N))) return rc;
  if ((rc = dalloc(c, c->urecNew, sizeof(T) * 20 * N))) return rc;
  if ((rc = dalloc(c, c->flux, sizeof(double) * 4 * F))) return rc;
  if ((rc = dalloc(c, c->lamA, sizeof(double) * F))) return rc;
  if ((rc = dalloc(c, c->dLam, sizeof(double) * F))) return rc;
  if ((rc = dalloc(c, c->scal, sizeof(double) * S_NSLOT))) return rc;
  if ((rc = dalloc(c, c->partial, sizeof(double) * 4 * grid_for(N)))) return rc;
  if ((rc = dalloc(c, c->flags, sizeof(unsigned)))) return rc;
  if ((rc = dalloc(c, c->nreduced, sizeof(unsigned long long)))) return rc;
  DG_CUDA(c, cudaMemset(c->u, 0, sizeof(double) * 4 * N));
  DG_CUDA(c, cudaMemset(c->urec, 0, sizeof(T) * 20 * N));
  DG_CUDA(c, cudaMemset(c->urecNew, 0, sizeof(T) * 20 * N));
  DG_CUDA(c, cudaMemset(c->dLam, 0, sizeof(double) * F));
  DG_CUDA(c, cudaMemset(c->scal, 0, sizeof(double) * S_NSLOT));
  DG_CUDA(c, cudaMemset(c->flags, 0, sizeof(unsigned)));
  DG_CUDA(c, cudaMemset(c->nreduced, 0, sizeof(unsigned long long)));
  if (c->sa) {
    for (double** q : {&c->saU, &c->saULast, &c->saRhs, &c->saInc, &c->saDinv, &c->saSrcJac})
      if ((rc = dalloc(c, *q, sizeof(double) * N))) return rc;
    if ((rc = dalloc(c, c->saFlux, sizeof(double) * F)) || (rc = dalloc(c, c->saUrec, sizeof(T) * 5 * N)) ||
        (rc = dalloc(c, c->saUrecNew, sizeof(T) * 5 * N)))
      return rc;
    for (double* q : {c->saU, c->saULast, c->saRhs, c->saInc, c->saSrcJac}) DG_CUDA(c, cudaMemset(q, 0, sizeof(double) * N));
    DG_CUDA(c, cudaMemset(c->saFlux, 0, sizeof(double) * F));
    DG_CUDA(c, cudaMemset(c->saUrec, 0, sizeof(T) * 5 * N));
    DG_CUDA(c, cudaMemset(c->saUrecNew, 0, sizeof(T) * 5 * N));
  }
  DG_CUDA(c, cudaDeviceSynchronize());
  return 0;
}

}  // namespace

// SA-context drivers, defined with their kernels at the end of this file
namespace {
int sa_vr_steps(dndsg_ctx* c, int nsweeps, cudaStream_t s);
int sa_eval_dt(dndsg_ctx* c, double cfl, double maxDt, cudaStream_t s);
int sa_eval_rhs(dndsg_ctx* c, cudaStream_t s);
int sa_implicit(dndsg_ctx* c, double cfl, double dtPhys, double alpha, int nRec, int volWise, cudaStream_t s);
}  // namespace

// ====================================================================== C ABI
extern "C" {

int dndsg_create(const dndsg_mesh_desc* mesh, const dndsg_settings* settings, int device, dndsg_ctx** out) {
  if (!out) return DNDSG_BAD_ARGUMENT;
  *out = nullptr;
  dndsg_ctx* c = new dndsg_ctx();
  *out = c;
  if (!mesh || !settings) return fail(c, DNDSG_BAD_ARGUMENT, "null mesh or settings");
  c->s = *settings;
  c->device = device;
  if (c->s.nvars != 4 && c->s.nvars != 5) return fail(c, DNDSG_UNSUPPORTED, "nvars must be 4 (NS_2D) or 5 (with SA)");
  c->sa = c->s.nvars == 5;
  if (c->sa && !(c->s.mu_gas > 0)) return fail(c, DNDSG_UNSUPPORTED, "the SA model needs mu_gas > 0");
  if (c->sa && c->s.limiter) return fail(c, DNDSG_UNSUPPORTED, "the SA contexts run without the limiter");
  if (c->s.rec_order != 2) return fail(c, DNDSG_UNSUPPORTED, "rec_order must be 2 (P2)");
  if (c->s.sor_instead) return fail(c, DNDSG_UNSUPPORTED, "the GPU VR sweep is Jacobi (sor_instead must be 0)");
  if (c->s.riemann != 1 && c->s.riemann != 2) return fail(c, DNDSG_UNSUPPORTED, "riemann must be 1 (Roe) or 2 (HLLC)");
  if (mesh->n_cells <= 0 || mesh->n_faces <= 0 || mesh->n_cells > INT32_MAX || mesh->n_faces > INT32_MAX)
    return fail(c, DNDSG_BAD_ARGUMENT, "mesh sizes out of range");
  c->N = mesh->n_cells;
  c->F = mesh->n_faces;
  c->fp32 = c->s.precision == 1;
  bool anyQuad = false;
  for (int64_t i = 0; i < c->N; i++) if (mesh->cell_nodes[4 * i + 3] >= 0) { anyQuad = true; break; }
  c->nfmax = anyQuad ? 4 : 3;
  int rc = set_device(c);
  if (rc) return rc;
  if (cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) c->sms = 148;
  // internal face order: interior faces first, then boundary faces, so the hot
  // flux kernel carries no boundary-condition code
  const int64_t F = c->F;
  c->facePerm.reserve(F);
  for (int64_t f = 0; f < F; f++) if (mesh->face_cells[2 * f + 1] >= 0) c->facePerm.push_back(f);
  c->Fi = (int64_t)c->facePerm.size();
  for (int64_t f = 0; f < F; f++) if (mesh->face_cells[2 * f + 1] < 0) c->facePerm.push_back(f);
  std::vector<int32_t> fn(2 * F), fc(2 * F), fb(F);
  std::vector<double> fs(mesh->face_shift ? 2 * F : 0);
  for (int64_t k = 0; k < F; k++) {
    int64_t f = c->facePerm[k];
    fn[2 * k] = mesh->face_nodes[2 * f]; fn[2 * k + 1] = mesh->face_nodes[2 * f + 1];
    fc[2 * k] = mesh->face_cells[2 * f]; fc[2 * k + 1] = mesh->face_cells[2 * f + 1];
    fb[k] = mesh->face_bc[f];
    if (mesh->face_shift) { fs[2 * k] = mesh->face_shift[2 * f]; fs[2 * k + 1] = mesh->face_shift[2 * f + 1]; }
  }
  dndsg_mesh_desc pm = *mesh;
  pm.face_nodes = fn.data(); pm.face_cells = fc.data(); pm.face_bc = fb.data();
  pm.face_shift = mesh->face_shift ? fs.data() : nullptr;
  rc = c->fp32 ? setup_run<float>(c, &pm) : setup_run<double>(c, &pm);
  return rc;
}

void dndsg_destroy(dndsg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  for (auto& g : c->stepGraph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (c->capStream) cudaStreamDestroy(c->capStream);
  for (void* p : c->allocs) cudaFree(p);
  delete c;
}

const char* dndsg_last_error(dndsg_ctx* c) { return c ? c->err.c_str() : "null context"; }
int64_t dndsg_n_cells(dndsg_ctx* c) { return c ? c->N : -1; }
int64_t dndsg_n_faces(dndsg_ctx* c) { return c ? c->F : -1; }

int dndsg_set_u(dndsg_ctx* c, const double* u, void* s) {
  if (!c || !u) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) {  // [N][5] -> flow [N][4] + U5 [N]
    std::vector<double> a(4 * c->N), b(c->N);
    for (int64_t i = 0; i < c->N; i++) {
      for (int v = 0; v < 4; v++) a[4 * i + v] = u[5 * i + v];
      b[i] = u[5 * i + 4];
    }
    DG_CUDA(c, cudaMemcpy(c->u, a.data(), sizeof(double) * 4 * c->N, cudaMemcpyHostToDevice));
    DG_CUDA(c, cudaMemcpy(c->saU, b.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice));
    return 0;
  }
  DG_CUDA(c, cudaMemcpyAsync(c->u, u, sizeof(double) * 4 * c->N, cudaMemcpyHostToDevice, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  return 0;
}
int dndsg_get_u(dndsg_ctx* c, double* u, void* s) {
  if (!c || !u) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) {
    DG_CUDA(c, cudaStreamSynchronize(st(s)));
    std::vector<double> a(4 * c->N), b(c->N);
    DG_CUDA(c, cudaMemcpy(a.data(), c->u, sizeof(double) * 4 * c->N, cudaMemcpyDeviceToHost));
    DG_CUDA(c, cudaMemcpy(b.data(), c->saU, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < c->N; i++) {
      for (int v = 0; v < 4; v++) u[5 * i + v] = a[4 * i + v];
      u[5 * i + 4] = b[i];
    }
    return observe_timeout(c, st(s));
  }
  DG_CUDA(c, cudaMemcpyAsync(u, c->u, sizeof(double) * 4 * c->N, cudaMemcpyDeviceToHost, st(s)));
  return observe_timeout(c, st(s));
}
int dndsg_get_dt(dndsg_ctx* c, double* dt, void* s) {
  if (!c || !dt) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  DG_CUDA(c, cudaMemcpyAsync(dt, c->dt, sizeof(double) * c->N, cudaMemcpyDeviceToHost, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  return 0;
}

}  // extern "C"

namespace {
// host-side split / merge of [N][5][5] coefficients of an SA context, in the context's precision
template <class T>
int sa_urec_io(dndsg_ctx* c, double* r, bool set) {
  const int64_t N = c->N;
  std::vector<T> a(20 * N), b(5 * N);
  if (set) {
    for (int64_t i = 0; i < N; i++)
      for (int q = 0; q < 5; q++) {
        for (int v = 0; v < 4; v++) a[20 * i + 4 * q + v] = (T)r[25 * i + 5 * q + v];
        b[5 * i + q] = (T)r[25 * i + 5 * q + 4];
      }
    DG_CUDA(c, cudaMemcpy(c->urec, a.data(), sizeof(T) * 20 * N, cudaMemcpyHostToDevice));
    DG_CUDA(c, cudaMemcpy(c->saUrec, b.data(), sizeof(T) * 5 * N, cudaMemcpyHostToDevice));
  } else {
    DG_CUDA(c, cudaDeviceSynchronize());
    DG_CUDA(c, cudaMemcpy(a.data(), c->urec, sizeof(T) * 20 * N, cudaMemcpyDeviceToHost));
    DG_CUDA(c, cudaMemcpy(b.data(), c->saUrec, sizeof(T) * 5 * N, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < N; i++)
      for (int q = 0; q < 5; q++) {
        for (int v = 0; v < 4; v++) r[25 * i + 5 * q + v] = (double)a[20 * i + 4 * q + v];
        r[25 * i + 5 * q + 4] = (double)b[5 * i + q];
      }
  }
  return 0;
}
}  // namespace

extern "C" {

int dndsg_set_urec(dndsg_ctx* c, const double* r, void* s) {
  if (!c || !r) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return c->fp32 ? sa_urec_io<float>(c, const_cast<double*>(r), true) : sa_urec_io<double>(c, const_cast<double*>(r), true);
  const int64_t n = 20 * c->N;
  if (!c->fp32) {
    DG_CUDA(c, cudaMemcpyAsync(c->urec, r, sizeof(double) * n, cudaMemcpyHostToDevice, st(s)));
  } else {
    double* tmp;
    DG_CUDA(c, cudaMallocAsync((void**)&tmp, sizeof(double) * n, st(s)));
    DG_CUDA(c, cudaMemcpyAsync(tmp, r, sizeof(double) * n, cudaMemcpyHostToDevice, st(s)));
    k_cvt_to<float><<<grid_for(n), kBlock, 0, st(s)>>>(tmp, (float*)c->urec, n);
    DG_CUDA(c, cudaFreeAsync(tmp, st(s)));
  }
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  return check_launch(c);
}
int dndsg_get_urec(dndsg_ctx* c, double* r, void* s) {
  if (!c || !r) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return c->fp32 ? sa_urec_io<float>(c, r, false) : sa_urec_io<double>(c, r, false);
  const int64_t n = 20 * c->N;
  if (!c->fp32) {
    DG_CUDA(c, cudaMemcpyAsync(r, c->urec, sizeof(double) * n, cudaMemcpyDeviceToHost, st(s)));
  } else {
    double* tmp;
    DG_CUDA(c, cudaMallocAsync((void**)&tmp, sizeof(double) * n, st(s)));
    k_cvt_from<float><<<grid_for(n), kBlock, 0, st(s)>>>((const float*)c->urec, tmp, n);
    DG_CUDA(c, cudaMemcpyAsync(r, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, st(s)));
    DG_CUDA(c, cudaFreeAsync(tmp, st(s)));
  }
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  return check_launch(c);
}

int dndsg_device_buffer(dndsg_ctx* c, int which, void** ptr, int64_t* bytes) {
  if (!c || !ptr) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  switch (which) {
    case DNDSG_BUF_U: *ptr = c->u; if (bytes) *bytes = sizeof(double) * 4 * c->N; return 0;
    case DNDSG_BUF_UREC: *ptr = c->urec; if (bytes) *bytes = (int64_t)c->tsize() * 20 * c->N; return 0;
    case DNDSG_BUF_RHS: *ptr = c->rhs; if (bytes) *bytes = sizeof(double) * 4 * c->N; return 0;
    case DNDSG_BUF_DT: *ptr = c->dt; if (bytes) *bytes = sizeof(double) * c->N; return 0;
    case DNDSG_BUF_SA_U:
      if (!c->sa) break;
      *ptr = c->saU; if (bytes) *bytes = sizeof(double) * c->N; return 0;
    case DNDSG_BUF_SA_UREC:
      if (!c->sa) break;
      *ptr = c->saUrec; if (bytes) *bytes = (int64_t)c->tsize() * 5 * c->N; return 0;
  }
  return fail(c, DNDSG_BAD_ARGUMENT, "unknown buffer id");
}

int dndsg_get_time(dndsg_ctx* c, double* t, void* s) {
  if (!c || !t) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  DG_CUDA(c, cudaMemcpyAsync(t, c->scal + S_T, sizeof(double), cudaMemcpyDeviceToHost, st(s)));
  return observe_timeout(c, st(s));
}
int dndsg_set_time(dndsg_ctx* c, double t, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  DG_CUDA(c, cudaMemcpyAsync(c->scal + S_T, &t, sizeof(double), cudaMemcpyHostToDevice, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  return 0;
}

int dndsg_vr_jacobi_step(dndsg_ctx* c, int nsweeps, double* inc_out, void* s) {
  if (!c || nsweeps < 0) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) {
    if (inc_out) return fail(c, DNDSG_UNSUPPORTED, "SA contexts report no sweep increment");
    return sa_vr_steps(c, nsweeps, st(s));
  }
  for (int k = 0; k < nsweeps; k++) {
    bool last = inc_out && k == nsweeps - 1;
    if (last) k_init_dtmin<<<1, 1, 0, st(s)>>>(c->scal);
    if (c->fp32) run_vr<float>(c, last, st(s));
    else run_vr<double>(c, last, st(s));
  }
  int rc = check_launch(c);
  if (rc) return rc;
  if (inc_out) {
    double v = 0;
    DG_CUDA(c, cudaMemcpyAsync(&v, c->scal + S_INC, sizeof(double), cudaMemcpyDeviceToHost, st(s)));
    DG_CUDA(c, cudaStreamSynchronize(st(s)));
    *inc_out = v / double(c->N);
  }
  return 0;
}

static int limiter_api(dndsg_ctx* c, int version, int if_all, double* indicator_out, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (!c->limFace) return fail(c, DNDSG_UNSUPPORTED, "context was created without the limiter (settings.limiter = 0)");
  if (version == 3) {
    if (c->fp32) run_limiter_v3<float>(c, if_all, st(s));
    else run_limiter_v3<double>(c, if_all, st(s));
  } else {
    if (c->fp32) run_limiter_v2<float>(c, if_all, st(s));
    else run_limiter_v2<double>(c, if_all, st(s));
  }
  int rc = check_launch(c);
  if (rc) return rc;
  if (indicator_out) {
    DG_CUDA(c, cudaMemcpyAsync(indicator_out, c->indicator, sizeof(double) * c->N, cudaMemcpyDeviceToHost, st(s)));
    DG_CUDA(c, cudaStreamSynchronize(st(s)));
  }
  return 0;
}

int dndsg_limiter_wbap(dndsg_ctx* c, int if_all, double* indicator_out, void* s) {
  return limiter_api(c, 3, if_all, indicator_out, s);
}

int dndsg_limiter_wbap_v2(dndsg_ctx* c, int if_all, double* indicator_out, void* s) {
  return limiter_api(c, 2, if_all, indicator_out, s);
}

int dndsg_eval_dt(dndsg_ctx* c, double cfl, double max_dt, int use_local_dt, double* dt_min_out, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) {
    int rc0 = sa_eval_dt(c, cfl, max_dt, st(s));
    if (rc0) return rc0;
  } else if (c->fp32) run_dt<float>(c, cfl, max_dt, false, st(s));
  else run_dt<double>(c, cfl, max_dt, false, st(s));
  if (!use_local_dt) k_fill_dt<<<grid_for(c->N), kBlock, 0, st(s)>>>(c->dt, c->N, c->scal);
  int rc = check_launch(c);
  if (rc) return rc;
  if (dt_min_out) {
    unsigned long long bits = 0;
    DG_CUDA(c, cudaMemcpyAsync(&bits, c->scal + S_DTMIN, sizeof(bits), cudaMemcpyDeviceToHost, st(s)));
    DG_CUDA(c, cudaStreamSynchronize(st(s)));
    std::memcpy(dt_min_out, &bits, sizeof(double));
  }
  return 0;
}

int dndsg_eval_rhs(dndsg_ctx* c, double t, double* rhs_out, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) {
    int rc0 = sa_eval_rhs(c, st(s));
    if (rc0) return rc0;
    if (rhs_out) {
      DG_CUDA(c, cudaStreamSynchronize(st(s)));
      std::vector<double> a(4 * c->N), b(c->N);
      DG_CUDA(c, cudaMemcpy(a.data(), c->rhs, sizeof(double) * 4 * c->N, cudaMemcpyDeviceToHost));
      DG_CUDA(c, cudaMemcpy(b.data(), c->saRhs, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < c->N; i++) {
        for (int v = 0; v < 4; v++) rhs_out[5 * i + v] = a[4 * i + v];
        rhs_out[5 * i + 4] = b[i];
      }
    }
    return 0;
  }
  if (c->fp32) run_rhs<float>(c, t, st(s));
  else run_rhs<double>(c, t, st(s));
  int rc = check_launch(c);
  if (rc) return rc;
  if (rhs_out) {
    DG_CUDA(c, cudaMemcpyAsync(rhs_out, c->rhs, sizeof(double) * 4 * c->N, cudaMemcpyDeviceToHost, st(s)));
    DG_CUDA(c, cudaStreamSynchronize(st(s)));
  }
  return 0;
}

int dndsg_ssprk3_step(dndsg_ctx* c, double cfl, double t_end, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "SA contexts run the implicit path (dndsg_implicit_iteration)");
  if (c->fp32) run_step<float>(c, cfl, t_end, st(s));
  else run_step<double>(c, cfl, t_end, st(s));
  return check_launch(c);
}

// n SSP-RK3 steps, pairs of them replayed from a CUDA graph: on small meshes a step is a handful of
// microseconds of work behind 14 launches, and one graph launch replaces 28.  The graph is captured
// (on a private stream) the first time a cfl / t_end / buffer parity is seen and kept.
int dndsg_ssprk3_steps(dndsg_ctx* c, double cfl, double t_end, int64_t n, void* s) {
  if (!c || n < 0) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "SA contexts run the implicit path (dndsg_implicit_iteration)");
  int rc;
  if ((rc = set_device(c))) return rc;
  if (n >= 2) {
    int slot = -1;
    for (int k = 0; k < 2; k++)
      if (c->stepGraph[k].exec && c->stepGraph[k].urec == c->urec) slot = k;
    if (slot < 0) slot = c->stepGraph[0].exec ? 1 : 0;
    dndsg_ctx::StepGraph& g = c->stepGraph[slot];
    if (!g.exec || g.cfl != cfl || g.tEnd != t_end) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
      if (!c->capStream) DG_CUDA(c, cudaStreamCreateWithFlags(&c->capStream, cudaStreamNonBlocking));
      void* urec0 = c->urec;
      DG_CUDA(c, cudaStreamBeginCapture(c->capStream, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < 2; k++) {  // six buffer swaps: urec is back in its buffer afterwards
        if (c->fp32) run_step<float>(c, cfl, t_end, c->capStream);
        else run_step<double>(c, cfl, t_end, c->capStream);
      }
      cudaGraph_t graph = nullptr;
      const cudaError_t e = cudaStreamEndCapture(c->capStream, &graph);
      if (e != cudaSuccess) return fail(c, DNDSG_CUDA_ERROR, std::string("step capture: ") + cudaGetErrorString(e));
      const cudaError_t e2 = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e2 != cudaSuccess) {
        g.exec = nullptr;
        return fail(c, DNDSG_CUDA_ERROR, std::string("step graph: ") + cudaGetErrorString(e2));
      }
      g.cfl = cfl;
      g.tEnd = t_end;
      g.urec = urec0;
    }
    for (int64_t k = 0; k < n / 2; k++) DG_CUDA(c, cudaGraphLaunch(g.exec, st(s)));
  }
  if (n & 1) {
    if (c->fp32) run_step<float>(c, cfl, t_end, st(s));
    else run_step<double>(c, cfl, t_end, st(s));
  }
  return check_launch(c);
}

// ---- partitioned runs: owned-cell mask, SSP-RK3 by stage, halo pack / unpack
int dndsg_set_owned(dndsg_ctx* c, const uint8_t* owned) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c))) return rc;
  // work queued earlier on any stream (a caller's non-blocking stream included) may still read the
  // mask or replay a step graph: let it finish before either changes
  DG_CUDA(c, cudaDeviceSynchronize());
  // the step graphs of dndsg_ssprk3_steps hold the mask pointer of their capture: recapture
  for (auto& g : c->stepGraph) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = dndsg_ctx::StepGraph{};
  }
  if (!owned) {
    c->owned = nullptr;
    return 0;
  }
  if (!c->ownedBuf && (rc = dalloc(c, c->ownedBuf, sizeof(uint8_t) * c->N))) return rc;
  DG_CUDA(c, cudaMemcpy(c->ownedBuf, owned, sizeof(uint8_t) * c->N, cudaMemcpyHostToDevice));
  c->owned = c->ownedBuf;
  return 0;
}

int dndsg_rk_dt(dndsg_ctx* c, double cfl, double* dt_min_out, void* s) {
  if (!c || !dt_min_out || !(cfl > 0)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "SA contexts run the implicit path");
  int rc;
  if ((rc = set_device(c))) return rc;
  if (c->fp32) run_dt<float>(c, cfl, 1e100, true, st(s));
  else run_dt<double>(c, cfl, 1e100, true, st(s));
  if ((rc = check_launch(c))) return rc;
  unsigned long long bits = 0;
  DG_CUDA(c, cudaMemcpyAsync(&bits, c->scal + S_DTMIN, sizeof(bits), cudaMemcpyDeviceToHost, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  std::memcpy(dt_min_out, &bits, sizeof(double));
  return 0;
}

int dndsg_rk_set_dt(dndsg_ctx* c, double dt, void* s) {
  if (!c || !(dt >= 0)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c))) return rc;
  DG_CUDA(c, cudaMemcpyAsync(c->scal + S_DT, &dt, sizeof(double), cudaMemcpyHostToDevice, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  return 0;
}

int dndsg_rk_vr(dndsg_ctx* c, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->fp32) run_vr<float>(c, false, st(s));
  else run_vr<double>(c, false, st(s));
  return check_launch(c);
}

int dndsg_rk_limit(dndsg_ctx* c, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (!c->s.limiter) return 0;
  if (c->fp32) run_limiter<float>(c, 0, st(s));
  else run_limiter<double>(c, 0, st(s));
  return check_launch(c);
}

int dndsg_rk_stage(dndsg_ctx* c, int stage, void* s) {
  if (!c || stage < 0 || stage > 2) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->fp32) run_rk_stage<float>(c, stage, st(s));
  else run_rk_stage<double>(c, stage, st(s));
  return check_launch(c);
}

int dndsg_rk_finish(dndsg_ctx* c, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  k_advance_time<<<1, 1, 0, st(s)>>>(c->scal);
  return check_launch(c);
}

int dndsg_halo_pack(dndsg_ctx* c, int what, const int32_t* cells, int64_t n, void* buf, void* s) {
  if (!c || (what != DNDSG_HALO_U && what != DNDSG_HALO_UREC) || n < 0 || (n && (!cells || !buf)))
    return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (n == 0) return 0;
  const int w = what == DNDSG_HALO_U ? 4 : 20;
  if (what == DNDSG_HALO_U)
    k_halo_copy<double, true><<<grid_for(n * w), kBlock, 0, st(s)>>>(c->u, cells, n, w, (double*)buf);
  else if (c->fp32)
    k_halo_copy<float, true><<<grid_for(n * w), kBlock, 0, st(s)>>>((float*)c->urec, cells, n, w, (float*)buf);
  else
    k_halo_copy<double, true><<<grid_for(n * w), kBlock, 0, st(s)>>>((double*)c->urec, cells, n, w, (double*)buf);
  return check_launch(c);
}

int dndsg_halo_unpack(dndsg_ctx* c, int what, const int32_t* cells, int64_t n, const void* buf, void* s) {
  if (!c || (what != DNDSG_HALO_U && what != DNDSG_HALO_UREC) || n < 0 || (n && (!cells || !buf)))
    return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (n == 0) return 0;
  const int w = what == DNDSG_HALO_U ? 4 : 20;
  if (what == DNDSG_HALO_U)
    k_halo_copy<double, false><<<grid_for(n * w), kBlock, 0, st(s)>>>(c->u, cells, n, w, (double*)buf);
  else if (c->fp32)
    k_halo_copy<float, false><<<grid_for(n * w), kBlock, 0, st(s)>>>((float*)c->urec, cells, n, w, (float*)buf);
  else
    k_halo_copy<double, false><<<grid_for(n * w), kBlock, 0, st(s)>>>((double*)c->urec, cells, n, w, (double*)buf);
  return check_launch(c);
}

int dndsg_residual(dndsg_ctx* c, int p, int vol_wise, double* out, void* s) {
  if (!c || !out) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  unsigned nb = grid_for(c->N);
  k_residual<<<nb, kBlock, 0, st(s)>>>(c->rhs, c->vol, c->N, p, vol_wise, c->partial, c->owned);
  int rc = check_launch(c);
  if (rc) return rc;
  std::vector<double> part(4 * (size_t)nb);
  DG_CUDA(c, cudaMemcpyAsync(part.data(), c->partial, sizeof(double) * 4 * nb, cudaMemcpyDeviceToHost, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  for (int v = 0; v < 4; v++) {
    double a = 0;
    for (unsigned b = 0; b < nb; b++) a = p < 3 ? a + part[4 * b + v] : std::max(a, part[4 * b + v]);
    out[v] = p < 3 ? std::pow(a, 1.0 / p) : a;
  }
  if (c->sa) {  // the U5 component (host reduction)
    std::vector<double> r(c->N), vol(c->N);
    DG_CUDA(c, cudaMemcpy(r.data(), c->saRhs, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
    DG_CUDA(c, cudaMemcpy(vol.data(), c->vol, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
    double a = 0;
    for (int64_t i = 0; i < c->N; i++) {
      const double x = std::fabs(r[i]);
      if (p < 3) a += std::pow(x, (double)p) * (vol_wise ? vol[i] : 1.0);
      else a = std::max(a, x);
    }
    out[4] = p < 3 ? std::pow(a, 1.0 / p) : a;
  }
  return 0;
}

int dndsg_face_values(dndsg_ctx* c, double t, double* out, void* s) {
  if (!c || !out) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "face values are reported for 4-variable contexts");
  double* d;
  size_t bytes = sizeof(double) * 24 * c->F;
  DG_CUDA(c, cudaMallocAsync((void**)&d, bytes, st(s)));
  if (c->fp32) k_face_values<float><<<grid_for(c->F), kBlock, 0, st(s)>>>(view<float>(c), t, d);
  else k_face_values<double><<<grid_for(c->F), kBlock, 0, st(s)>>>(view<double>(c), t, d);
  int rc = check_launch(c);
  if (rc) return rc;
  std::vector<double> tmp(24 * (size_t)c->F);
  DG_CUDA(c, cudaMemcpyAsync(tmp.data(), d, bytes, cudaMemcpyDeviceToHost, st(s)));
  DG_CUDA(c, cudaFreeAsync(d, st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  for (int64_t k = 0; k < c->F; k++) std::memcpy(out + 24 * c->facePerm[k], tmp.data() + 24 * k, 24 * sizeof(double));
  return 0;
}

int dndsg_get_status(dndsg_ctx* c, uint32_t* flags, uint64_t* n_reduced, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  unsigned f = 0;
  unsigned long long r = 0;
  DG_CUDA(c, cudaMemcpyAsync(&f, c->flags, sizeof(f), cudaMemcpyDeviceToHost, st(s)));
  DG_CUDA(c, cudaMemcpyAsync(&r, c->nreduced, sizeof(r), cudaMemcpyDeviceToHost, st(s)));
  DG_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(unsigned), st(s)));
  DG_CUDA(c, cudaMemsetAsync(c->nreduced, 0, sizeof(unsigned long long), st(s)));
  DG_CUDA(c, cudaStreamSynchronize(st(s)));
  if (flags) *flags = f;
  if (n_reduced) *n_reduced = r;
  if (f & kFlagTimeout) {
    c->dead = true;
    return fail(c, DNDSG_TIMEOUT, "a bounded wait in a kernel ran out (timeout flag); the context refuses further work");
  }
  return 0;
}

}  // extern "C"

// ====================================================================== allocation-free RHS
// Some callers cannot call cudaMalloc at the point where they need a residual:
// real-time loops where the implicit device synchronisation of cudaMalloc is
// not acceptable, host frameworks that own all device memory and forbid
// allocations after start-up, and code running inside another library's
// callback where allocating is not allowed.
// dndsg_eval_rhs_noalloc serves them: it allocates nothing and keeps its only
// scratch -- the per-face flux buffer between the face kernel and the cell
// gather -- in the file-scope array below, sized for at most
// DNDSG_NOALLOC_MAX_FACES faces (8 MiB; every GPU that loads this library holds
// it until the process exits).
namespace {
constexpr int64_t kNoAllocMaxFaces = DNDSG_NOALLOC_MAX_FACES;
static __device__ __align__(256) double g_noalloc_flux[kNoAllocMaxFaces * 4];
constexpr int kMaxDevices = 64;
double* g_noalloc_ptr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;

// Host code must not pass g_noalloc_flux itself to a kernel (on the host it is
// only a stand-in symbol); the device address comes from cudaGetSymbolAddress,
// once per device, with that device current.  The lookup is serialised, so two
// host threads making their first call on one device at the same time look it
// up once.  A device reset (cudaDeviceReset) invalidates the cached address;
// the library does not support calls after one.
int noalloc_scratch(dndsg_ctx* c, double** out) {
  if (c->device < 0 || c->device >= kMaxDevices) return fail(c, DNDSG_BAD_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[c->device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_flux);
    if (e != cudaSuccess)
      return fail(c, DNDSG_CUDA_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[c->device] = (double*)p;
  }
  *out = g_noalloc_ptr[c->device];
  return 0;
}

// the kernels of dndsg_eval_rhs (face fluxes, then the gather into rhs) over the caller's arrays,
// with the face fluxes in the scratch array
template <class T>
void run_rhs_noalloc(dndsg_ctx* c, const double* u, const void* urec, double* rhs, double* scratch, double t,
                     cudaStream_t s) {
  HotView<T> h = view<T>(c);
  h.u = const_cast<double*>(u);
  h.urec = (const T*)urec;
  h.rhs = rhs;
  h.flux = scratch;
  launch_flux_h<T>(c, h, 0, t, 0.0, s);
  k_cell_update<T, -1><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
}  // namespace

extern "C" int dndsg_eval_rhs_noalloc(dndsg_ctx* c, const double* u, const void* urec, double* rhs, double t,
                                      void* s) {
  if (c && (c->s.mu_gas > 0 || c->sa))
    return fail(c, DNDSG_UNSUPPORTED, "the allocation-free RHS covers the inviscid model only (mu_gas = 0)");
  if (!c || !u || !urec || !rhs) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  // the kernels read and write these arrays in 16-byte vectors
  if (!aligned16(u) || !aligned16(urec) || !aligned16(rhs))
    return fail(c, DNDSG_BAD_ARGUMENT, "dndsg_eval_rhs_noalloc: u, urec and rhs must be 16-byte aligned");
  if (c->F > kNoAllocMaxFaces)
    return fail(c, DNDSG_BAD_ARGUMENT,
                "dndsg_eval_rhs_noalloc: mesh has " + std::to_string(c->F) + " faces, more than its scratch limit of " +
                    std::to_string(kNoAllocMaxFaces));
  int rc = set_device(c);
  if (rc) return rc;
  double* scratch = nullptr;
  if ((rc = noalloc_scratch(c, &scratch))) return rc;
  if (c->fp32) run_rhs_noalloc<float>(c, u, urec, rhs, scratch, t, st(s));
  else run_rhs_noalloc<double>(c, u, urec, rhs, scratch, t, st(s));
  return check_launch(c);
}

// ====================================================================== learned VR warm start
struct dndsg_mlp {
  int device = 0;
  float *P = nullptr, *M = nullptr, *V = nullptr, *G = nullptr;
  __nv_bfloat16* W = nullptr;
  double* loss = nullptr;
  unsigned* flags = nullptr;  // kFlagTimeout from the tensor-core forward
  int64_t step = 0;
  bool attrFwd = false, attrTrain = false;
  int featureMode = 0;  // the feature design the network is trained for (dndsg_mlp_set_features)
  std::string err;
};

namespace {
int mfail(dndsg_mlp* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  return code;
}
#define DG_MCUDA(m, call)                                                                                 \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess) return mfail(m, DNDSG_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static_assert(kIn == DNDSG_MLP_IN && kOut == DNDSG_MLP_OUT && kNParam == DNDSG_MLP_NPARAM, "header constants");
MlpDev mlp_dev(const dndsg_mlp* m) { return MlpDev{m->P, m->W}; }

template <class T>
__global__ void k_mlp_features(HotView<T> h, MlpIters<T> it, int mode, float* X, float* Sc) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= h.N) return;
  float x[kInP], sc[4];
  if (mode == 0) mlp_cell_features<T>(i, h, it, x, sc);
  else mlp_cell_features_prev<T>(i, h, it.x0, it.geom, x, sc);
  if (X)
    for (int k = 0; k < kIn; k++) X[i * kIn + k] = x[k];
  for (int v = 0; v < 4; v++) Sc[i * 4 + v] = sc[v];
}

template <class T>
__global__ void k_mlp_target(int64_t n, const T* start, const T* conv, const float* Sc, float* Tg) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n * 20) return;
  const int64_t i = e / 20;
  const int v = (int)(e - i * 20) & 3;
  const double t = ((double)conv[e] - (double)start[e]) / (double)Sc[i * 4 + v];
  Tg[e] = (float)(t > 1e3 ? 1e3 : (t < -1e3 ? -1e3 : t));  // clamped like the features
}

// per cell: keep the sweep from the learned start where its Jacobi increment is the smaller one
template <class T>
__global__ void k_vr_gate(int64_t n, const T* x0, const T* y0, const T* xm, const T* ym, T* out, double* incAcc,
                          unsigned long long* accepted) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double inc = 0;
  int acc = 0;
  if (i < n) {
    double d0 = 0, dm = 0;
    for (int k = 0; k < 20; k++) {
      double a = (double)y0[i * 20 + k] - (double)x0[i * 20 + k], b = (double)ym[i * 20 + k] - (double)xm[i * 20 + k];
      d0 += a * a;
      dm += b * b;
    }
    acc = dm < d0;  // false for a NaN increment
    const T* src = acc ? ym : y0;
    for (int k = 0; k < 20; k++) out[i * 20 + k] = src[i * 20 + k];
    inc = acc ? dm : d0;
  }
  inc = warp_sum(inc);
  unsigned na = __popc(__ballot_sync(0xffffffffu, acc != 0));
  if ((threadIdx.x & 31) == 0) {
    if (inc != 0.0) atomicAdd(incAcc, inc);
    if (na) atomicAdd(accepted, (unsigned long long)na);
  }
}

__global__ void k_zero_scalar(double* p) { *p = 0.0; }

// one Jacobi sweep from src into dst (the kernels of run_vr); with inc the increment norm
// accumulates into scal[S_INC]
template <class T>
void launch_vr_from(dndsg_ctx* c, const void* src, void* dst, bool inc, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  h.urec = (const T*)src;
  h.urecNew = (T*)dst;
  const bool r1 = c->s.jacobi_relax == 1.0;
  if (inc) {
    if (r1) k_vr<T, true, true><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal + S_INC);
    else k_vr<T, false, true><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal + S_INC);
  } else if (r1) {
    constexpr int TILE = vr_tile<T>();
    const unsigned grid = (unsigned)((c->N + TILE - 1) / TILE);
    if (c->nfmax == 3) k_vr_tma4<T, TILE, 3><<<grid, TILE * 4, (size_t)TILE * 3 * 30 * sizeof(T), s>>>(h, c->flags);
    else k_vr_tma4<T, TILE, 4><<<grid, TILE * 4, (size_t)TILE * 4 * 30 * sizeof(T), s>>>(h, c->flags);
    if (c->nWallCells > 0) k_vr_wall_fixup<T><<<grid_for(4 * c->nWallCells), kBlock, 0, s>>>(h, c->wallCells, c->nWallCells);
  } else {
    k_vr<T, false, false><<<grid_for(c->N), kBlock, 0, s>>>(h, nullptr);
  }
}

int read_scalar(dndsg_ctx* c, const double* dsrc, double* out, cudaStream_t s) {
  DG_CUDA(c, cudaMemcpyAsync(out, dsrc, sizeof(double), cudaMemcpyDeviceToHost, s));
  DG_CUDA(c, cudaStreamSynchronize(s));
  return 0;
}

template <class T>
int ensure_mlp_buffers(dndsg_ctx* c) {
  if (c->mlpM) return 0;
  const size_t bytes = sizeof(T) * 20 * c->N;
  int rc;
  if ((rc = dalloc(c, c->mlpM, bytes)) || (rc = dalloc(c, c->mlpA, bytes)) || (rc = dalloc(c, c->mlpB, bytes)) ||
      (rc = dalloc(c, c->mlpH, bytes)) || (rc = dalloc(c, c->mlpSc, sizeof(float) * 4 * c->N)) ||
      (rc = dalloc(c, c->accCount, sizeof(unsigned long long))))
    return rc;
  DG_CUDA(c, cudaFuncSetAttribute(k_mlp_tc<TcCellFeatures<T, 0>, TcWarmStart<T>>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
  DG_CUDA(c, cudaFuncSetAttribute(k_mlp_tc<TcCellFeatures<T, 1>, TcWarmStart<T>>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
  return 0;
}

template <class T>
MlpIters<T> iters(dndsg_ctx* c, const void* x0, const void* x1, const void* x2) {
  return MlpIters<T>{(const T*)x0, (const T*)x1, (const T*)x2, c->mlpGeom};
}

// Jacobi sweeps until the rms coefficient increment sqrt(sum |dx|^2 / N) <= tol (or max_sweeps).
// With a network: two plain sweeps x0 -> x1 -> x2, the learned start xm from (x0, x1, x2), then
// J(x2) (the plain path's third sweep) and J(xm) gated per cell, then plain sweeps to tol.
// hX / hT (device, may be null) receive the features after the first two sweeps and the
// training targets (converged - x2) / r at the end (harvesting runs without a network).
template <class T>
int vr_to_tol(dndsg_ctx* c, const dndsg_mlp* m, double tol, int maxSweeps, int* sweepsOut, int64_t* accOut,
              float* hX, float* hT, cudaStream_t s) {
  int rc = 0, sweeps = 0;
  double inc = 0;
  const bool harvest = hX || hT;
  if (m && harvest) return fail(c, DNDSG_BAD_ARGUMENT, "harvesting runs without a network");
  if (accOut) *accOut = 0;
  auto converged = [&]() { return sweeps > 0 && std::sqrt(inc / double(c->N)) <= tol; };
  const int mode = c->mlpFeatureMode;
  if (m && m->featureMode != mode)
    return fail(c, DNDSG_BAD_ARGUMENT, "the network's feature design differs from the context's");
  if (mode == 1 && (m || harvest) && maxSweeps >= (m ? 2 : 1)) {
    // the configured input: features of the start x0 itself (neighbour mean differences, x0)
    if ((rc = ensure_mlp_buffers<T>(c))) return rc;
    k_mlp_features<T><<<grid_for(c->N), kBlock, 0, s>>>(view<T>(c), iters<T>(c, c->urec, nullptr, nullptr), 1, hX,
                                                         c->mlpSc);
    if ((rc = check_launch(c))) return rc;
    if (m) {
      DG_CUDA(c, cudaMemsetAsync(c->accCount, 0, sizeof(unsigned long long), s));
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
      const int64_t tiles = (c->N + kTcRows - 1) / kTcRows;
      k_mlp_tc<<<(unsigned)std::min<int64_t>(tiles, 4 * sms), kTcRows, sizeof(TcSmem), s>>>(
          mlp_dev(m), TcCellFeatures<T, 1>{view<T>(c), iters<T>(c, c->urec, nullptr, nullptr)},
          TcWarmStart<T>{(const T*)c->urec, (T*)c->mlpM}, c->N, c->flags);
      launch_vr_from<T>(c, c->urec, c->mlpA, false, s);  // J(x0)
      launch_vr_from<T>(c, c->mlpM, c->mlpH, false, s);  // J(xm)
      k_zero_scalar<<<1, 1, 0, s>>>(c->scal + S_INC);
      k_vr_gate<T><<<grid_for(c->N), kBlock, 0, s>>>(c->N, (const T*)c->urec, (const T*)c->mlpA,
                                                     (const T*)c->mlpM, (const T*)c->mlpH, (T*)c->mlpB,
                                                     c->scal + S_INC, c->accCount);
      std::swap(c->urec, c->mlpB);
      sweeps = 2;
      if ((rc = check_launch(c))) return rc;
      if (accOut) {
        unsigned long long a = 0;
        DG_CUDA(c, cudaMemcpyAsync(&a, c->accCount, sizeof(a), cudaMemcpyDeviceToHost, s));
        DG_CUDA(c, cudaStreamSynchronize(s));
        *accOut = (int64_t)a;
      }
      if ((rc = read_scalar(c, c->scal + S_INC, &inc, s))) return rc;
    } else if (hT) {
      DG_CUDA(c, cudaMemcpyAsync(c->mlpH, c->urec, sizeof(T) * 20 * c->N, cudaMemcpyDeviceToDevice, s));
    }
  } else if (mode == 0 && (m || harvest) && maxSweeps >= (m ? 4 : 2)) {
    if ((rc = ensure_mlp_buffers<T>(c))) return rc;
    // x1 = J(x0) into A, x2 = J(x1) into B (with its increment)
    launch_vr_from<T>(c, c->urec, c->mlpA, false, s);
    k_zero_scalar<<<1, 1, 0, s>>>(c->scal + S_INC);
    launch_vr_from<T>(c, c->mlpA, c->mlpB, true, s);
    sweeps = 2;
    k_mlp_features<T><<<grid_for(c->N), kBlock, 0, s>>>(view<T>(c), iters<T>(c, c->urec, c->mlpA, c->mlpB), 0, hX,
                                                         c->mlpSc);
    if ((rc = check_launch(c))) return rc;
    if (m) {
      DG_CUDA(c, cudaMemsetAsync(c->accCount, 0, sizeof(unsigned long long), s));
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
      const int64_t tiles = (c->N + kTcRows - 1) / kTcRows;
      k_mlp_tc<<<(unsigned)std::min<int64_t>(tiles, 4 * sms), kTcRows, sizeof(TcSmem), s>>>(
          mlp_dev(m), TcCellFeatures<T, 0>{view<T>(c), iters<T>(c, c->urec, c->mlpA, c->mlpB)},
          TcWarmStart<T>{(const T*)c->mlpB, (T*)c->mlpM}, c->N, c->flags);
      launch_vr_from<T>(c, c->mlpB, c->urecNew, false, s);  // J(x2)
      launch_vr_from<T>(c, c->mlpM, c->mlpH, false, s);     // J(xm)
      k_zero_scalar<<<1, 1, 0, s>>>(c->scal + S_INC);
      k_vr_gate<T><<<grid_for(c->N), kBlock, 0, s>>>(c->N, (const T*)c->mlpB, (const T*)c->urecNew,
                                                     (const T*)c->mlpM, (const T*)c->mlpH, (T*)c->mlpA,
                                                     c->scal + S_INC, c->accCount);
      std::swap(c->urec, c->mlpA);
      sweeps = 4;
      if ((rc = check_launch(c))) return rc;
      if (accOut) {
        unsigned long long a = 0;
        DG_CUDA(c, cudaMemcpyAsync(&a, c->accCount, sizeof(a), cudaMemcpyDeviceToHost, s));
        DG_CUDA(c, cudaStreamSynchronize(s));
        *accOut = (int64_t)a;
      }
    } else {
      if (hT) DG_CUDA(c, cudaMemcpyAsync(c->mlpH, c->mlpB, sizeof(T) * 20 * c->N, cudaMemcpyDeviceToDevice, s));
      std::swap(c->urec, c->mlpB);
    }
    if ((rc = read_scalar(c, c->scal + S_INC, &inc, s))) return rc;
  }
  while (sweeps < maxSweeps && !converged()) {
    k_zero_scalar<<<1, 1, 0, s>>>(c->scal + S_INC);
    launch_vr_from<T>(c, c->urec, c->urecNew, true, s);
    std::swap(c->urec, c->urecNew);
    if ((rc = check_launch(c))) return rc;
    sweeps++;
    if ((rc = read_scalar(c, c->scal + S_INC, &inc, s))) return rc;
  }
  if (hT && c->mlpH) {
    const int64_t n20 = c->N * 20;
    k_mlp_target<T><<<(unsigned)((n20 + kBlock - 1) / kBlock), kBlock, 0, s>>>(c->N, (const T*)c->mlpH,
                                                                               (const T*)c->urec, c->mlpSc, hT);
    if ((rc = check_launch(c))) return rc;
  }
  if (sweepsOut) *sweepsOut = sweeps;
  return 0;
}

template <class T>
int run_step_tol(dndsg_ctx* c, const dndsg_mlp* m, double cfl, double tEnd, double tol, int maxSweeps,
                 int* sweepsOut, float* hX, float* hT, cudaStream_t s) {
  run_dt<T>(c, cfl, 1e100, true, s);
  k_dt_finalize<<<1, 1, 0, s>>>(c->scal, tEnd);
  const double cst[3] = {0.0, 1.0, 0.5};
  int total = 0, rc = 0;
  const size_t xs = (size_t)c->N * kIn, ts = (size_t)c->N * 20;
  for (int stg = 0; stg < 3; stg++) {
    int sw = 0;
    if ((rc = vr_to_tol<T>(c, m, tol, maxSweeps, &sw, nullptr, hX ? hX + stg * xs : nullptr,
                           hT ? hT + stg * ts : nullptr, s)))
      return rc;
    total += sw;
    if (c->s.limiter) run_limiter<T>(c, 0, s);
    launch_flux<T>(c, 1, 0.0, cst[stg], s);
    HotView<T> h = view<T>(c);
    if (stg == 0) k_cell_update<T, 0><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
    else if (stg == 1) k_cell_update<T, 1><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
    else k_cell_update<T, 2><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
  }
  k_advance_time<<<1, 1, 0, s>>>(c->scal);
  if (sweepsOut) *sweepsOut = total;
  return check_launch(c);
}
}  // namespace

extern "C" {

int dndsg_mlp_set_params(dndsg_mlp* m, const float* params) {
  if (!m || !params) return DNDSG_BAD_ARGUMENT;
  DG_MCUDA(m, cudaSetDevice(m->device));
  DG_MCUDA(m, cudaMemcpy(m->P, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice));
  DG_MCUDA(m, cudaMemset(m->M, 0, sizeof(float) * kNParam));
  DG_MCUDA(m, cudaMemset(m->V, 0, sizeof(float) * kNParam));
  k_mlp_to_bf16<<<(kNParam + 255) / 256, 256>>>(m->P, m->W);
  DG_MCUDA(m, cudaGetLastError());
  DG_MCUDA(m, cudaDeviceSynchronize());
  m->step = 0;
  return 0;
}

int dndsg_mlp_create(int device, uint64_t seed, dndsg_mlp** out) {
  if (!out) return DNDSG_BAD_ARGUMENT;
  *out = nullptr;
  dndsg_mlp* m = new dndsg_mlp();
  m->device = device;
  auto bail = [&](int code) { dndsg_mlp_destroy(m); return code; };
  if (cudaSetDevice(device) != cudaSuccess) return bail(DNDSG_CUDA_ERROR);
  if (cudaMalloc(&m->P, sizeof(float) * kNParam) != cudaSuccess ||
      cudaMalloc(&m->M, sizeof(float) * kNParam) != cudaSuccess ||
      cudaMalloc(&m->V, sizeof(float) * kNParam) != cudaSuccess ||
      cudaMalloc(&m->G, sizeof(float) * kNParam) != cudaSuccess ||
      cudaMalloc(&m->W, sizeof(__nv_bfloat16) * kNW) != cudaSuccess || cudaMalloc(&m->loss, sizeof(double)) != cudaSuccess ||
      cudaMalloc(&m->flags, sizeof(unsigned)) != cudaSuccess || cudaMemset(m->flags, 0, sizeof(unsigned)) != cudaSuccess)
    return bail(DNDSG_CUDA_ERROR);
  // Glorot-uniform weights from a 64-bit LCG, zero biases and padding
  std::vector<float> p(kNParam, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int rows, int ld, int rowsReal, int colsReal) {
    const double a = std::sqrt(6.0 / (colsReal + rowsReal));
    for (int n = 0; n < rows; n++)
      for (int k = 0; k < ld; k++) p[off + n * ld + k] = (n < rowsReal && k < colsReal) ? (float)((2 * uni() - 1) * a) : 0.f;
  };
  fill(kOffW1, kHid, kInP, kHid, kIn);
  fill(kOffW2, kHid, kHid, kHid, kHid);
  fill(kOffW3, kHid, kHid, kHid, kHid);
  fill(kOffW4, kOutP, kHid, kOut, kHid);
  int rc = dndsg_mlp_set_params(m, p.data());
  if (rc) return bail(rc);
  *out = m;
  return 0;
}

void dndsg_mlp_destroy(dndsg_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  for (void* q : {(void*)m->P, (void*)m->M, (void*)m->V, (void*)m->G, (void*)m->W, (void*)m->loss, (void*)m->flags})
    if (q) cudaFree(q);
  delete m;
}

const char* dndsg_mlp_last_error(dndsg_mlp* m) { return m ? m->err.c_str() : "null network"; }

int dndsg_mlp_get_params(dndsg_mlp* m, float* params) {
  if (!m || !params) return DNDSG_BAD_ARGUMENT;
  DG_MCUDA(m, cudaSetDevice(m->device));
  DG_MCUDA(m, cudaMemcpy(params, m->P, sizeof(float) * kNParam, cudaMemcpyDeviceToHost));
  return 0;
}

int dndsg_mlp_forward(dndsg_mlp* m, const float* X, int64_t n, float* Y, void* s) {
  if (!m || !X || !Y || n < 0) return DNDSG_BAD_ARGUMENT;
  DG_MCUDA(m, cudaSetDevice(m->device));
  if (!m->attrFwd) {
    DG_MCUDA(m, cudaFuncSetAttribute(k_mlp_tc<TcFeaturesX, TcOutY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(TcSmem)));
    m->attrFwd = true;
  }
  if (n == 0) return 0;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  k_mlp_tc<<<(unsigned)std::min<int64_t>(tiles, 4 * sms), kTcRows, sizeof(TcSmem), st(s)>>>(
      mlp_dev(m), TcFeaturesX{X}, TcOutY{Y}, n, m->flags);
  DG_MCUDA(m, cudaGetLastError());
  unsigned f = 0;  // a tensor-core completion that timed out (the bounded wait ran out)
  DG_MCUDA(m, cudaMemcpyAsync(&f, m->flags, sizeof(f), cudaMemcpyDeviceToHost, st(s)));
  DG_MCUDA(m, cudaStreamSynchronize(st(s)));
  if (f) return mfail(m, DNDSG_TIMEOUT, "tensor-core completion wait timed out");
  return 0;
}

}  // extern "C"

namespace {
int mlp_grad(dndsg_mlp* m, const float* X, const float* Tg, int64_t n, cudaStream_t s) {
  if (!m->attrTrain) {
    DG_MCUDA(m, cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(TrTcSmem)));
    m->attrTrain = true;
  }
  DG_MCUDA(m, cudaMemsetAsync(m->G, 0, sizeof(float) * kNParam, s));
  DG_MCUDA(m, cudaMemsetAsync(m->loss, 0, sizeof(double), s));
  if (n == 0) return 0;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, sms));  // one CTA per SM
  k_mlp_train_tc<<<grid, kTrThreads, sizeof(TrTcSmem), s>>>(mlp_dev(m), X, Tg, n, 1.0f / (float)(n * kOut), m->G,
                                                         m->loss, m->flags);
  DG_MCUDA(m, cudaGetLastError());
  return 0;
}
}  // namespace

extern "C" {

int dndsg_mlp_gradient(dndsg_mlp* m, const float* X, const float* Tg, int64_t n, double* loss, float* grad, void* s) {
  if (!m || !X || !Tg || n <= 0) return DNDSG_BAD_ARGUMENT;
  DG_MCUDA(m, cudaSetDevice(m->device));
  int rc = mlp_grad(m, X, Tg, n, st(s));
  if (rc) return rc;
  double l = 0;
  DG_MCUDA(m, cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st(s)));
  if (grad) DG_MCUDA(m, cudaMemcpyAsync(grad, m->G, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, st(s)));
  unsigned f = 0;
  DG_MCUDA(m, cudaMemcpyAsync(&f, m->flags, sizeof(f), cudaMemcpyDeviceToHost, st(s)));
  DG_MCUDA(m, cudaStreamSynchronize(st(s)));
  if (f) return mfail(m, DNDSG_TIMEOUT, "tensor-core completion wait timed out");
  if (loss) *loss = l / (double)(n * kOut);
  return 0;
}

int dndsg_mlp_train_step(dndsg_mlp* m, const float* X, const float* Tg, int64_t n, float lr, double* loss, void* s) {
  if (!m || !X || !Tg || n <= 0 || !(lr > 0)) return DNDSG_BAD_ARGUMENT;
  DG_MCUDA(m, cudaSetDevice(m->device));
  int rc = mlp_grad(m, X, Tg, n, st(s));
  if (rc) return rc;
  m->step++;
  const double b1 = 0.9, b2 = 0.999;
  const float c1 = (float)(1.0 / (1.0 - std::pow(b1, (double)m->step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow(b2, (double)m->step)));
  k_mlp_adam<<<(kNParam + 255) / 256, 256, 0, st(s)>>>(m->P, m->M, m->V, m->G, m->W, lr, (float)b1, (float)b2, 1e-8f,
                                                        c1, c2);
  DG_MCUDA(m, cudaGetLastError());
  if (loss) {
    double l = 0;
    DG_MCUDA(m, cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st(s)));
    DG_MCUDA(m, cudaStreamSynchronize(st(s)));
    *loss = l / (double)(n * kOut);
  }
  return 0;
}

int dndsg_mlp_set_features(dndsg_mlp* m, int mode) {
  if (!m || (mode != 0 && mode != 1)) return DNDSG_BAD_ARGUMENT;
  m->featureMode = mode;
  return 0;
}

int dndsg_set_warm_start_features(dndsg_ctx* c, int mode) {
  if (!c || (mode != 0 && mode != 1)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  c->mlpFeatureMode = mode;
  return 0;
}

int dndsg_mlp_features(dndsg_ctx* c, float* X, float* scales, void* s) {
  if (!c || !X || !scales) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "the learned warm start is for 4-variable contexts");
  int rc = c->fp32 ? ensure_mlp_buffers<float>(c) : ensure_mlp_buffers<double>(c);
  if (rc) return rc;
  // design 1: the features of the current coefficients themselves
  if (c->mlpFeatureMode == 1) {
    if (c->fp32)
      k_mlp_features<float><<<grid_for(c->N), kBlock, 0, st(s)>>>(
          view<float>(c), iters<float>(c, c->urec, nullptr, nullptr), 1, X, scales);
    else
      k_mlp_features<double><<<grid_for(c->N), kBlock, 0, st(s)>>>(
          view<double>(c), iters<double>(c, c->urec, nullptr, nullptr), 1, X, scales);
    return check_launch(c);
  }
  // x1 = J(x0), x2 = J(x1) into work buffers; the context's coefficients are left as they are
  if (c->fp32) {
    launch_vr_from<float>(c, c->urec, c->mlpA, false, st(s));
    launch_vr_from<float>(c, c->mlpA, c->mlpB, false, st(s));
    k_mlp_features<float><<<grid_for(c->N), kBlock, 0, st(s)>>>(view<float>(c), iters<float>(c, c->urec, c->mlpA, c->mlpB),
                                                                 0, X, scales);
  } else {
    launch_vr_from<double>(c, c->urec, c->mlpA, false, st(s));
    launch_vr_from<double>(c, c->mlpA, c->mlpB, false, st(s));
    k_mlp_features<double><<<grid_for(c->N), kBlock, 0, st(s)>>>(view<double>(c),
                                                                  iters<double>(c, c->urec, c->mlpA, c->mlpB), 0, X, scales);
  }
  return check_launch(c);
}

int dndsg_vr_to_tolerance(dndsg_ctx* c, const dndsg_mlp* m, double tol, int max_sweeps, int* sweeps_out,
                          int64_t* accepted_out, float* harvest_x, float* harvest_t, void* s) {
  if (!c || max_sweeps < 1 || !(tol >= 0)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "the learned warm start is for 4-variable contexts");
  if (m && m->device != c->device) return fail(c, DNDSG_BAD_ARGUMENT, "network and context on different devices");
  int rc = c->fp32 ? vr_to_tol<float>(c, m, tol, max_sweeps, sweeps_out, accepted_out, harvest_x, harvest_t, st(s))
                   : vr_to_tol<double>(c, m, tol, max_sweeps, sweeps_out, accepted_out, harvest_x, harvest_t, st(s));
  return rc ? rc : observe_timeout(c, st(s));
}

int dndsg_ssprk3_step_tol(dndsg_ctx* c, const dndsg_mlp* m, double cfl, double t_end, double tol, int max_sweeps,
                          int* sweeps_out, float* harvest_x, float* harvest_t, void* s) {
  if (!c || max_sweeps < 1 || !(tol >= 0)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "the learned warm start is for 4-variable contexts");
  if (m && m->device != c->device) return fail(c, DNDSG_BAD_ARGUMENT, "network and context on different devices");
  int rc = c->fp32 ? run_step_tol<float>(c, m, cfl, t_end, tol, max_sweeps, sweeps_out, harvest_x, harvest_t, st(s))
                   : run_step_tol<double>(c, m, cfl, t_end, tol, max_sweeps, sweeps_out, harvest_x, harvest_t, st(s));
  return rc ? rc : observe_timeout(c, st(s));
}

}  // extern "C"

// ====================================================================== implicit path (LU-SGS, BDF1)
namespace {

// fluxJacobian0_Right_Times_du (DNDS_FV_EulerEvaluator.hpp:928-956) for 2-D Euler:
// the inviscid flux increment of dU about U through the unit normal n
// (IdealGasUIncrement, GasInviscidFluxFacialIncrement, DNDS_Gas.hpp:122-146) minus lam dU
__device__ __forceinline__ void flux_jac_times_du(const double U[4], double nx, double ny, const double dU[4],
                                                  double lam, double gamma, double dF[4]) {
  const double ir = 1.0 / U[0];
  const double vx = U[1] * ir, vy = U[2] * ir;
  const double p = (gamma - 1) * (U[3] - 0.5 * U[0] * (vx * vx + vy * vy));
  const double dvx = (dU[1] - vx * dU[0]) * ir, dvy = (dU[2] - vy * dU[0]) * ir;
  const double dp = (gamma - 1) * (dU[3] - 0.5 * (dU[1] * vx + dU[2] * vy + U[1] * dvx + U[2] * dvy));
  const double vn = vx * nx + vy * ny, dvn = dvx * nx + dvy * ny;
  dF[0] = dU[1] * nx + dU[2] * ny - lam * dU[0];
  dF[1] = dU[1] * vn + U[1] * dvn + nx * dp - lam * dU[1];
  dF[2] = dU[2] * vn + U[2] * dvn + ny * dp - lam * dU[2];
  dF[3] = (dU[3] + dp) * vn + (U[3] + p) * dvn - lam * dU[3];
}

// LUSGSMatrixInit (DNDS_FV_EulerEvaluator.cpp:995-1047), no source term: the diagonal is one
// scalar per cell, D_i = alpha/dt_i + 1/dtPhys + sum_f (alpha/2) lambda_f A_f / V_i, where dt_i is
// the EvaluateDt step (dTau = dt_i / alpha) and lamA holds lambda_f A_f
template <class T>
__global__ void __launch_bounds__(kBlock) k_lusgs_init(HotView<T> h, double dtPhysInv, double alpha, double* Dinv,
                                                       double* D) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= h.N) return;
  double sum = 0;
  for (int k = 0; k < h.nfmax; k++) {
    const int32_t sf = h.cellFace[aos(i, k, h.nfmax)];
    if (sf == kEmptySlot) continue;
    sum += h.lamA[sf >= 0 ? sf : ~sf];
  }
  const double d = alpha / h.dt[i] + dtPhysInv + 0.5 * alpha * sum / h.vol[i];
  Dinv[i] = 1.0 / d;
  D[i] = d;
}

// rhs of the first-order BDF pseudo-time system (ImplicitBDFDualTimeStep::Step,
// DNDS_ODE.hpp:455-465): alpha R(u) - (u - uLast) / dtPhys, in place on rhs
__global__ void k_bdf_rhs(int64_t n4, const double* u, const double* uLast, double alpha, double dtPhysInv,
                          double* rhs) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n4) return;
  rhs[e] = alpha * rhs[e] - u[e] * dtPhysInv + uLast[e] * dtPhysInv;
}

// one batch of UpdateLUSGSForward (FWD) or UpdateLUSGSBackward (DNDS_FV_EulerEvaluator.cpp:
// 1149-1357): a neighbour j is "before" cell i when rank[j] < rank[i].  With rank = colour and
// one batch per colour this is the reference's sweep in the colour-sorted scan order; with
// rank = scan position and one batch per dependency level it is the reference's sequential
// sweep in that scan order, level by level.  No two cells of a batch are neighbours and every
// neighbour a cell reads was finished in an earlier batch, so the result does not depend on the
// order within a batch.  inc is updated in place, as the reference calls both sweeps.
template <class T, bool FWD>
__device__ __forceinline__ void lusgs_cell(const HotView<T>& h, const int32_t* rankOf, int64_t i, double alpha,
                                           const double* Dinv, const double* rhs, double* inc) {
  const int ci = rankOf[i];
  double buf[4];
  if (FWD) load4<T>(&rhs[i * 4], buf);
  else buf[0] = buf[1] = buf[2] = buf[3] = 0.0;
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
    const double area = h.faceArea[f];
    double U[4], dU[4], dF[4];
    load4<T>(&h.u[(int64_t)j * 4], U);
    load4<T>(&inc[(int64_t)j * 4], dU);
    flux_jac_times_du(U, sg * h.faceNormal[2 * f], sg * h.faceNormal[2 * f + 1], dU, h.lamA[f] / area, h.gamma, dF);
    for (int v = 0; v < 4; v++) buf[v] += scale * area * dF[v];
  }
  const double di = Dinv[i];
  double* o = &inc[i * 4];
  if (FWD) {
    for (int v = 0; v < 4; v++) o[v] = di * buf[v];
  } else {
    for (int v = 0; v < 4; v++) o[v] += di * buf[v];
  }
}

template <class T, bool FWD>
__global__ void __launch_bounds__(kBlock) k_lusgs_batch(HotView<T> h, const int32_t* rankOf,
                                                        const int32_t* cells, int64_t n, double alpha,
                                                        const double* Dinv, const double* rhs, double* inc) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) lusgs_cell<T, FWD>(h, rankOf, cells[t], alpha, Dinv, rhs, inc);
}

// the parts of one LU-SGS cell update that do not depend on the increments of earlier cells
struct LusgsPre {
  int64_t i;
  bool use[4];  // slot k holds a neighbour that enters this sweep (static slot index: registers)
  int32_t j[4];
  double U[4][4], nx[4], ny[4], lam[4], w[4];
  double base[4], di;
};

// everything of the cell at schedule position t that does not depend on this sweep's increments.
// nbF / nbJ [t][4] hold, per face slot, the slot's face (cellFace encoding) and the neighbour when
// that neighbour enters this sweep (-1 otherwise), so every load here is independent of the others
template <class T, bool FWD>
__device__ __forceinline__ void lusgs_prefetch(const HotView<T>& h, const int32_t* cells, const int32_t* nbF,
                                               const int32_t* nbJ, int64_t t, double alpha, const double* Dinv,
                                               const double* rhs, LusgsPre& p) {
  const int64_t i = cells[t];
  const int4 sf4 = reinterpret_cast<const int4*>(nbF)[t];
  const int4 j4 = reinterpret_cast<const int4*>(nbJ)[t];
  const int32_t sfa[4] = {sf4.x, sf4.y, sf4.z, sf4.w}, ja[4] = {j4.x, j4.y, j4.z, j4.w};
  p.i = i;
  if (FWD) load4<T>(&rhs[i * 4], p.base);
  p.di = Dinv[i];
  const double scale = -0.5 * alpha / h.vol[i];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const bool use = ja[k] >= 0;
    const int32_t sf = sfa[k];
    const int32_t f = use ? (sf >= 0 ? sf : ~sf) : 0;   // index 0 is a valid face: loads stay unconditional
    const int64_t j = use ? ja[k] : i;
    const double sg = sf >= 0 ? 1.0 : -1.0;
    const double area = h.faceArea[f];
    p.use[k] = use;
    p.j[k] = (int32_t)j;
    load4<T>(&h.u[j * 4], p.U[k]);
    p.nx[k] = sg * h.faceNormal[2 * f];
    p.ny[k] = sg * h.faceNormal[2 * f + 1];
    p.lam[k] = h.lamA[f] / area;
    p.w[k] = scale * area;
  }
}

constexpr int kRecMaxLevels = 4095;  // level offsets of one sweep held in shared memory

// ---- scan-order sweep over precomputed neighbour records.
// The neighbour term of UpdateLUSGSForward/Backward, w_q (dF(U_q; n_q, dU_q) - lam_q dU_q)
// (fluxJacobian0_Right_Times_du, DNDS_FV_EulerEvaluator.hpp:928-956), is linear in the neighbour's
// increment dU_q, and everything else in it is fixed during the sweep.  So one parallel pass writes,
// per schedule position, the dU-independent quantities of its up to 4 neighbour terms, and the
// sequential level walk is left with a short product per neighbour over increments that mostly sit
// in a shared-memory ring.  With a = nx dU1 + ny dU2 - vn dU0 (= rho dvn) and
// dp = (gamma - 1)(dU3 - vx dU1 - vy dU2 + kq dU0), kq = |v|^2 / 2:
//   dF = (nx dU1 + ny dU2, vn dU1 + vx a + nx dp, vn dU2 + vy a + ny dp, H a + vn (dU3 + dp)),
// the term is w dF - wl dU (wl = w lam), and the U5 row of an SA context adds c a + (w vn - wl) dU5
// with c = w nuTilde_q / rho_q.  Ten doubles per neighbour instead of the 4x4 matrix (16, plus 4 for
// the U5 row): the walk moves every record through one SM's shared memory, and record bytes are
// what its levels wait on.  Fields are grouped in 16-byte pairs and read as such.
struct __align__(16) LuSlot {
  double vx, vy, vn, H, kq, wl, nx, ny, w, c;
};
struct __align__(16) LuMatF {
  LuSlot s[4];      // per face slot
  double x0[4];     // forward: the BDF rhs, where the sum starts; backward: the forward increment, added to di * sum
  double di;
  int32_t i, nu;    // cell; number of neighbours that enter this sweep, in s / j / p [0, nu) in face-slot order
  int32_t j[4];     // neighbour cell
  int32_t p[4];     // neighbour schedule position in this sweep (-1: not in the ring; read global memory)
};
struct __align__(16) LuMatS {
  LuMatF f;
  double x0S, diS;  // the U5 part of x0 and di
  double pad[2];    // 432-B stride: 16-byte loads of 32 consecutive records hit every bank evenly
};
static_assert(sizeof(LuMatF) == 400 && sizeof(LuMatS) == 432, "records are bulk-copied in 16-byte units");
template <bool SA>
using LuMat = typename std::conditional<SA, LuMatS, LuMatF>::type;
__device__ __forceinline__ LuMatF& mat_flow(LuMatF& r) { return r; }
__device__ __forceinline__ LuMatF& mat_flow(LuMatS& r) { return r.f; }
__device__ __forceinline__ const LuMatF& mat_flow(const LuMatF& r) { return r; }
__device__ __forceinline__ const LuMatF& mat_flow(const LuMatS& r) { return r.f; }

// the neighbour term w dF - wl dU of one record slot (fields as in LuSlot) added to buf, and its U5
// row c a + (w vn - wl) dS added to bufS when SA
template <bool SA>
__device__ __forceinline__ void lu_term(double vx, double vy, double vn, double H, double kq, double wl, double nx,
                                        double ny, double w, double c, const double d[4], double dS, double g1,
                                        double buf[4], double& bufS) {
  const double dmn = nx * d[1] + ny * d[2];
  const double a = dmn - vn * d[0];
  const double dp = g1 * (d[3] - vx * d[1] - vy * d[2] + kq * d[0]);
  const double dF[4] = {dmn, vn * d[1] + vx * a + nx * dp, vn * d[2] + vy * a + ny * dp, H * a + vn * (d[3] + dp)};
  for (int v = 0; v < 4; v++) buf[v] += w * dF[v] - wl * d[v];
  if constexpr (SA) bufS += c * a + (w * vn - wl) * dS;
}

// writes the record of every schedule position of one sweep, all positions in parallel.  In a
// partitioned backward sweep a neighbour in another part (position kGhostPos) is a ghost: its
// increment is the one after the forward sweep, which is what inc holds while this kernel runs, so
// its term is summed here and folded into x0 (x0 = dU_fwd + di * ghost terms) instead of taking a
// slot of the walk
constexpr int32_t kGhostPos = -2;
template <class T, bool FWD, bool SA>
__global__ void __launch_bounds__(kBlock) k_lusgs_pack_mat(HotView<T> h, SaView<T> sa, const int32_t* cells,
                                                           const int32_t* nbF, const int32_t* nbJ, const int32_t* nbP,
                                                           int64_t n, double alpha, const double* Dinv,
                                                           const double* rhs, const double* inc, LuMat<SA>* rec) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  LusgsPre p;
  lusgs_prefetch<T, FWD>(h, cells, nbF, nbJ, t, alpha, Dinv, rhs, p);
  LuMatF& f = mat_flow(rec[t]);
  const int4 p4 = reinterpret_cast<const int4*>(nbP)[t];
  const int32_t pa[4] = {p4.x, p4.y, p4.z, p4.w};
  const double g1 = h.gamma - 1;
  int nu = 0;
  for (int k = 0; k < 4; k++) {  // the used slots first, in slot order (the order of lusgs_cell's sum)
    f.j[k] = p.i;
    f.p[k] = 0;
  }
  double ghost[4] = {0, 0, 0, 0}, ghostS = 0.0;
  bool anyGhost = false;
  for (int k = 0; k < 4; k++) {
    if (!p.use[k]) continue;
    const double* U = p.U[k];
    const double ir = 1.0 / U[0];
    const double vx = U[1] * ir, vy = U[2] * ir, q2 = vx * vx + vy * vy;
    const double pr = g1 * (U[3] - 0.5 * U[0] * q2);
    LuSlot q;
    q.vx = vx;
    q.vy = vy;
    q.vn = vx * p.nx[k] + vy * p.ny[k];
    q.H = (U[3] + pr) * ir;
    q.kq = 0.5 * q2;
    q.wl = p.w[k] * p.lam[k];
    q.nx = p.nx[k];
    q.ny = p.ny[k];
    q.w = p.w[k];
    q.c = SA ? p.w[k] * sa.u[p.j[k]] * ir : 0.0;
    if (!FWD && pa[k] == kGhostPos) {
      double d[4];
      load4<double>(&inc[(int64_t)p.j[k] * 4], d);
      lu_term<SA>(q.vx, q.vy, q.vn, q.H, q.kq, q.wl, q.nx, q.ny, q.w, q.c, d, SA ? sa.inc[p.j[k]] : 0.0, g1, ghost,
                  ghostS);
      anyGhost = true;
      continue;
    }
    f.s[nu] = q;
    f.j[nu] = p.j[k];
    f.p[nu] = pa[k];
    nu++;
  }
  for (int k = nu; k < 4; k++) f.s[k] = LuSlot{};
  double add[4] = {0, 0, 0, 0};
  if (!FWD) load4<double>(&inc[p.i * 4], add);
  if (anyGhost)
    for (int v = 0; v < 4; v++) add[v] += p.di * ghost[v];
  for (int v = 0; v < 4; v++) f.x0[v] = FWD ? p.base[v] : add[v];
  f.di = p.di;
  f.i = (int32_t)p.i;
  f.nu = nu;
  if constexpr (SA) {
    LuMatS& r = rec[t];
    const double diS = sa.Dinv[p.i];
    r.diS = diS;
    r.x0S = FWD ? sa.rhs[p.i] : sa.inc[p.i] + (anyGhost ? diS * ghostS : 0.0);
    r.pad[0] = r.pad[1] = 0.0;
  }
}

constexpr int kRecBlock = 128;  // threads of the level walk, and records buffered per level
constexpr int kMatRing = 256;   // (a power of 2) increments of the most recent schedule positions kept in shared memory
constexpr int kRecStages = 2;   // levels of records in flight: the current one and the next (3 measured no faster)
constexpr uint32_t kBulkChunk = 16384;
template <bool SA>
constexpr size_t mat_smem() {
  return 32 + sizeof(int32_t) * (kRecMaxLevels + 1) + sizeof(double) * kMatRing * (SA ? 5 : 4) +
         sizeof(LuMat<SA>) * kRecStages * kRecBlock;
}
static_assert(mat_smem<true>() <= 227 * 1024, "level walk fits the shared memory of one block");

// one position of the level walk.  A neighbour's increment comes from the ring when the record
// gives its position (the schedule set that up: written there by this walk and not yet
// overwritten), else (position -1) from global memory.  The sum runs over the slots in the order
// of lusgs_cell.
__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
// the ring holds 32 B per position, two 16-B halves; the halves of every other group of four
// positions are swapped, so 16-B accesses by 32 consecutive positions spread over all banks
__device__ __forceinline__ double2* ring_half(double* ringF, int32_t pos, int h) {
  const int r = pos & (kMatRing - 1);
  return reinterpret_cast<double2*>(ringF + 4 * r + 2 * (h ^ ((r >> 2) & 1)));
}
template <bool FWD, bool SA, class T>
__device__ __forceinline__ void lusgs_mat_cell(const SaView<T>& sa, const LuMat<SA>& r, int32_t t, double* ringF,
                                               double* ringS, double* inc, double g1) {
  const LuMatF& f = mat_flow(r);
  const double2 x01 = ld2(&f.x0[0]), x23 = ld2(&f.x0[2]);
  const double x0[4] = {x01.x, x01.y, x23.x, x23.y};
  double buf[4], bufS = 0.0, x0S = 0.0, diS = 0.0;
  for (int v = 0; v < 4; v++) buf[v] = FWD ? x0[v] : 0.0;
  if constexpr (SA) {
    const double2 sd = ld2(&r.x0S);
    x0S = sd.x;
    diS = sd.y;
    bufS = FWD ? x0S : 0.0;
  }
  const int4 p4 = *reinterpret_cast<const int4*>(f.p);
  const int32_t pa[4] = {p4.x, p4.y, p4.z, p4.w};
  const int nu = f.nu;
  // the neighbours' increments, all ring reads issued together (any position is a valid ring
  // slot; values past nu are never used); the rare neighbour outside the ring from global memory
  double dU[4][4], dS[4] = {0, 0, 0, 0};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double2 a = *ring_half(ringF, pa[q], 0), b = *ring_half(ringF, pa[q], 1);
    dU[q][0] = a.x; dU[q][1] = a.y; dU[q][2] = b.x; dU[q][3] = b.y;
    if constexpr (SA) dS[q] = ringS[pa[q] & (kMatRing - 1)];
  }
  if ((pa[0] | pa[1] | pa[2] | pa[3]) < 0) {
    const int4 j4 = *reinterpret_cast<const int4*>(f.j);
    const int32_t ja[4] = {j4.x, j4.y, j4.z, j4.w};
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < nu && pa[q] < 0) {
        load4<double>(&inc[(int64_t)ja[q] * 4], dU[q]);
        if constexpr (SA) dS[q] = sa.inc[ja[q]];
      }
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (q >= nu) break;
    const double* sl = &f.s[q].vx;
    const double2 vxy = ld2(sl), vnH = ld2(sl + 2), kwl = ld2(sl + 4), nxy = ld2(sl + 6), wc = ld2(sl + 8);
    lu_term<SA>(vxy.x, vxy.y, vnH.x, vnH.y, kwl.x, kwl.y, nxy.x, nxy.y, wc.x, wc.y, dU[q], dS[q], g1, buf, bufS);
  }
  double o[4];
  for (int v = 0; v < 4; v++) o[v] = FWD ? f.di * buf[v] : x0[v] + f.di * buf[v];
  double2* g = reinterpret_cast<double2*>(&inc[(int64_t)f.i * 4]);
  g[0] = *ring_half(ringF, t, 0) = make_double2(o[0], o[1]);
  g[1] = *ring_half(ringF, t, 1) = make_double2(o[2], o[3]);
  if constexpr (SA) {
    const double oS = FWD ? diS * bufS : x0S + diS * bufS;
    sa.inc[f.i] = oS;
    ringS[t & (kMatRing - 1)] = oS;
  }
}

// a whole level-scheduled sweep in one block, one thread per position and a producer warp.  The
// producer bulk-copies the next level's records (contiguous in schedule order) into the other half
// of a shared-memory double buffer on an mbarrier while the other warps finish the current level;
// the block barrier per level publishes the increments (global memory and the ring).  Positions of
// a level beyond kRecBlock read their records from global memory.  A bulk copy that does not land
// in time sets kFlagTimeout and ends the walk.  Partitioned sweeps (partLev non-null) launch one
// block per part, each walking its own levels (partLev[b] to partLev[b + 1] of off) with its own
// ring: the parts share no dependency inside a sweep, so the blocks never wait on one another.
template <bool SA>
constexpr int mat_threads() { return kRecBlock + 32; }
template <class T, bool FWD, bool SA>
__global__ void __launch_bounds__(mat_threads<SA>()) k_lusgs_levels_mat(SaView<T> sa, const LuMat<SA>* rec,
                                                                        const int64_t* off, int nlev,
                                                                        const int32_t* partLev, double* inc,
                                                                        double g1, unsigned* flags) {
  using R = LuMat<SA>;
  constexpr int NT = kRecBlock;
  extern __shared__ __align__(16) unsigned char smraw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smraw);
  int32_t* so = reinterpret_cast<int32_t*>(smraw + 32);
  double* ringF = reinterpret_cast<double*>(smraw + 32 + sizeof(int32_t) * (kRecMaxLevels + 1));
  double* ringS = ringF + 4 * kMatRing;
  R* buf = reinterpret_cast<R*>(ringS + (SA ? kMatRing : 0));
  const int tid = threadIdx.x;
  const bool producer = tid == NT;
  if (partLev) {  // one block per part: this part's levels
    const int32_t l0 = partLev[blockIdx.x];
    nlev = partLev[blockIdx.x + 1] - l0;
    off += l0;
  }
  for (int l = tid; l <= nlev; l += blockDim.x) so[l] = (int32_t)off[l];
  if (tid == 0) {
    for (int k = 0; k < kRecStages; k++) mbar_init(smem_u32(&bars[k]), 1);
    fence_mbar_init();
  }
  __syncthreads();
  // level l uses buffer and mbarrier l % kRecStages, in phase (l / kRecStages) & 1
  auto issue = [&](int l) {  // producer
    const int32_t b = so[l];
    const int32_t n = min(so[l + 1] - b, kRecBlock);
    const uint32_t bar = smem_u32(&bars[l % kRecStages]), bytes = (uint32_t)(n * sizeof(R));
    const uint32_t dst = smem_u32(buf + (l % kRecStages) * kRecBlock);
    const char* src = reinterpret_cast<const char*>(rec + b);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, bytes);
    for (uint32_t o = 0; o < bytes; o += kBulkChunk) bulk_g2s(dst + o, src + o, min(kBulkChunk, bytes - o), bar);
  };
  if (producer)
    for (int k = 0; k < kRecStages - 1 && k < nlev; k++) issue(k);
  int l = 0;
  bool failed = false;
  int32_t b = so[0], e = nlev > 0 ? so[1] : 0;
  for (; l < nlev; l++) {
    // the buffer of level l + kRecStages - 1 held level l - 1, finished at the last barrier
    if (producer && l + kRecStages - 1 < nlev) issue(l + kRecStages - 1);
    const int32_t e2 = so[min(l + 2, nlev)];  // the next level's end, read ahead
    const int stage = l % kRecStages;
    bool ok = true;
    if (tid < NT && b + tid < e) {
      ok = mbar_wait(smem_u32(&bars[stage]), (l / kRecStages) & 1, kWaitLimit);
      if (ok) {
        // the record from the shared buffer, as a shared-memory reference (ld.shared, not generic loads)
        lusgs_mat_cell<FWD, SA>(sa, buf[stage * kRecBlock + tid], b + tid, ringF, ringS, inc, g1);
        for (int32_t t = b + tid + kRecBlock; t < e; t += kRecBlock)
          lusgs_mat_cell<FWD, SA>(sa, rec[t], t, ringF, ringS, inc, g1);
      }
    }
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    b = e;
    e = e2;
  }
  if (failed && producer) {  // let the copies in flight (levels l to l + kRecStages - 1) land before the block exits
    atomicOr(flags, kFlagTimeout);
    for (int k = l; k < l + kRecStages && k < nlev; k++)
      mbar_wait(smem_u32(&bars[k % kRecStages]), (k / kRecStages) & 1, kWaitLimit);
  }
}

// a whole sweep of narrow batches (dependency levels) in one thread block: the levels run one
// after another with a block barrier between them, which makes a level's increments visible to
// the next; no grid-wide synchronisation and no waiting on flags
constexpr int kLevelBlock = 512;
template <class T, bool FWD>
__global__ void __launch_bounds__(kLevelBlock) k_lusgs_levels(HotView<T> h, const int32_t* rankOf,
                                                              const int32_t* cells, const int64_t* off, int nlev,
                                                              double alpha, const double* Dinv, const double* rhs,
                                                              double* inc) {
  for (int l = 0; l < nlev; l++) {
    const int64_t b = off[l], e = off[l + 1];
    for (int64_t t = b + threadIdx.x; t < e; t += blockDim.x) lusgs_cell<T, FWD>(h, rankOf, cells[t], alpha, Dinv, rhs, inc);
    __syncthreads();
  }
}

// x += inc, with the L1 norm of inc per variable (volume-weighted on request) into acc[4]
__global__ void __launch_bounds__(kBlock) k_add_inc(int64_t N, double* u, const double* inc, const double* vol,
                                                    int volWise, double* acc) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double a[4] = {0, 0, 0, 0};
  if (i < N) {
    const double w = volWise ? vol[i] : 1.0;
    for (int v = 0; v < 4; v++) {
      const double d = inc[i * 4 + v];
      u[i * 4 + v] += d;
      a[v] = fabs(d) * w;
    }
  }
  for (int v = 0; v < 4; v++) block_add(a[v], &acc[v]);
}

// the wall force: minus the sum of the Riemann fluxes of the Wall_Euler / Wall_NoSlip faces
// (fluxWallSum, DNDS_FV_EulerEvaluator.cpp:510-516), from the last flux evaluation
__global__ void __launch_bounds__(kBlock) k_wall_flux(int64_t Fi, int64_t F, const int32_t* faceBC,
                                                      const double* flux, double* acc) {
  const int64_t f = Fi + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double a[4] = {0, 0, 0, 0};
  if (f < F) {
    const int bc = faceBC[f];
    if (bc == BC_WALL_NOSLIP || bc == BC_WALL_EULER)
      for (int v = 0; v < 4; v++) a[v] = -flux[f * 4 + v];
  }
  for (int v = 0; v < 4; v++) {
    const double r = warp_sum(a[v]);
    if ((threadIdx.x & 31) == 0 && r != 0.0) atomicAdd(&acc[v], r);
  }
}

// cell adjacency over the interior faces (CSR), from the device face table
int lusgs_adjacency(dndsg_ctx* c, std::vector<int64_t>& deg, std::vector<int32_t>& adj) {
  const int64_t N = c->N, F = c->F;
  std::vector<int32_t> L(F), R(F);
  DG_CUDA(c, cudaMemcpy(L.data(), c->faceL, sizeof(int32_t) * F, cudaMemcpyDeviceToHost));
  DG_CUDA(c, cudaMemcpy(R.data(), c->faceR, sizeof(int32_t) * F, cudaMemcpyDeviceToHost));
  deg.assign(N + 1, 0);
  for (int64_t f = 0; f < F; f++)
    if (R[f] >= 0) { deg[L[f] + 1]++; deg[R[f] + 1]++; }
  for (int64_t i = 0; i < N; i++) deg[i + 1] += deg[i];
  adj.assign(deg[N], 0);
  std::vector<int64_t> fill(deg.begin(), deg.end() - 1);
  for (int64_t f = 0; f < F; f++)
    if (R[f] >= 0) { adj[fill[L[f]]++] = R[f]; adj[fill[R[f]]++] = L[f]; }
  return 0;
}

// cells grouped by key (0..nkey-1), in cell order within a group
void group_by(const std::vector<int32_t>& key, int nkey, std::vector<int32_t>& cells, std::vector<int64_t>& off) {
  const int64_t N = (int64_t)key.size();
  off.assign(nkey + 1, 0);
  for (int64_t i = 0; i < N; i++) off[key[i] + 1]++;
  for (int k = 0; k < nkey; k++) off[k + 1] += off[k];
  cells.assign(N, 0);
  std::vector<int64_t> pos(off.begin(), off.end() - 1);
  for (int64_t i = 0; i < N; i++) cells[pos[key[i]]++] = (int32_t)i;
}

int upload_schedule(dndsg_ctx* c, const std::vector<int32_t>& rank, const std::vector<int32_t>& fwd,
                    const std::vector<int32_t>& bwd) {
  const int64_t N = c->N;
  DG_CUDA(c, cudaMemcpy(c->rankOf, rank.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->fwdCells, fwd.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->bwdCells, bwd.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
  return 0;
}

// default schedule: greedy distance-1 colouring in cell order; forward runs the colours up,
// backward down
int ensure_lusgs(dndsg_ctx* c) {
  if (c->rankOf) return 0;
  const int64_t N = c->N;
  std::vector<int64_t> deg;
  std::vector<int32_t> adj;
  int rc;
  if ((rc = lusgs_adjacency(c, deg, adj))) return rc;
  std::vector<int32_t> col(N, -1);
  int ncol = 0;
  for (int64_t i = 0; i < N; i++) {
    uint64_t used = 0;
    for (int64_t k = deg[i]; k < deg[i + 1]; k++) {
      const int cj = col[adj[k]];
      if (cj >= 0 && cj < 64) used |= 1ull << cj;
    }
    int cc = 0;
    while (cc < 64 && (used >> cc & 1)) cc++;
    if (cc >= 64) return fail(c, DNDSG_SETUP_ERROR, "colouring needs more than 64 colours");
    col[i] = cc;
    ncol = std::max(ncol, cc + 1);
  }
  std::vector<int32_t> fwd, bwd;
  group_by(col, ncol, fwd, c->fwdOff);
  std::vector<int32_t> rev(N);
  for (int64_t i = 0; i < N; i++) rev[i] = ncol - 1 - col[i];
  group_by(rev, ncol, bwd, c->bwdOff);
  if ((rc = dalloc(c, c->rankOf, sizeof(int32_t) * N)) || (rc = dalloc(c, c->fwdCells, sizeof(int32_t) * N)) ||
      (rc = dalloc(c, c->bwdCells, sizeof(int32_t) * N)) || (rc = dalloc(c, c->Dinv, sizeof(double) * N)) ||
      (rc = dalloc(c, c->Dmat, sizeof(double) * N)) ||
      (rc = dalloc(c, c->inc, sizeof(double) * 4 * N)) || (rc = dalloc(c, c->resAcc, sizeof(double) * 16)))
    return rc;
  c->colourHost = col;
  c->lusgsOrder = 0;
  DG_CUDA(c, cudaMemset(c->inc, 0, sizeof(double) * 4 * N));
  return upload_schedule(c, col, fwd, bwd);
}

// the reference's sequential sweep in a given scan order, level-scheduled: the forward level of a
// cell is one more than the largest forward level of its neighbours earlier in the scan (the
// backward level likewise over the later ones), and each level is one batch.  With parts (the
// reference on several ranks, DNDS_FV_EulerEvaluator.cpp:1177-1181, 1313-1317) every part sweeps its
// own cells in the scan order: levels count only neighbours of the same part, the schedule holds
// part after part (each part's levels contiguous), and a neighbour in another part enters the
// backward sweep only, as a ghost (kGhostPos) with its post-forward increment
int set_scan_order(dndsg_ctx* c, const int64_t* scan2cell) {
  int rc;
  if ((rc = ensure_lusgs(c))) return rc;
  const int64_t N = c->N;
  std::vector<int32_t> pos(N, -1), order(N);
  for (int64_t s = 0; s < N; s++) {
    const int64_t i = scan2cell ? scan2cell[s] : s;
    if (i < 0 || i >= N || pos[i] >= 0) return fail(c, DNDSG_BAD_ARGUMENT, "scan order is not a permutation");
    pos[i] = (int32_t)s;
    order[s] = (int32_t)i;
  }
  if (scan2cell) c->scanHost.assign(scan2cell, scan2cell + N);
  else c->scanHost.clear();
  const int P = c->lusgsParts;
  std::vector<int32_t> part(N, 0);
  if (P > 1) part = c->lusgsPart;
  std::vector<int64_t> deg;
  std::vector<int32_t> adj;
  if ((rc = lusgs_adjacency(c, deg, adj))) return rc;
  std::vector<int32_t> lf(N, 0), lb(N, 0), nlf(P, 0), nlb(P, 0);
  for (int64_t s = 0; s < N; s++) {
    const int32_t i = order[s];
    int l = 0;
    for (int64_t k = deg[i]; k < deg[i + 1]; k++)
      if (pos[adj[k]] < s && part[adj[k]] == part[i]) l = std::max(l, lf[adj[k]] + 1);
    lf[i] = l;
    nlf[part[i]] = std::max(nlf[part[i]], l + 1);
  }
  for (int64_t s = N - 1; s >= 0; s--) {
    const int32_t i = order[s];
    int l = 0;
    for (int64_t k = deg[i]; k < deg[i + 1]; k++)
      if (pos[adj[k]] > s && part[adj[k]] == part[i]) l = std::max(l, lb[adj[k]] + 1);
    lb[i] = l;
    nlb[part[i]] = std::max(nlb[part[i]], l + 1);
  }
  // schedule keys: the part's first level plus the level within the part
  std::vector<int32_t> baseF(P + 1, 0), baseB(P + 1, 0);
  for (int p = 0; p < P; p++) {
    baseF[p + 1] = baseF[p] + nlf[p];
    baseB[p + 1] = baseB[p] + nlb[p];
  }
  const int fMax = *std::max_element(nlf.begin(), nlf.end()), bMax = *std::max_element(nlb.begin(), nlb.end());
  if (P > 1 && (std::max(fMax, bMax) > kRecMaxLevels || c->nfmax > 4))  // checked before anything changes
    return fail(c, DNDSG_UNSUPPORTED, "partitioned sweeps need at most 4 faces per cell and " +
                                          std::to_string(kRecMaxLevels) + " levels per part");
  c->fwdPartMax = fMax;
  c->bwdPartMax = bMax;
  const int nf = baseF[P], nb = baseB[P];
  for (int64_t i = 0; i < N; i++) {
    lf[i] += baseF[part[i]];
    lb[i] += baseB[part[i]];
  }
  std::vector<int32_t> fwd, bwd;
  group_by(lf, nf, fwd, c->fwdOff);
  group_by(lb, nb, bwd, c->bwdOff);
  for (int32_t** d : {&c->fwdPartLev, &c->bwdPartLev}) {
    if (*d) {
      auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)*d);
      if (it != c->allocs.end()) c->allocs.erase(it);
      cudaFree(*d);
      *d = nullptr;
    }
  }
  if (P > 1) {
    if ((rc = dalloc(c, c->fwdPartLev, sizeof(int32_t) * (P + 1))) || (rc = dalloc(c, c->bwdPartLev, sizeof(int32_t) * (P + 1))))
      return rc;
    DG_CUDA(c, cudaMemcpy(c->fwdPartLev, baseF.data(), sizeof(int32_t) * (P + 1), cudaMemcpyHostToDevice));
    DG_CUDA(c, cudaMemcpy(c->bwdPartLev, baseB.data(), sizeof(int32_t) * (P + 1), cudaMemcpyHostToDevice));
  }
  c->maxLevelWidth = 0;
  for (int k = 0; k < nf; k++) c->maxLevelWidth = std::max(c->maxLevelWidth, c->fwdOff[k + 1] - c->fwdOff[k]);
  for (int k = 0; k < nb; k++) c->maxLevelWidth = std::max(c->maxLevelWidth, c->bwdOff[k + 1] - c->bwdOff[k]);
  for (int64_t** d : {&c->fwdOffDev, &c->bwdOffDev}) {
    if (*d) {
      auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)*d);
      if (it != c->allocs.end()) c->allocs.erase(it);
      cudaFree(*d);
      *d = nullptr;
    }
  }
  if ((rc = dalloc(c, c->fwdOffDev, sizeof(int64_t) * (nf + 1))) || (rc = dalloc(c, c->bwdOffDev, sizeof(int64_t) * (nb + 1))))
    return rc;
  DG_CUDA(c, cudaMemcpy(c->fwdOffDev, c->fwdOff.data(), sizeof(int64_t) * (nf + 1), cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->bwdOffDev, c->bwdOff.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice));
  // per schedule position: the face slots and the neighbours that enter each sweep
  std::vector<int32_t> slots((size_t)aos_size(N, c->nfmax)), L(c->F), R(c->F);
  DG_CUDA(c, cudaMemcpy(slots.data(), c->cellFace, sizeof(int32_t) * slots.size(), cudaMemcpyDeviceToHost));
  DG_CUDA(c, cudaMemcpy(L.data(), c->faceL, sizeof(int32_t) * c->F, cudaMemcpyDeviceToHost));
  DG_CUDA(c, cudaMemcpy(R.data(), c->faceR, sizeof(int32_t) * c->F, cudaMemcpyDeviceToHost));
  auto records = [&](const std::vector<int32_t>& cellsOf, bool forward, std::vector<int32_t>& nf,
                     std::vector<int32_t>& nj, std::vector<int32_t>& np) {
    nf.assign(4 * N, kEmptySlot);
    nj.assign(4 * N, -1);
    np.assign(4 * N, -1);
    std::vector<int32_t> at(N);
    for (int64_t t = 0; t < N; t++) at[cellsOf[t]] = (int32_t)t;
    for (int64_t t = 0; t < N; t++) {
      const int64_t i = cellsOf[t];
      for (int k = 0; k < c->nfmax && k < 4; k++) {
        const int32_t sf = slots[aos(i, k, c->nfmax)];
        nf[4 * t + k] = sf;
        if (sf == kEmptySlot) continue;
        const int32_t f = sf >= 0 ? sf : ~sf;
        const int32_t j = sf >= 0 ? R[f] : L[f];
        if (j < 0) continue;
        if (part[j] != part[i]) {
          if (!forward) {
            nj[4 * t + k] = j;
            np[4 * t + k] = kGhostPos;
          }
        } else if (forward ? pos[j] < pos[i] : pos[j] > pos[i]) {
          nj[4 * t + k] = j;
          np[4 * t + k] = at[j];
        }
      }
    }
  };
  // the level walk keeps the increments of the last kMatRing positions in a ring; a neighbour at
  // position pj is still there during level l when pj + kMatRing >= off[l + 1] (the position that
  // overwrites its slot comes later).  Otherwise the walk reads global memory: position -1.
  auto ring_or_global = [&](const std::vector<int64_t>& off, std::vector<int32_t>& np) {
    for (size_t l = 0; l + 1 < off.size(); l++)
      for (int64_t t = off[l]; t < off[l + 1]; t++)
        for (int k = 0; k < 4; k++)
          if (np[4 * t + k] >= 0 && np[4 * t + k] + kMatRing < off[l + 1]) np[4 * t + k] = -1;
  };
  std::vector<int32_t> ff, fj, fp, bf, bj, bp;
  records(fwd, true, ff, fj, fp);
  records(bwd, false, bf, bj, bp);
  ring_or_global(c->fwdOff, fp);
  ring_or_global(c->bwdOff, bp);
  if (!c->fwdNbF)
    if ((rc = dalloc(c, c->fwdNbF, sizeof(int32_t) * 4 * N)) || (rc = dalloc(c, c->fwdNbJ, sizeof(int32_t) * 4 * N)) ||
        (rc = dalloc(c, c->bwdNbF, sizeof(int32_t) * 4 * N)) || (rc = dalloc(c, c->bwdNbJ, sizeof(int32_t) * 4 * N)) ||
        (rc = dalloc(c, c->fwdNbP, sizeof(int32_t) * 4 * N)) || (rc = dalloc(c, c->bwdNbP, sizeof(int32_t) * 4 * N)))
      return rc;
  DG_CUDA(c, cudaMemcpy(c->fwdNbP, fp.data(), sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->bwdNbP, bp.data(), sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->fwdNbF, ff.data(), sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->fwdNbJ, fj.data(), sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->bwdNbF, bf.data(), sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  DG_CUDA(c, cudaMemcpy(c->bwdNbJ, bj.data(), sizeof(int32_t) * 4 * N, cudaMemcpyHostToDevice));
  if (!c->lusgsMat && (rc = dalloc(c, c->lusgsMat, (c->sa ? sizeof(LuMatS) : sizeof(LuMatF)) * N))) return rc;
  for (const void* fn : {(const void*)k_lusgs_levels_mat<float, true, false>, (const void*)k_lusgs_levels_mat<float, false, false>,
                         (const void*)k_lusgs_levels_mat<double, true, false>, (const void*)k_lusgs_levels_mat<double, false, false>})
    DG_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mat_smem<false>()));
  for (const void* fn : {(const void*)k_lusgs_levels_mat<float, true, true>, (const void*)k_lusgs_levels_mat<float, false, true>,
                         (const void*)k_lusgs_levels_mat<double, true, true>, (const void*)k_lusgs_levels_mat<double, false, true>})
    DG_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mat_smem<true>()));
  c->lusgsOrder = 1;
  return upload_schedule(c, pos, fwd, bwd);
}

template <class T>
void launch_lusgs_sweep(dndsg_ctx* c, bool forward, double alpha, const double* rhs, double* inc, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  const std::vector<int64_t>& off = forward ? c->fwdOff : c->bwdOff;
  const int32_t* cells = forward ? c->fwdCells : c->bwdCells;
  const int nb = (int)off.size() - 1;
  // many narrow levels: one block walks them all over records packed in parallel beforehand
  // (a launch per level would cost more than the work)
  if (c->lusgsOrder == 1 && (forward ? c->fwdPartMax : c->bwdPartMax) <= kRecMaxLevels && c->nfmax <= 4) {
    const int64_t* od = forward ? c->fwdOffDev : c->bwdOffDev;
    const int32_t* nf = forward ? c->fwdNbF : c->bwdNbF;
    const int32_t* nj = forward ? c->fwdNbJ : c->bwdNbJ;
    const int32_t* np = forward ? c->fwdNbP : c->bwdNbP;
    const int32_t* pl = c->lusgsParts > 1 ? (forward ? c->fwdPartLev : c->bwdPartLev) : nullptr;
    const int nblk = c->lusgsParts > 1 ? c->lusgsParts : 1;
    SaView<T> none{};
    LuMatF* rec = (LuMatF*)c->lusgsMat;
    if (forward) {
      k_lusgs_pack_mat<T, true, false><<<grid_for(c->N), kBlock, 0, s>>>(h, none, cells, nf, nj, np, c->N, alpha, c->Dinv,
                                                                          rhs, inc, rec);
      k_lusgs_levels_mat<T, true, false><<<nblk, mat_threads<false>(), mat_smem<false>(), s>>>(none, rec, od, nb, pl, inc,
                                                                                              h.gamma - 1, c->flags);
    } else {
      k_lusgs_pack_mat<T, false, false><<<grid_for(c->N), kBlock, 0, s>>>(h, none, cells, nf, nj, np, c->N, alpha, c->Dinv,
                                                                           rhs, inc, rec);
      k_lusgs_levels_mat<T, false, false><<<nblk, mat_threads<false>(), mat_smem<false>(), s>>>(none, rec, od, nb, pl, inc,
                                                                                               h.gamma - 1, c->flags);
    }
    return;
  }
  if (c->lusgsOrder == 1 && c->maxLevelWidth <= 8 * kLevelBlock) {
    const int64_t* od = forward ? c->fwdOffDev : c->bwdOffDev;
    if (forward) k_lusgs_levels<T, true><<<1, kLevelBlock, 0, s>>>(h, c->rankOf, cells, od, nb, alpha, c->Dinv, rhs, inc);
    else k_lusgs_levels<T, false><<<1, kLevelBlock, 0, s>>>(h, c->rankOf, cells, od, nb, alpha, c->Dinv, rhs, inc);
    return;
  }
  for (int k = 0; k < nb; k++) {
    const int64_t b = off[k], n = off[k + 1] - b;
    if (n == 0) continue;
    if (forward)
      k_lusgs_batch<T, true><<<grid_for(n), kBlock, 0, s>>>(h, c->rankOf, cells + b, n, alpha, c->Dinv, rhs, inc);
    else
      k_lusgs_batch<T, false><<<grid_for(n), kBlock, 0, s>>>(h, c->rankOf, cells + b, n, alpha, c->Dinv, rhs, inc);
  }
}

// ImplicitBDFDualTimeStep::Step (DNDS_ODE.hpp:444-486), one pseudo-time iteration at order 1, with
// the EulerSolver lambdas (DNDS_FV_EulerSolver.hpp:713-925): fdtau (local EvaluateDt), frhs
// (n_rec Jacobi sweeps, limiter, EvaluateRHS), fsolve (LUSGSMatrixInit, forward, backward from a
// zero increment), then x += inc and the L1 norm of inc (the fstop residual) into resAcc
template <class T>
int run_implicit(dndsg_ctx* c, double cfl, double dtPhys, double alpha, int nRec, int volWise, double t,
                 cudaStream_t s) {
  int rc;
  if ((rc = ensure_lusgs(c))) return rc;
  run_dt<T>(c, cfl, 1e100, false, s);
  for (int k = 0; k < nRec; k++) run_vr<T>(c, false, s);
  if (c->s.limiter) run_limiter<T>(c, 0, s);
  run_rhs<T>(c, t, s);
  const double dtInv = 1.0 / dtPhys;
  const int64_t n4 = c->N * 4;
  k_bdf_rhs<<<(unsigned)((n4 + kBlock - 1) / kBlock), kBlock, 0, s>>>(n4, c->u, c->uLast, alpha, dtInv, c->rhs);
  HotView<T> h = view<T>(c);
  k_lusgs_init<T><<<grid_for(c->N), kBlock, 0, s>>>(h, dtInv, alpha, c->Dinv, c->Dmat);
  launch_lusgs_sweep<T>(c, true, alpha, c->rhs, c->inc, s);
  launch_lusgs_sweep<T>(c, false, alpha, c->rhs, c->inc, s);
  DG_CUDA(c, cudaMemsetAsync(c->resAcc, 0, sizeof(double) * 16, s));
  k_add_inc<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->u, c->inc, c->vol, volWise, c->resAcc);
  if (c->F > c->Fi)
    k_wall_flux<<<grid_for(c->F - c->Fi), kBlock, 0, s>>>(c->Fi, c->F, c->faceBC, c->flux, c->resAcc + 4);
  return check_launch(c);
}
}  // namespace

extern "C" {

int dndsg_lusgs_colours(dndsg_ctx* c, int32_t* colour_out, int* n_colours) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c)) || (rc = ensure_lusgs(c))) return rc;
  if (colour_out) std::memcpy(colour_out, c->colourHost.data(), sizeof(int32_t) * c->N);
  if (n_colours) *n_colours = 1 + *std::max_element(c->colourHost.begin(), c->colourHost.end());
  return 0;
}

int dndsg_lusgs_set_order(dndsg_ctx* c, int mode, const int64_t* scan2cell, int* n_batches) {
  if (!c || (mode != 0 && mode != 1)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c)) || (rc = ensure_lusgs(c))) return rc;
  if (mode == 1) {
    if ((rc = set_scan_order(c, scan2cell))) return rc;
  } else if (c->lusgsOrder != 0) {
    const int64_t N = c->N;
    const std::vector<int32_t>& col = c->colourHost;
    const int ncol = 1 + *std::max_element(col.begin(), col.end());
    std::vector<int32_t> fwd, bwd, rev(N);
    group_by(col, ncol, fwd, c->fwdOff);
    for (int64_t i = 0; i < N; i++) rev[i] = ncol - 1 - col[i];
    group_by(rev, ncol, bwd, c->bwdOff);
    c->lusgsOrder = 0;
    if ((rc = upload_schedule(c, col, fwd, bwd))) return rc;
  }
  if (n_batches)
    *n_batches = c->lusgsOrder == 1 ? c->fwdPartMax + c->bwdPartMax : (int)(c->fwdOff.size() - 1 + c->bwdOff.size() - 1);
  return 0;
}

int dndsg_lusgs_set_parts(dndsg_ctx* c, const int32_t* part, int n_parts, int* n_batches) {
  if (!c || (part && (n_parts < 1 || n_parts > 65535))) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c)) || (rc = ensure_lusgs(c))) return rc;
  if (part && n_parts > 1) {
    for (int64_t i = 0; i < c->N; i++)
      if (part[i] < 0 || part[i] >= n_parts) return fail(c, DNDSG_BAD_ARGUMENT, "part index out of range");
    c->lusgsPart.assign(part, part + c->N);
    c->lusgsParts = n_parts;
  } else {
    c->lusgsPart.clear();
    c->lusgsParts = 1;
  }
  if ((rc = set_scan_order(c, c->scanHost.empty() ? nullptr : c->scanHost.data()))) {
    c->lusgsPart.clear();
    c->lusgsParts = 1;
    return rc;
  }
  if (n_batches) *n_batches = c->fwdPartMax + c->bwdPartMax;
  return 0;
}

int dndsg_lusgs_matrix_init(dndsg_ctx* c, double dt_phys, double alpha, void* s) {
  if (!c || !(dt_phys > 0) || !(alpha > 0)) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c)) || (rc = ensure_lusgs(c))) return rc;
  if (c->fp32) k_lusgs_init<float><<<grid_for(c->N), kBlock, 0, st(s)>>>(view<float>(c), 1.0 / dt_phys, alpha, c->Dinv, c->Dmat);
  else k_lusgs_init<double><<<grid_for(c->N), kBlock, 0, st(s)>>>(view<double>(c), 1.0 / dt_phys, alpha, c->Dinv, c->Dmat);
  return check_launch(c);
}

static int lusgs_sweep_api(dndsg_ctx* c, bool fwd, double alpha, const double* rhs, double* inc, void* s) {
  if (!c || !rhs || !inc) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  if (c->sa) return fail(c, DNDSG_UNSUPPORTED, "SA contexts sweep inside dndsg_implicit_iteration");
  if (!c->rankOf) return fail(c, DNDSG_BAD_ARGUMENT, "dndsg_lusgs_matrix_init first");
  int rc;
  if ((rc = set_device(c))) return rc;
  if (c->fp32) launch_lusgs_sweep<float>(c, fwd, alpha, rhs, inc, st(s));
  else launch_lusgs_sweep<double>(c, fwd, alpha, rhs, inc, st(s));
  return check_launch(c);
}

int dndsg_lusgs_forward(dndsg_ctx* c, double alpha, const double* rhs, double* inc, void* s) {
  return lusgs_sweep_api(c, true, alpha, rhs, inc, s);
}

int dndsg_lusgs_backward(dndsg_ctx* c, double alpha, const double* rhs, double* inc, void* s) {
  return lusgs_sweep_api(c, false, alpha, rhs, inc, s);
}

int dndsg_bdf_begin(dndsg_ctx* c, void* s) {
  if (!c) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c))) return rc;
  DG_CUDA(c, cudaMemcpyAsync(c->uLast, c->u, sizeof(double) * 4 * c->N, cudaMemcpyDeviceToDevice, st(s)));
  if (c->sa) DG_CUDA(c, cudaMemcpyAsync(c->saULast, c->saU, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, st(s)));
  return 0;
}

int dndsg_implicit_iteration(dndsg_ctx* c, double cfl, double dt_phys, double alpha, int n_rec, int vol_wise,
                             double t, double* inc_res_out, double* wall_flux_out, void* s) {
  if (!c || !(cfl > 0) || !(dt_phys > 0) || !(alpha > 0) || n_rec < 0) return DNDSG_BAD_ARGUMENT;
  if (c->dead) return refuse_dead(c);
  int rc;
  if ((rc = set_device(c))) return rc;
  if (c->sa) rc = sa_implicit(c, cfl, dt_phys, alpha, n_rec, vol_wise, st(s));
  else
    rc = c->fp32 ? run_implicit<float>(c, cfl, dt_phys, alpha, n_rec, vol_wise, t, st(s))
                 : run_implicit<double>(c, cfl, dt_phys, alpha, n_rec, vol_wise, t, st(s));
  if (rc) return rc;
  if (inc_res_out || wall_flux_out) {
    double acc[16];
    DG_CUDA(c, cudaMemcpyAsync(acc, c->resAcc, sizeof(acc), cudaMemcpyDeviceToHost, st(s)));
    DG_CUDA(c, cudaStreamSynchronize(st(s)));
    if (inc_res_out) for (int v = 0; v < 4; v++) inc_res_out[v] = acc[v];
    if (wall_flux_out) for (int v = 0; v < 4; v++) wall_flux_out[v] = acc[4 + v];
    if (c->sa) {
      if (inc_res_out) inc_res_out[4] = acc[8];
      if (wall_flux_out) wall_flux_out[4] = acc[9];
    }
    return observe_timeout(c, st(s));
  }
  return 0;
}

}  // extern "C"

// ====================================================================== SA contexts (nvars 5)
namespace {

template <class T>
__global__ void __launch_bounds__(kBlock) k_sa_vr(HotView<T> h, SaView<T> sa) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < h.N) sa_vr_cell<T>(i, h, sa);
}

// one thread per (face, Gauss point), as for the cell source: three times the resident warps for the
// long per-point chain (Roe, gradients, viscous and U5 fluxes).  Thread g == 0 of each face sums the
// points in order.
constexpr int kSaFluxFaces = 64;
inline unsigned sa_flux_grid(int64_t n) { return (unsigned)((n + kSaFluxFaces - 1) / kSaFluxFaces); }
template <class T, int RIEMANN, bool BND>
__global__ void __launch_bounds__(kSaFluxFaces * 3) k_face_flux_sa(HotView<T> h, SaView<T> sa, int64_t f0, int64_t f1,
                                                                   unsigned* flags, unsigned long long* nred) {
  __shared__ double part[kSaFluxFaces * 3][5];
  const int64_t f = f0 + blockIdx.x * (int64_t)kSaFluxFaces + threadIdx.x / 3;
  const int g = threadIdx.x % 3;
  int r = 0;
  bool bad = false;
  if (f < f1) {
    double c[4], cS;
    r = face_flux_sa_point<T, RIEMANN, BND>(f, g, h, sa, c, cS, bad);
    for (int k = 0; k < 4; k++) part[threadIdx.x][k] = c[k];
    part[threadIdx.x][4] = cS;
  }
  __syncthreads();
  if (f < f1 && g == 0) {
    double acc[5] = {0, 0, 0, 0, 0};
    for (int q = 0; q < 3; q++)
      for (int k = 0; k < 5; k++) acc[k] -= part[threadIdx.x + q][k];
    for (int k = 0; k < 5; k++)
      if (!(acc[k] == acc[k])) bad = true;
    double* o = &h.flux[f * 4];
    *reinterpret_cast<double2*>(o) = make_double2(acc[0], acc[1]);
    *reinterpret_cast<double2*>(o + 2) = make_double2(acc[2], acc[3]);
    sa.flux[f] = acc[4];
  }
  unsigned anyBad = __ballot_sync(0xffffffffu, bad);
  int rs = __reduce_add_sync(0xffffffffu, r);
  if ((threadIdx.x & 31) == 0) {
    if (anyBad) atomicOr(flags, 1u);
    if (rs) atomicAdd(nred, (unsigned long long)rs);
  }
}

// one thread per (cell, quadrature point): the source's transcendental chain per point is long and
// one thread per cell left too few warps resident on a 65,536-cell mesh; thread ig == 0 of each cell
// then sums the points in order (the same sum as a sequential loop over the points)
constexpr int kSaRhsCells = 32;
template <class T>
__global__ void __launch_bounds__(kSaRhsCells * kSaGp) k_sa_cell_rhs(HotView<T> h, SaView<T> sa) {
  __shared__ double sv[kSaRhsCells * kSaGp], sj[kSaRhsCells * kSaGp];
  const int64_t i = blockIdx.x * (int64_t)kSaRhsCells + threadIdx.x / kSaGp;
  const int ig = threadIdx.x % kSaGp;
  double src = 0, jac = 0;
  if (i < h.N) sa_cell_point<T>(i, ig, h, sa, src, jac);
  sv[threadIdx.x] = src;
  sj[threadIdx.x] = jac;
  __syncthreads();
  if (ig == 0 && i < h.N) sa_cell_rhs<T>(i, h, sa, &sv[threadIdx.x], &sj[threadIdx.x]);
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_dt_face_sa(HotView<T> h, SaView<T> sa) {
  const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f < h.F) dt_face_sa<T>(f, h, sa);
}

template <class T, bool FWD>
__global__ void __launch_bounds__(kBlock) k_lusgs_batch_sa(HotView<T> h, SaView<T> sa, const int32_t* rankOf,
                                                           const int32_t* cells, int64_t n, double alpha,
                                                           const double* Dinv, const double* rhs, double* inc) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) lusgs_cell_sa<T, FWD>(h, sa, rankOf, cells[t], alpha, Dinv, rhs, inc);
}

// all narrow levels of one sweep in one block (as k_lusgs_levels), 5 variables
template <class T, bool FWD>
__global__ void __launch_bounds__(kLevelBlock) k_lusgs_levels_sa(HotView<T> h, SaView<T> sa, const int32_t* rankOf,
                                                                 const int32_t* cells, const int64_t* off, int nlev,
                                                                 double alpha, const double* Dinv, const double* rhs,
                                                                 double* inc) {
  for (int l = 0; l < nlev; l++) {
    const int64_t b = off[l], e = off[l + 1];
    for (int64_t t = b + threadIdx.x; t < e; t += blockDim.x)
      lusgs_cell_sa<T, FWD>(h, sa, rankOf, cells[t], alpha, Dinv, rhs, inc);
    __syncthreads();
  }
}

// the U5 diagonal: the flow one plus alpha * the source Jacobian (LUSGSMatrixInit), its inverse
// for the sweeps and (DS, may be null) itself for LUSGSMatrixVec
__global__ void k_sa_diag(int64_t N, const double* D, const double* srcJac, double alpha, double* DinvS, double* DS) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double d = D[i] + alpha * srcJac[i];
  DinvS[i] = 1.0 / d;
  if (DS) DS[i] = d;
}

// U5 parts of one pseudo-time iteration: the BDF rhs, CompressInc of rhs * dTau (dTau = dt / alpha)
__global__ void k_sa_rhs_fix(int64_t N, const double* u, const double* uLast, const double* dt, double alpha,
                             double dtPhysInv, double* rhs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  double r = alpha * rhs[i] - u[i] * dtPhysInv + uLast[i] * dtPhysInv;
  const double dTau = dt[i] / alpha;
  r = sa_compress_inc(u[i], r * dTau) / dTau;
  rhs[i] = r;
}

// CompressInc of the U5 increment, u5 += inc, its L1 norm, and the U5 wall flux
__global__ void __launch_bounds__(kBlock) k_sa_add_inc(int64_t N, double* u, double* inc, const double* vol,
                                                       int volWise, double* acc) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double a = 0;
  if (i < N) {
    const double d = sa_compress_inc(u[i], inc[i]);
    inc[i] = d;
    u[i] += d;
    a = fabs(d) * (volWise ? vol[i] : 1.0);
  }
  block_add(a, acc);
}

__global__ void __launch_bounds__(kBlock) k_sa_wall_flux(int64_t Fi, int64_t F, const int32_t* faceBC,
                                                         const double* flux, double* acc) {
  const int64_t f = Fi + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double a = 0;
  if (f < F && (faceBC[f] == BC_WALL_NOSLIP || faceBC[f] == BC_WALL_EULER)) a = -flux[f];
  a = warp_sum(a);
  if ((threadIdx.x & 31) == 0 && a != 0.0) atomicAdd(acc, a);
}

template <class T>
void run_vr_sa(dndsg_ctx* c, cudaStream_t s) {
  run_vr<T>(c, false, s);
  k_sa_vr<T><<<grid_for(c->N), kBlock, 0, s>>>(view<T>(c), sa_view<T>(c));
  std::swap(c->saUrec, c->saUrecNew);
}

template <class T>
void run_dt_sa(dndsg_ctx* c, double cfl, double maxDt, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  k_init_dtmin<<<1, 1, 0, s>>>(c->scal);
  k_dt_face_sa<T><<<grid_for(c->F), kBlock, 0, s>>>(h, sa_view<T>(c));
  k_dt_cell<T, false><<<grid_for(c->N), kBlock, 0, s>>>(h, cfl, maxDt, c->scal);
}

template <class T>
void run_rhs_sa(dndsg_ctx* c, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  SaView<T> sa = sa_view<T>(c);
  const int64_t Fi = c->Fi, F = c->F;
  if (c->s.riemann == 2) {
    if (Fi > 0) k_face_flux_sa<T, 2, false><<<sa_flux_grid(Fi), kSaFluxFaces * 3, 0, s>>>(h, sa, 0, Fi, c->flags, c->nreduced);
    if (F > Fi) k_face_flux_sa<T, 2, true><<<sa_flux_grid(F - Fi), kSaFluxFaces * 3, 0, s>>>(h, sa, Fi, F, c->flags, c->nreduced);
  } else {
    if (Fi > 0) k_face_flux_sa<T, 1, false><<<sa_flux_grid(Fi), kSaFluxFaces * 3, 0, s>>>(h, sa, 0, Fi, c->flags, c->nreduced);
    if (F > Fi) k_face_flux_sa<T, 1, true><<<sa_flux_grid(F - Fi), kSaFluxFaces * 3, 0, s>>>(h, sa, Fi, F, c->flags, c->nreduced);
  }
  k_cell_update<T, -1><<<grid_for(c->N), kBlock, 0, s>>>(h, c->scal);
  k_sa_cell_rhs<T><<<(unsigned)((c->N + kSaRhsCells - 1) / kSaRhsCells), kSaRhsCells * kSaGp, 0, s>>>(h, sa);
}

template <class T>
void launch_lusgs_sweep_sa(dndsg_ctx* c, bool forward, double alpha, const double* rhs4, double* inc4,
                           const double* rhs5, double* inc5, cudaStream_t s) {
  HotView<T> h = view<T>(c);
  SaView<T> sa = sa_view<T>(c);
  sa.rhs = const_cast<double*>(rhs5);  // read only by the sweeps
  sa.inc = inc5;
  const std::vector<int64_t>& off = forward ? c->fwdOff : c->bwdOff;
  const int32_t* cells = forward ? c->fwdCells : c->bwdCells;
  const int nb = (int)off.size() - 1;
  if (c->lusgsOrder == 1 && (forward ? c->fwdPartMax : c->bwdPartMax) <= kRecMaxLevels && c->nfmax <= 4) {
    const int64_t* od = forward ? c->fwdOffDev : c->bwdOffDev;
    const int32_t* nf = forward ? c->fwdNbF : c->bwdNbF;
    const int32_t* nj = forward ? c->fwdNbJ : c->bwdNbJ;
    const int32_t* np = forward ? c->fwdNbP : c->bwdNbP;
    const int32_t* pl = c->lusgsParts > 1 ? (forward ? c->fwdPartLev : c->bwdPartLev) : nullptr;
    const int nblk = c->lusgsParts > 1 ? c->lusgsParts : 1;
    LuMatS* rec = (LuMatS*)c->lusgsMat;
    if (forward) {
      k_lusgs_pack_mat<T, true, true><<<grid_for(c->N), kBlock, 0, s>>>(h, sa, cells, nf, nj, np, c->N, alpha, c->Dinv,
                                                                         rhs4, inc4, rec);
      k_lusgs_levels_mat<T, true, true><<<nblk, mat_threads<true>(), mat_smem<true>(), s>>>(sa, rec, od, nb, pl, inc4,
                                                                                           h.gamma - 1, c->flags);
    } else {
      k_lusgs_pack_mat<T, false, true><<<grid_for(c->N), kBlock, 0, s>>>(h, sa, cells, nf, nj, np, c->N, alpha, c->Dinv,
                                                                          rhs4, inc4, rec);
      k_lusgs_levels_mat<T, false, true><<<nblk, mat_threads<true>(), mat_smem<true>(), s>>>(sa, rec, od, nb, pl, inc4,
                                                                                            h.gamma - 1, c->flags);
    }
    return;
  }
  if (c->lusgsOrder == 1) {  // many narrow levels: one block walks them all
    const int64_t* od = forward ? c->fwdOffDev : c->bwdOffDev;
    if (forward)
      k_lusgs_levels_sa<T, true><<<1, kLevelBlock, 0, s>>>(h, sa, c->rankOf, cells, od, nb, alpha, c->Dinv, rhs4, inc4);
    else
      k_lusgs_levels_sa<T, false><<<1, kLevelBlock, 0, s>>>(h, sa, c->rankOf, cells, od, nb, alpha, c->Dinv, rhs4, inc4);
    return;
  }
  for (int k = 0; k < nb; k++) {
    const int64_t b = off[k], n = off[k + 1] - b;
    if (n == 0) continue;
    if (forward)
      k_lusgs_batch_sa<T, true><<<grid_for(n), kBlock, 0, s>>>(h, sa, c->rankOf, cells + b, n, alpha, c->Dinv, rhs4, inc4);
    else
      k_lusgs_batch_sa<T, false><<<grid_for(n), kBlock, 0, s>>>(h, sa, c->rankOf, cells + b, n, alpha, c->Dinv, rhs4, inc4);
  }
}

// one pseudo-time iteration of an SA context (as run_implicit, with the U5 equation and the
// positivity fixes of fsolve)
template <class T>
int run_implicit_sa(dndsg_ctx* c, double cfl, double dtPhys, double alpha, int nRec, int volWise, cudaStream_t s) {
  int rc;
  if ((rc = ensure_lusgs(c))) return rc;
  run_dt_sa<T>(c, cfl, 1e100, s);
  for (int k = 0; k < nRec; k++) run_vr_sa<T>(c, s);
  run_rhs_sa<T>(c, s);
  const double dtInv = 1.0 / dtPhys;
  const int64_t n4 = c->N * 4;
  k_bdf_rhs<<<(unsigned)((n4 + kBlock - 1) / kBlock), kBlock, 0, s>>>(n4, c->u, c->uLast, alpha, dtInv, c->rhs);
  k_sa_rhs_fix<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->saU, c->saULast, c->dt, alpha, dtInv, c->saRhs);
  HotView<T> h = view<T>(c);
  k_lusgs_init<T><<<grid_for(c->N), kBlock, 0, s>>>(h, dtInv, alpha, c->Dinv, c->Dmat);
  k_sa_diag<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->Dmat, c->saSrcJac, alpha, c->saDinv, nullptr);
  launch_lusgs_sweep_sa<T>(c, true, alpha, c->rhs, c->inc, c->saRhs, c->saInc, s);
  launch_lusgs_sweep_sa<T>(c, false, alpha, c->rhs, c->inc, c->saRhs, c->saInc, s);
  DG_CUDA(c, cudaMemsetAsync(c->resAcc, 0, sizeof(double) * 16, s));
  k_add_inc<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->u, c->inc, c->vol, volWise, c->resAcc);
  k_sa_add_inc<<<grid_for(c->N), kBlock, 0, s>>>(c->N, c->saU, c->saInc, c->vol, volWise, c->resAcc + 8);
  if (c->F > c->Fi) {
    k_wall_flux<<<grid_for(c->F - c->Fi), kBlock, 0, s>>>(c->Fi, c->F, c->faceBC, c->flux, c->resAcc + 4);
    k_sa_wall_flux<<<grid_for(c->F - c->Fi), kBlock, 0, s>>>(c->Fi, c->F, c->faceBC, c->saFlux, c->resAcc + 9);
  }
  return check_launch(c);
}

}  // namespace

namespace {
int sa_vr_steps(dndsg_ctx* c, int nsweeps, cudaStream_t s) {
  for (int k = 0; k < nsweeps; k++) {
    if (c->fp32) run_vr_sa<float>(c, s);
    else run_vr_sa<double>(c, s);
  }
  return check_launch(c);
}
int sa_eval_dt(dndsg_ctx* c, double cfl, double maxDt, cudaStream_t s) {
  if (c->fp32) run_dt_sa<float>(c, cfl, maxDt, s);
  else run_dt_sa<double>(c, cfl, maxDt, s);
  return check_launch(c);
}
int sa_eval_rhs(dndsg_ctx* c, cudaStream_t s) {
  if (c->fp32) run_rhs_sa<float>(c, s);
  else run_rhs_sa<double>(c, s);
  return check_launch(c);
}
int sa_implicit(dndsg_ctx* c, double cfl, double dtPhys, double alpha, int nRec, int volWise, cudaStream_t s) {
  return c->fp32 ? run_implicit_sa<float>(c, cfl, dtPhys, alpha, nRec, volWise, s)
                 : run_implicit_sa<double>(c, cfl, dtPhys, alpha, nRec, volWise, s);
}
}  // namespace

#include "dndsg_dual.cuh"
