// dndsg_mlp.cuh -- learned warm start for the VR coefficients (no counterpart in
// the reference): a per-cell MLP 64 -> 64 -> 64 -> 64 -> 20 (SiLU), BF16 weights
// and activations, FP32 accumulation, on the 5th-generation tensor cores
// (tcgen05.mma with the accumulators in tensor memory): inference (k_mlp_tc) and
// training (k_mlp_train_tc: forward, backward with the weight and input
// gradients, then Adam on the FP32 master parameters).
//
// The network extrapolates the Jacobi sequence: from the starting coefficients
// x0 and two plain sweeps x1 = J(x0), x2 = J(x1) it proposes the converged
// coefficients x* (for an error dominated by one slow mode of eigenvalue l,
// x* - x2 = (x2 - x1) l / (1 - l); the network learns the local, many-mode
// version of that from the solver's own iterations).
// Features of cell i (d1 = x1 - x0, d2 = x2 - x1):
//   x[4k + v]      = du_k[v] / s_v,  du_k = u_j(k) - u_i over the face slots k < 4
//                    (zero for boundary or absent slots), s_v = max_k |du_k[v]|
//   x[16 + 4q + v] = d1[q][v] / r_v,  r_v = max_q |d1[q][v]|
//   x[36 + 4q + v] = d2[q][v] / r_v
//   x[56 + 2k + d] = slot k's face centre in the cell's own polynomial frame,
//                    (xi, eta) = Pinv (x_f - c_i)
// Output y[4q + v] = (x* - x2)[q][v] / r_v.  Increments and the remaining error
// are linear in the error of x0 and the sweep acts on each variable alike, so
// this scaling makes the learned map homogeneous of degree one per variable.
// Scales are floored so that a converged or uniform region gives finite features.
#pragma once
#include <cuda_bf16.h>

#include "dndsg_bodies.cuh"

namespace dg {

constexpr int kIn = 64, kInP = 64, kHid = 64, kOut = 20, kOutP = 32;
// FP32 master parameters, contiguous: W1[64][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[32][64] b4[32]
// (W[n][k]: output unit n, input k; padded rows/columns are kept at zero)
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kInP, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid,
              kOffB4 = kOffW4 + kOutP * kHid, kNParam = kOffB4 + kOutP;
// BF16 weight copy (the matrices only), same order without biases
constexpr int kWOff1 = 0, kWOff2 = kWOff1 + kHid * kInP, kWOff3 = kWOff2 + kHid * kHid, kWOff4 = kWOff3 + kHid * kHid,
              kNW = kWOff4 + kOutP * kHid;

DG_HD float sigm(float z) {
#if defined(__CUDA_ARCH__)
  return 1.0f / (1.0f + __expf(-z));
#else
  return 1.0f / (1.0f + expf(-z));
#endif
}
DG_HD float silu(float z) { return z * sigm(z); }
DG_HD float silu_grad(float z) {
  float s = sigm(z);
  return s * (1.0f + z * (1.0f - s));
}

// the coefficient iterates the features are taken from
template <class T>
struct MlpIters {
  const T* x0;
  const T* x1;
  const T* x2;
  const float* geom;  // [N][8] slot face centres in each cell's own frame
};

// features of one cell into x[64] and the output scales r[4]
template <class T>
DG_HD void mlp_cell_features(int64_t i, const HotView<T>& h, const MlpIters<T>& it, float x[kInP], float r[4]) {
  double du[4][4], ui[4];
  for (int v = 0; v < 4; v++) ui[v] = h.u[i * 4 + v];
  for (int k = 0; k < 4; k++)
    for (int v = 0; v < 4; v++) du[k][v] = 0.0;
  for (int k = 0; k < h.nfmax && k < 4; k++) {
    if (h.vrMode[aos(i, k, h.nfmax)] != VR_INNER) continue;
    const int64_t j = h.vrNbr[aos(i, k, h.nfmax)];
    for (int v = 0; v < 4; v++) du[k][v] = h.u[j * 4 + v] - ui[v];
  }
  double d1[20], d2[20];
  for (int e = 0; e < 20; e++) {
    const double a = it.x0[i * 20 + e], b = it.x1[i * 20 + e], c = it.x2[i * 20 + e];
    d1[e] = b - a;
    d2[e] = c - b;
  }
  auto clampf = [](double a) { return (float)(a > 1e3 ? 1e3 : (a < -1e3 ? -1e3 : a)); };
  for (int v = 0; v < 4; v++) {
    double m = 0, md = 0;
    for (int k = 0; k < 4; k++) m = dmax(m, fabs(du[k][v]));
    for (int q = 0; q < 5; q++) md = dmax(md, fabs(d1[4 * q + v]));
    const double s = dmax(m, dmax(1e-12 * fabs(ui[v]), 1e-30));
    const double rv = dmax(md, 1e-30);
    r[v] = (float)rv;
    for (int k = 0; k < 4; k++) x[4 * k + v] = clampf(du[k][v] / s);
    for (int q = 0; q < 5; q++) {
      x[16 + 4 * q + v] = clampf(d1[4 * q + v] / (double)r[v]);
      x[36 + 4 * q + v] = clampf(d2[4 * q + v] / (double)r[v]);
    }
  }
  for (int k = 0; k < 8; k++) x[56 + k] = it.geom[i * 8 + k];
}

// The second input design, the one the configuration names: the neighbour mean differences to up to 4
// neighbours and the previous-step coefficients x0 (the coefficients the reconstruction starts from:
// those the previous stage or step left), before any sweep:
//   x[4k + v]      = du_k[v] / s_v   as above
//   x[16 + 4q + v] = x0[q][v] / s_v  (coefficients are mean differences over lengths: the same scale)
//   x[36 .. 55]    = 0
//   x[56 + 2k + d] = slot k's face centre in the cell's own polynomial frame
// Output y[4q + v] = (x* - x0)[q][v] / s_v, returned scales r = s.
template <class T>
DG_HD void mlp_cell_features_prev(int64_t i, const HotView<T>& h, const T* x0, const float* geom, float x[kInP],
                                  float r[4]) {
  double du[4][4], ui[4];
  for (int v = 0; v < 4; v++) ui[v] = h.u[i * 4 + v];
  for (int k = 0; k < 4; k++)
    for (int v = 0; v < 4; v++) du[k][v] = 0.0;
  for (int k = 0; k < h.nfmax && k < 4; k++) {
    if (h.vrMode[aos(i, k, h.nfmax)] != VR_INNER) continue;
    const int64_t j = h.vrNbr[aos(i, k, h.nfmax)];
    for (int v = 0; v < 4; v++) du[k][v] = h.u[j * 4 + v] - ui[v];
  }
  auto clampf = [](double a) { return (float)(a > 1e3 ? 1e3 : (a < -1e3 ? -1e3 : a)); };
  for (int v = 0; v < 4; v++) {
    double m = 0;
    for (int k = 0; k < 4; k++) m = dmax(m, fabs(du[k][v]));
    const double sv = dmax(m, dmax(1e-12 * fabs(ui[v]), 1e-30));
    r[v] = (float)sv;
    for (int k = 0; k < 4; k++) x[4 * k + v] = clampf(du[k][v] / sv);
    for (int q = 0; q < 5; q++) x[16 + 4 * q + v] = clampf((double)x0[i * 20 + 4 * q + v] / sv);
  }
  for (int k = 36; k < 56; k++) x[k] = 0.f;
  for (int k = 0; k < 8; k++) x[56 + k] = geom[i * 8 + k];
}

}  // namespace dg

#if defined(__CUDACC__)
namespace dg {
typedef __nv_bfloat16 bf16;

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct MlpDev {
  const float* P;   // FP32 master parameters [kNParam]
  const bf16* W;    // BF16 weight matrices [kNW]
};

// ---------------------------------------------------------------- inference on the tensor cores (tcgen05)
// 128 rows (cells) per tile, one per thread of a 128-thread CTA.  Each layer is one 128 x N x 64
// product, four tcgen05.mma (kind::f16: BF16 operands in shared memory, FP32 accumulator in
// tensor memory, K = 16 each) issued by one thread and completed on an mbarrier; every thread then
// reads its own accumulator row with tcgen05.ld (warp w owns tensor-memory lanes 32w..32w+31, which
// are rows 32w..32w+31 of the 128-row accumulator), adds the bias, applies SiLU and writes the next
// layer's operand row.  Operands use the K-major, no-swizzle canonical layout: 8-row x 16-byte core
// matrices, core matrices along K 128 B apart (leading byte offset), 8-row groups 1024 B apart
// (stride byte offset), so the K step k0 of an instruction starts 32 k0 / 16 bytes further.
constexpr int kTcRows = 128;
constexpr int kTcCols = 64;  // tensor-memory columns: the widest layer (N = 64, FP32)
struct TcSmem {
  alignas(128) unsigned char W[4][kHid * 64 * 2];  // W1..W4 (W4: 32 rows used), core-matrix layout
  alignas(128) unsigned char A[kTcRows * 64 * 2];  // the current layer's input rows, same layout
  float b[3 * kHid + kOutP];
  uint64_t bar;
  uint32_t tmem;
};

// tensor memory: every resident CTA holds kTcCols of the SM's 512 columns, and an allocation that
// cannot be met waits; the launch keeps at most 4 CTAs per SM (shared memory and registers allow 4)
static_assert(sizeof(TcSmem) > 233472 / 9, "at most 8 CTAs of k_mlp_tc per SM");

// the bias of layer l, entry k, from the FP32 master parameters
__device__ __forceinline__ float tc_bias_s(const float* P, int layer, int k) {
  const int off = layer == 0 ? kOffB1 : layer == 1 ? kOffB2 : layer == 2 ? kOffB3 : kOffB4;
  return P[off + k];
}

// byte offset of element (row, k) of a 64-wide K-major operand in the core-matrix layout
__device__ __forceinline__ uint32_t cm_off(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
// shared-memory matrix descriptor: start address, leading byte offset 128, stride byte offset 1024,
// descriptor version 1, no swizzle (all addresses and offsets in 16-byte units)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M = 128, N
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16 consecutive FP32 columns of this thread's accumulator row
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// SiLU through the identity sigmoid(z) = (1 + tanh(z / 2)) / 2 with the hardware tanh: one
// special-function operation per activation instead of an exponential and a reciprocal (the
// special-function unit bounds this kernel's epilogue); its error (about 2^-11 relative) is below
// the BF16 rounding the activation gets next
__device__ __forceinline__ float silu_tanh(float z) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
  return 0.5f * z * (1.0f + t);
}

constexpr int kTcRowsX = kTcRows;
__device__ __forceinline__ uint32_t cm_off_x(int row, int k) { return cm_off(row, k); }

// one 64-value row of the layer input, as BF16, into the operand buffer
__device__ __forceinline__ void tc_store_row(unsigned char* A, int row, const float* x) {
  for (int kc = 0; kc < 8; kc++) {
    __nv_bfloat162 p[4];
    for (int e = 0; e < 4; e++) p[e] = __floats2bfloat162_rn(x[8 * kc + 2 * e], x[8 * kc + 2 * e + 1]);
    *reinterpret_cast<uint4*>(A + cm_off(row, 8 * kc)) = *reinterpret_cast<uint4*>(p);
  }
}

// inputs and outputs of the tensor-core forward
// Src::kTile: the whole tile is loaded by the CTA together (coalesced), else row by row;
// Dst::kTile: the outputs go through shared memory and leave as one contiguous block
struct TcFeaturesX {  // given features X [n][64]
  static constexpr bool kTile = true;
  const float* X;
  // the 128 x 64 tile starting at row r0 into the operand buffer, 32 B of X per thread and step
  __device__ void load_tile(int64_t r0, int64_t n, unsigned char* A) const {
    for (int e = threadIdx.x; e < kTcRowsX * 8; e += blockDim.x) {
      const int row = e >> 3, kc = e & 7;
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (r0 + row < n) {
        const float4* q = reinterpret_cast<const float4*>(X + (r0 + row) * kIn + 8 * kc);
        const float4 a = q[0], b = q[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
      }
      __nv_bfloat162 p[4];
      for (int j = 0; j < 4; j++) p[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
      *reinterpret_cast<uint4*>(A + cm_off_x(row, 8 * kc)) = *reinterpret_cast<uint4*>(p);
    }
  }
  __device__ void load(int64_t, int64_t, float*, float*) const {}
};
struct TcOutY {  // Y [n][20] = the network output
  static constexpr bool kTile = true;
  float* Y;
  // stage [128][20] FP32 (in the free operand buffer) -> one contiguous store of the tile
  __device__ void store_tile(int64_t r0, int64_t n, const float* stage) const {
    const int64_t m = min((int64_t)kTcRowsX, n - r0) * kOut;
    for (int64_t e = threadIdx.x; e < m; e += blockDim.x) Y[r0 * kOut + e] = stage[e];
  }
  __device__ void store(int64_t, int64_t, const float*, const float*) const {}
};
template <class T, int MODE>
struct TcCellFeatures {  // the warm-start features of cell r (MODE 0: Jacobi extrapolation, 1: previous coefficients)
  static constexpr bool kTile = false;
  HotView<T> h;
  MlpIters<T> it;
  __device__ void load(int64_t r, int64_t n, float x[kInP], float sc[4]) const {
    if (r < n) {
      if (MODE == 0) mlp_cell_features<T>(r, h, it, x, sc);
      else mlp_cell_features_prev<T>(r, h, it.x0, it.geom, x, sc);
    } else {
      for (int k = 0; k < kInP; k++) x[k] = 0.f;
      for (int v = 0; v < 4; v++) sc[v] = 0.f;
    }
  }
  __device__ void load_tile(int64_t, int64_t, unsigned char*) const {}
};
template <class T>
struct TcWarmStart {  // dst = base + y r (base: x2 for MODE 0, x0 for MODE 1)
  static constexpr bool kTile = false;
  const T* x2;
  T* dst;
  __device__ void store(int64_t r, int64_t n, const float* y, const float* sc) const {
    if (r < n)
      for (int o = 0; o < kOut; o++) dst[r * 20 + o] = (T)((double)x2[r * 20 + o] + (double)y[o] * (double)sc[o & 3]);
  }
  __device__ void store_tile(int64_t, int64_t, const float*) const {}
};

template <class Src, class Dst>
__global__ void __launch_bounds__(kTcRows) k_mlp_tc(MlpDev m, Src src, Dst dst, int64_t n, unsigned* flags) {
  extern __shared__ __align__(128) unsigned char raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  // the weights (row-major [N][64] BF16 in global memory) into the core-matrix layout, 16 B at a time
  for (int e = tid; e < (3 * kHid + kOutP) * 8; e += blockDim.x) {
    const int row = e >> 3, kc = e & 7;
    const int layer = row < 3 * kHid ? row / kHid : 3, rl = row - layer * kHid;
    const int woff = layer == 0 ? kWOff1 : layer == 1 ? kWOff2 : layer == 2 ? kWOff3 : kWOff4;
    *reinterpret_cast<uint4*>(S.W[layer] + cm_off(rl, 8 * kc)) =
        *reinterpret_cast<const uint4*>(m.W + woff + rl * 64 + 8 * kc);
  }
  for (int e = tid; e < 3 * kHid + kOutP; e += blockDim.x) {
    const int off = e < kHid ? kOffB1 + e : e < 2 * kHid ? kOffB2 + e - kHid : e < 3 * kHid ? kOffB3 + e - 2 * kHid
                                                                                          : kOffB4 + e - 3 * kHid;
    S.b[e] = m.P[off];
  }
  const uint32_t bar = smem_u32(&S.bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = S.tmem, trow = tbase + ((uint32_t)(warp * 32) << 16);
  const uint32_t aAddr = smem_u32(S.A);
  uint32_t phase = 0;
  bool failed = false;
  for (int64_t tile = blockIdx.x; tile * kTcRows < n && !failed; tile += gridDim.x) {
    const int64_t r = tile * kTcRows + tid;
    float x[kInP], sc[4] = {0.f, 0.f, 0.f, 0.f};
    if constexpr (Src::kTile) {
      src.load_tile(tile * kTcRows, n, S.A);
    } else {
      src.load(r, n, x, sc);
      tc_store_row(S.A, tid, x);
    }
    for (int layer = 0; layer < 4 && !failed; layer++) {
      const int N = layer < 3 ? kHid : kOutP;
      proxy_fence_smem();  // the operand rows written by this thread, to the tensor cores
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t wAddr = smem_u32(S.W[layer]);
        for (int ks = 0; ks < 4; ks++)
          umma_bf16(tbase, umma_desc(aAddr + 256 * ks), umma_desc(wAddr + 256 * ks), layer < 3 ? umma_idesc(kHid)
                                                                                              : umma_idesc(kOutP),
                    ks > 0);
        umma_commit(bar);
      }
      const bool ok = mbar_wait(bar, phase, kWaitLimit);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      tc_fence_after();
      float z[64];
      for (int c0 = 0; c0 < N; c0 += 16) tmem_ld16(trow + c0, z + c0);
      tmem_wait_ld();
      if (layer < 3) {
        for (int k = 0; k < 64; k++) x[k] = silu_tanh(z[k] + S.b[layer * kHid + k]);
        tc_store_row(S.A, tid, x);
      } else {
        float y[kOut];
        for (int o = 0; o < kOut; o++) y[o] = z[o] + S.b[3 * kHid + o];
        if constexpr (Dst::kTile) {  // the operand buffer is free once the last product completed
          float* stage = reinterpret_cast<float*>(S.A);
          for (int o = 0; o < kOut; o++) stage[tid * kOut + o] = y[o];
          __syncthreads();
          dst.store_tile(tile * kTcRows, n, stage);
        } else {
          dst.store(r, n, y, sc);
        }
      }
    }
    tc_fence_before();
    __syncthreads();  // every row is read out before the next tile's products overwrite the accumulator
    tc_fence_after();
  }
  if (failed && tid == 0) {
    atomicOr(flags, kFlagTimeout);
    mbar_wait(bar, phase ^ 1u, kWaitLimit);  // the last commit, if it is still in flight
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTcCols) : "memory");
  }
}

// loss = mean over rows and the 20 outputs of (y - t)^2; gradients accumulate into G
// ---------------------------------------------------------------- training on the tensor cores (tcgen05)
// 128 rows per tile, 512 threads (16 columns of one row each); one CTA per SM holding all 512
// tensor-memory columns:
//   cols   0-191  the pre-activations z1, z2, z3 of the tile (FP32, kept for the backward pass)
//   cols 192-255  the layer-4 output, then each backward product dH = dz W
//   cols 256-511  dW1 .. dW4, accumulated over all of the CTA's tiles (M = 64: output unit u in
//                 tensor-memory lane (u & 15) + 32 (u >> 4), the half-subpartition layout of M = 64)
// Every operand stays in the one layout it is written in, the K-major core-matrix layout of the forward
// products ([rows][64 units], cm_off); the products that need an operand transposed read it as an
// MN-major operand instead (the same bytes: MN-blocks of 8 units 128 B apart, K-blocks of 8 rows 1024 B
// apart), so nothing is copied transposed:
//   forward       z_l  = h_{l-1} W_l^T       A h_{l-1} K-major, B W_l K-major         M 128, N 64 | 32, K 64
//   input grad    dH   = dz_l W_l            A dz_l K-major,    B W_l MN-major         M 128, N 64, K 64 | 32
//   weight grad   dW_l += dz_l^T h_{l-1}     A dz_l MN-major,   B h_{l-1} MN-major     M 64, N 64, K 128
constexpr int kTrCols = 512;
struct TrTcSmem {
  alignas(128) unsigned char Wf[3 * kHid * 128 + kOutP * 128];  // W_l [N][64], core-matrix layout
  alignas(128) unsigned char X[kTcRows * 128];                   // the tile's features [128][64]
  alignas(128) unsigned char H[3][kTcRows * 128];                // h1, h2, h3 [128][64]
  alignas(128) unsigned char DZ[kTcRows * 128];                  // dz_l [128][64] (dz4: units >= 32 zero)
  float gb[3 * kHid + kOutP];                                    // bias gradients of the CTA
  uint64_t bar;
  uint32_t tmem;
  unsigned char pad[8192];  // more than half of an SM's shared memory: one CTA per SM
};
static_assert(sizeof(TrTcSmem) > 233472 / 2, "one CTA per SM: it holds all 512 tensor-memory columns");

// MN-major shared-memory descriptor of the same core-matrix layout: leading byte offset (K-blocks of 8 rows)
// 1024, stride byte offset (MN-blocks of 8 units) 128, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(1024 >> 4) << 16) | ((uint64_t)(128 >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor of kind::f16 with the operands' majors (a_major bit 15, b_major bit 16) and M
__host__ __device__ constexpr uint32_t umma_idesc_mk(int m, int n, bool aMN, bool bMN) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (aMN ? (1u << 15) : 0u) | (bMN ? (1u << 16) : 0u) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
// one butterfly round of a 16-column warp sum: lanes L and L ^ O trade halves of their W columns, each
// keeping the half its bit O selects, summed with the partner's copy of the same columns
template <int W, int O>
__device__ __forceinline__ void tr_bfly(float* v, int lane) {
  const bool up = (lane & O) != 0;
#pragma unroll
  for (int k = 0; k < W; k++) {
    const float send = up ? v[k] : v[k + W], keep = up ? v[k + W] : v[k];
    v[k] = keep + __shfl_xor_sync(0xffffffffu, send, O);
  }
}
// the sums over the warp's 32 rows of 16 column values v (destroyed), added into gb[0 .. 15]: four
// butterfly rounds halve the columns a lane holds (8 + 4 + 2 + 1 shuffles, against 5 per column for
// 16 separate reductions), a last one completes the sum, and 16 lanes add one column each
__device__ __forceinline__ void tr_bias_sum16(float* v, float* gb) {
  const int lane = threadIdx.x & 31;
  tr_bfly<8, 16>(v, lane);
  tr_bfly<4, 8>(v, lane);
  tr_bfly<2, 4>(v, lane);
  tr_bfly<1, 2>(v, lane);
  const float sum = v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
  const int c = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
  if ((lane & 1) == 0) atomicAdd(&gb[c], sum);
}
// 16 values of a row, as BF16, into columns c0 .. c0 + 15 of a 64-wide K-major operand (c0 % 8 == 0)
__device__ __forceinline__ void tc_store16(unsigned char* A, int row, int c0, const float* x) {
#pragma unroll
  for (int h = 0; h < 2; h++) {
    __nv_bfloat162 p[4];
    for (int e = 0; e < 4; e++) p[e] = __floats2bfloat162_rn(x[8 * h + 2 * e], x[8 * h + 2 * e + 1]);
    *reinterpret_cast<uint4*>(A + cm_off(row, c0 + 8 * h)) = *reinterpret_cast<uint4*>(p);
  }
}

// 512 threads: warp w reads tensor-memory lanes 32 (w % 4) .. + 31, i.e. tile rows 32 q + lane (q = w % 4),
// and handles columns 16 g .. 16 g + 15 (g = w / 4) of every 64-wide layer, so the epilogues of a
// tile (bias, activation, operand store, bias-gradient sums) are spread over 16 warps
constexpr int kTrThreads = 512;
__global__ void __launch_bounds__(kTrThreads, 1) k_mlp_train_tc(MlpDev m, const float* X, const float* Tg, int64_t n,
                                                                float invCount, float* G, double* lossAcc,
                                                                unsigned* flags) {
  extern __shared__ __align__(128) unsigned char raw[];
  TrTcSmem& S = *reinterpret_cast<TrTcSmem*>(raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3, g = warp >> 2, row = 32 * q + lane;
  // the weights (row-major [N][64] BF16 in global memory) into the core-matrix layout, 16 B at a time
  for (int e = tid; e < (3 * kHid + kOutP) * 8; e += blockDim.x) {
    const int row = e >> 3, kc = e & 7;
    const int layer = row < 3 * kHid ? row / kHid : 3, rl = row - layer * kHid;
    const int woff = layer == 0 ? kWOff1 : layer == 1 ? kWOff2 : layer == 2 ? kWOff3 : kWOff4;
    *reinterpret_cast<uint4*>(S.Wf + layer * kHid * 128 + cm_off(rl, 8 * kc)) =
        *reinterpret_cast<const uint4*>(m.W + woff + rl * 64 + 8 * kc);
  }
  for (int e = tid; e < 3 * kHid + kOutP; e += blockDim.x) S.gb[e] = 0.f;
  const uint32_t bar = smem_u32(&S.bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kTrCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tb = S.tmem, lane0 = (uint32_t)(q * 32) << 16, col0 = 16u * g;
  const uint32_t aX = smem_u32(S.X), aDZ = smem_u32(S.DZ), aW = smem_u32(S.Wf);
  const uint32_t aH[3] = {smem_u32(S.H[0]), smem_u32(S.H[1]), smem_u32(S.H[2])};
  constexpr uint32_t idFwd64 = umma_idesc_mk(kTcRows, kHid, false, false);
  constexpr uint32_t idFwd32 = umma_idesc_mk(kTcRows, kOutP, false, false);
  constexpr uint32_t idDH = umma_idesc_mk(kTcRows, kHid, false, true);
  constexpr uint32_t idDW = umma_idesc_mk(64, kHid, true, true);
  uint32_t phase = 0;
  bool failed = false, first = true;
  double lossLocal = 0.0;
  // all threads: make the operand writes visible to the tensor cores, then tid 0 issues `issue`
  auto run = [&](auto issue) -> bool {
    proxy_fence_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      issue();
      umma_commit(bar);
    }
    const bool ok = mbar_wait(bar, phase, kWaitLimit);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) return false;
    tc_fence_after();
    return true;
  };
  for (int64_t tile = blockIdx.x; tile * kTcRows < n && !failed; tile += gridDim.x) {
    const int64_t r0 = tile * kTcRows, r = r0 + row;
    // x: coalesced 32-B pieces into the K-major operand
    for (int e = tid; e < kTcRows * 8; e += blockDim.x) {
      const int row = e >> 3, kc = e & 7;
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (r0 + row < n) {
        const float4* q = reinterpret_cast<const float4*>(X + (r0 + row) * kIn + 8 * kc);
        const float4 a = q[0], b = q[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
      }
      __nv_bfloat162 p[4];
      for (int j = 0; j < 4; j++) p[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
      *reinterpret_cast<uint4*>(S.X + cm_off(row, 8 * kc)) = *reinterpret_cast<uint4*>(p);
    }
    // ---- forward: z_l into tensor memory, h_l = SiLU(z_l + b_l) into H[l]
    for (int l = 0; l < 4 && !failed; l++) {
      const uint32_t dcol = l < 3 ? 64u * l : 192u;
      const uint32_t aIn = l == 0 ? aX : aH[l - 1], aWl = aW + (uint32_t)l * kHid * 128;
      if (!run([&] {
            for (int ks = 0; ks < 4; ks++)
              umma_bf16(tb + dcol, umma_desc(aIn + 256 * ks), umma_desc(aWl + 256 * ks), l < 3 ? idFwd64 : idFwd32,
                        ks > 0);
          })) {
        failed = true;
        break;
      }
      if (l < 3) {
        float h[16];
        tmem_ld16(tb + lane0 + dcol + col0, h);
        tmem_wait_ld();
        for (int k = 0; k < 16; k++) h[k] = silu(h[k] + tc_bias_s(m.P, l, col0 + k));
        tc_store16(S.H[l], row, col0, h);
      } else {  // y = z4 + b4, dz4 = 2 (y - t) / count on the 20 outputs (column groups 0 and 1)
        float dz[16];
        for (int k = 0; k < 16; k++) dz[k] = 0.f;
        if (g < 2) {
          float z[16];
          tmem_ld16(tb + lane0 + 192 + col0, z);
          tmem_wait_ld();
          for (int k = 0; k < 16; k++) {
            const int o = col0 + k;
            if (o < kOut && r < n) {
              const float dd = z[k] + tc_bias_s(m.P, 3, o) - Tg[r * kOut + o];
              lossLocal += (double)dd * dd;
              dz[k] = 2.f * dd * invCount;
            }
          }
        }
        tc_store16(S.DZ, row, col0, dz);  // units 32 .. 63 stay zero
        if (g < 2) tr_bias_sum16(dz, S.gb + 3 * kHid + col0);
      }
    }
    // ---- backward: dW_l += dz_l^T h_{l-1}; dH = dz_l W_l; dz_{l-1} = dH SiLU'(z_{l-1} + b_{l-1})
    for (int l = 3; l >= 0 && !failed; l--) {
      const uint32_t aPrev = l > 0 ? aH[l - 1] : aX, aWl = aW + (uint32_t)l * kHid * 128;
      const bool acc = !first;
      if (!run([&] {
            for (int ks = 0; ks < kTcRows / 16; ks++)
              umma_bf16(tb + 256 + 64u * l, umma_desc_mn(aDZ + 2048 * ks), umma_desc_mn(aPrev + 2048 * ks), idDW,
                        acc || ks > 0);
            if (l > 0) {
              const int kst = l == 3 ? kOutP / 16 : kHid / 16;  // K = the layer's output units
              for (int ks = 0; ks < kst; ks++)
                umma_bf16(tb + 192, umma_desc(aDZ + 256 * ks), umma_desc_mn(aWl + 2048 * ks), idDH, ks > 0);
            }
          })) {
        failed = true;
        break;
      }
      if (l > 0) {
        float dh[16], z[16];
        tmem_ld16(tb + lane0 + 192 + col0, dh);
        tmem_ld16(tb + lane0 + 64u * (l - 1) + col0, z);
        tmem_wait_ld();
        for (int k = 0; k < 16; k++)
          dh[k] = r < n ? dh[k] * silu_grad(z[k] + tc_bias_s(m.P, l - 1, col0 + k)) : 0.f;
        tc_store16(S.DZ, row, col0, dh);
        tr_bias_sum16(dh, S.gb + (l - 1) * kHid + col0);
      }
    }
    first = false;
  }
  if (failed && tid == 0) {
    atomicOr(flags, kFlagTimeout);
    mbar_wait(bar, phase ^ 1u, kWaitLimit);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // the CTA's weight gradients and bias gradients into G: dW_l unit u = 16 q + t in lane t < 16 of the
  // warps of lane quarter q, columns 16 g .. 16 g + 15
  if (!failed && !first) {
    const int u = 16 * q + lane;
    const bool mine = lane < 16;
    for (int l = 0; l < 4; l++) {
      const int N = l < 3 ? kHid : kOutP;
      const int woff = l == 0 ? kOffW1 : l == 1 ? kOffW2 : l == 2 ? kOffW3 : kOffW4;
      float gv[16];
      tmem_ld16(tb + lane0 + 256 + 64u * l + col0, gv);
      tmem_wait_ld();
      if (mine && u < N)
        for (int k = 0; k < 16; k++)
          if (gv[k] != 0.f) atomicAdd(&G[woff + u * 64 + col0 + k], gv[k]);
    }
    for (int e = tid; e < 3 * kHid + kOutP; e += blockDim.x) {
      const int off = e < kHid ? kOffB1 + e : e < 2 * kHid ? kOffB2 + e - kHid : e < 3 * kHid ? kOffB3 + e - 2 * kHid
                                                                                            : kOffB4 + e - 3 * kHid;
      if (S.gb[e] != 0.f) atomicAdd(&G[off], S.gb[e]);
    }
  }
  lossLocal = warp_sum_d(lossLocal);
  if ((tid & 31) == 0 && lossLocal != 0.0) atomicAdd(lossAcc, lossLocal);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tb), "r"(kTrCols) : "memory");
  }
}

// Adam (Kingma & Ba) on the FP32 master parameters; padded entries stay zero; refreshes the BF16 copy
__global__ void k_mlp_adam(float* P, float* Mo, float* V, const float* G, bf16* W, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kNParam) return;
  bool pad = false;
  int wi = -1;
  if (e < kOffB1) { pad = (e % kInP) >= kIn; wi = kWOff1 + e; }
  else if (e >= kOffW2 && e < kOffB2) wi = kWOff2 + (e - kOffW2);
  else if (e >= kOffW3 && e < kOffB3) wi = kWOff3 + (e - kOffW3);
  else if (e >= kOffW4 && e < kOffB4) { pad = (e - kOffW4) / kHid >= kOut; wi = kWOff4 + (e - kOffW4); }
  else if (e >= kOffB4) pad = (e - kOffB4) >= kOut;
  if (pad) { P[e] = 0.f; if (wi >= 0) W[wi] = __float2bfloat16(0.f); return; }
  const float g = G[e];
  const float m = b1 * Mo[e] + (1.f - b1) * g, v = b2 * V[e] + (1.f - b2) * g * g;
  Mo[e] = m;
  V[e] = v;
  const float p = P[e] - lr * (m * c1) / (sqrtf(v * c2) + eps);
  P[e] = p;
  if (wi >= 0) W[wi] = __float2bfloat16(p);
}
__global__ void k_mlp_to_bf16(const float* P, bf16* W) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kNParam) return;
  int wi = -1;
  if (e < kOffB1) wi = kWOff1 + e;
  else if (e >= kOffW2 && e < kOffB2) wi = kWOff2 + (e - kOffW2);
  else if (e >= kOffW3 && e < kOffB3) wi = kWOff3 + (e - kOffW3);
  else if (e >= kOffW4 && e < kOffB4) wi = kWOff4 + (e - kOffW4);
  if (wi >= 0) W[wi] = __float2bfloat16(P[e]);
}

}  // namespace dg
#endif
