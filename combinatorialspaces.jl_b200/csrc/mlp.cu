// The learned multigrid smoother: a per-vertex MLP 16 -> 64 -> 64 -> 1 (ReLU) over scale-free
// 1-ring features (the vertex's and its neighbours' residuals over their largest magnitude, the
// couplings a_ij / a_ii, the diagonal margin, the valence).  Its output y gives the correction
// x_i += (s_i / a_ii) y_i, s_i the residual scale, so damped Jacobi is the network y = ω f_0.
//
// Inference runs on the tensor cores: one warp evaluates 32 samples with mma.sync m16n8k16
// (BF16 operands, FP32 accumulation); the first layer's accumulator fragments become the
// second layer's A fragments in registers, and the last layer is a quad shuffle reduction.
//
// Training minimises the energy-norm error left by one smoothing step.  With r = A e and ⋆0 A
// symmetric positive definite, ||e - δ||²_{⋆0 A} = ||e||²_{⋆0 A} + δᵀ ⋆0 A δ - 2 δᵀ ⋆0 r, so every
// (residual, error) pair enters through its residual alone:
//   L = (1/S) Σ_s (δ_sᵀ ⋆0 A δ_s - 2 δ_sᵀ ⋆0 r_s) / n_s,  n_s = Σ_i ⋆0_i r_si² / a_ii,
//   dL/dδ = 2 ⋆0 (A δ - r) / (S n_s).
// The forward pass over every vertex of the fields is the inference kernel; the backward pass
// recomputes the forward in FP32 on the CUDA cores (same BF16 roundings; gradients reach the FP32
// master weights straight through) for a batch of vertex samples, drawn with replacement when the
// fields hold more vertices than the batch; the parameter gradient is reduced in a fixed order;
// Adam updates the masters and refreshes the BF16 copies.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "mlp.cuh"
#include "ops.cuh"

void op_apply_impl(dec_op* op, const void* x, void* y, double alpha, double beta, void* stream);

namespace decb {

// ---------------------------------------------------------------------------------------------
// tensor-core inference
// ---------------------------------------------------------------------------------------------
constexpr int kMlpThreads = 256;  // 8 warps
constexpr int kMlpWarps = kMlpThreads / 32;
constexpr int kTile = 32;         // samples per warp tile (two m16 row tiles)
// Shared-memory row strides in BF16 elements, padded so that the fragment loads of a warp hit
// 32 distinct banks: 12 words per feature / W1 row, 36 words per W2 row.
constexpr int kXsStride = 24, kW1Stride = 24, kW2Stride = 72;

struct MlpSmem {
  __align__(16) __nv_bfloat16 w1[kMlpH * kW1Stride];
  __align__(16) __nv_bfloat16 w2[kMlpH * kW2Stride];
  float b1[kMlpH], b2[kMlpH], w3[kMlpH], b3;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ void load_weights(MlpSmem& sm, const MlpWeights& w) {
  for (int i = threadIdx.x; i < kMlpH * kMlpIn; i += blockDim.x) sm.w1[(i / kMlpIn) * kW1Stride + i % kMlpIn] = w.w1[i];
  for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) sm.w2[(i / kMlpH) * kW2Stride + i % kMlpH] = w.w2[i];
  for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
    sm.b1[i] = w.b1[i];
    sm.b2[i] = w.b2[i];
    sm.w3[i] = w.w3[i];
  }
  if (threadIdx.x == 0) sm.b3 = w.b3[0];
  __syncthreads();
}

// Stores one sample's 16 features as a BF16 row of the warp's tile.
__device__ __forceinline__ void store_row(__nv_bfloat16* xs, int row, const float (&f)[16]) {
  uint4 lo, hi;
  lo.x = pack_bf16(f[0], f[1]);
  lo.y = pack_bf16(f[2], f[3]);
  lo.z = pack_bf16(f[4], f[5]);
  lo.w = pack_bf16(f[6], f[7]);
  hi.x = pack_bf16(f[8], f[9]);
  hi.y = pack_bf16(f[10], f[11]);
  hi.z = pack_bf16(f[12], f[13]);
  hi.w = pack_bf16(f[14], f[15]);
  uint4* p = reinterpret_cast<uint4*>(xs + row * kXsStride);
  p[0] = lo;
  p[1] = hi;
}

// The MLP on one warp tile of 32 samples (rows of xs).  Returns, in every lane, y of the lane's
// own row.
__device__ __forceinline__ float mlp_tile32(const MlpSmem& sm, const __nv_bfloat16* xs) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t* X = reinterpret_cast<const uint32_t*>(xs);
  const uint32_t* W1 = reinterpret_cast<const uint32_t*>(sm.w1);
  const uint32_t* W2 = reinterpret_cast<const uint32_t*>(sm.w2);
  constexpr int XW = kXsStride / 2, W1W = kW1Stride / 2, W2W = kW2Stride / 2;  // words per row
  uint32_t a[2][4];
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int r0 = 16 * m + g;
    a[m][0] = X[r0 * XW + t];
    a[m][1] = X[(r0 + 8) * XW + t];
    a[m][2] = X[r0 * XW + t + 4];
    a[m][3] = X[(r0 + 8) * XW + t + 4];
  }
  // layer 1: z1 = W1 x + b1 on 8 column tiles of 8 units; relu + BF16 pack into layer-2 A
  uint32_t a2[2][4][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t b0 = W1[(8 * j + g) * W1W + t], b1 = W1[(8 * j + g) * W1W + t + 4];
    const float bb0 = sm.b1[8 * j + 2 * t], bb1 = sm.b1[8 * j + 2 * t + 1];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      float c[4] = {bb0, bb1, bb0, bb1};
      mma16816(c, a[m], b0, b1);
      const uint32_t lo = pack_bf16(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f));
      const uint32_t hi = pack_bf16(fmaxf(c[2], 0.f), fmaxf(c[3], 0.f));
      if ((j & 1) == 0) {
        a2[m][j >> 1][0] = lo;
        a2[m][j >> 1][1] = hi;
      } else {
        a2[m][j >> 1][2] = lo;
        a2[m][j >> 1][3] = hi;
      }
    }
  }
  // layers 2 and 3: y = w3 · relu(W2 h1 + b2) + b3, two column tiles at a time (four
  // independent accumulator chains per k step)
  float p[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
  for (int jp = 0; jp < 4; ++jp) {
    float c[2][2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int jt = 2 * jp + u;
      const float bb0 = sm.b2[8 * jt + 2 * t], bb1 = sm.b2[8 * jt + 2 * t + 1];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        c[u][m][0] = bb0;
        c[u][m][1] = bb1;
        c[u][m][2] = bb0;
        c[u][m][3] = bb1;
      }
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int jt = 2 * jp + u;
        const uint32_t b0 = W2[(8 * jt + g) * W2W + 8 * kk + t], b1 = W2[(8 * jt + g) * W2W + 8 * kk + t + 4];
#pragma unroll
        for (int m = 0; m < 2; ++m) mma16816(c[u][m], a2[m][kk], b0, b1);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int jt = 2 * jp + u;
      const float w0 = sm.w3[8 * jt + 2 * t], w1 = sm.w3[8 * jt + 2 * t + 1];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        p[m][0] += fmaxf(c[u][m][0], 0.f) * w0 + fmaxf(c[u][m][1], 0.f) * w1;
        p[m][1] += fmaxf(c[u][m][2], 0.f) * w0 + fmaxf(c[u][m][3], 0.f) * w1;
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      p[m][h] += __shfl_xor_sync(0xffffffffu, p[m][h], 1);
      p[m][h] += __shfl_xor_sync(0xffffffffu, p[m][h], 2);
    }
  // row 16m + 8h + g' lives in quad g' as p[m][h]; lane L takes row L
  const int src = (lane & 7) * 4, m = lane >> 4, h = (lane >> 3) & 1;
  const float v00 = __shfl_sync(0xffffffffu, p[0][0], src), v01 = __shfl_sync(0xffffffffu, p[0][1], src);
  const float v10 = __shfl_sync(0xffffffffu, p[1][0], src), v11 = __shfl_sync(0xffffffffu, p[1][1], src);
  const float v = m == 0 ? (h == 0 ? v00 : v01) : (h == 0 ? v10 : v11);
  return v + sm.b3;
}

// y = MLP(x) for n samples of 16 FP32 features (tensor cores).
__global__ void __launch_bounds__(kMlpThreads) k_mlp_eval_tc(int64_t n, const float* __restrict__ x,
                                                             float* __restrict__ y, MlpWeights w) {
  __shared__ MlpSmem sm;
  __shared__ __align__(16) __nv_bfloat16 xs[kMlpWarps][kTile * kXsStride];
  load_weights(sm, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  for (int64_t tile = (int64_t)blockIdx.x * kMlpWarps + warp; tile < ntiles; tile += (int64_t)gridDim.x * kMlpWarps) {
    const int64_t q = tile * kTile + lane;
    float f[16];
    if (q < n) {
      const float4* src = reinterpret_cast<const float4*>(x + q * 16);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float4 t4 = src[v];
        f[4 * v] = t4.x;
        f[4 * v + 1] = t4.y;
        f[4 * v + 2] = t4.z;
        f[4 * v + 3] = t4.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    store_row(xs[warp], lane, f);
    __syncwarp();
    const float yv = mlp_tile32(sm, xs[warp]);
    if (q < n) y[q] = yv;
    __syncwarp();
  }
}

// Per-row feature table of a multigrid level (split operator: diagonal + W off-diagonal slots in
// the reference's column order, real slots first, padding = own column with value 0):
// tab[2i] = (c0, c1, c2, c3), tab[2i+1] = (c4, c5, 1 - Σ_j |a_ij| / a_ii, nn / 6) with
// c_s = a_ij / a_ii of the first nn = min(6, real slots) slots, zero beyond; the same float
// arithmetic as the per-sample feature function.
__global__ void k_mlp_table(int n, int W, const int32_t* __restrict__ col, const double* __restrict__ off,
                            const double* __restrict__ diag, float4* __restrict__ tab) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float di = (float)diag[i];
    float cp[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, sabs = 0.f;
    int nn = 0;
    for (int s = 0; s < W; ++s) {
      const int c = col[(size_t)i * W + s];
      const float o = (float)off[(size_t)i * W + s];
      if (c == i && o == 0.f) continue;
      sabs += fabsf(o);
      if (nn < 6) cp[nn++] = o / di;
    }
    tab[2 * (size_t)i] = make_float4(cp[0], cp[1], cp[2], cp[3]);
    tab[2 * (size_t)i + 1] = make_float4(cp[4], cp[5], 1.f - sabs / di, (float)nn * (1.0f / 6.0f));
  }
}

void build_mlp_table(int n, int W, const int32_t* col, const double* off, const double* diag, DArr<float4>& tab) {
  tab.alloc(2 * (size_t)n);
  k_mlp_table<<<grid_for(n, 256), 256>>>(n, W, col, off, diag, tab.p);
  DEC_CHECK_LAUNCH();
}

// Learned smoothing step on a multigrid level (panel layout [panel][row][K]):
// out = x + (s_i / a_ii) MLP(features(r)), x taken as zero when zero_x.  The coupling features
// come from the level's table; the residual features are gathered per sample.
template <class T, int K>
__global__ void __launch_bounds__(kMlpThreads, 3) k_mlp_smooth(MlpWeights w, int n, int W, const int32_t* __restrict__ col,
                                                            const float4* __restrict__ tab, const T* __restrict__ diag,
                                                            const T* __restrict__ r, const T* __restrict__ x,
                                                            int zero_x, T* __restrict__ out, size_t pstride) {
  __shared__ MlpSmem sm;
  __shared__ __align__(16) __nv_bfloat16 xs[kMlpWarps][kTile * kXsStride];
  load_weights(sm, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t po = (size_t)blockIdx.y * pstride;
  const int64_t nq = (int64_t)n * K;
  const int64_t ntiles = (nq + kTile - 1) / kTile;
  for (int64_t tile = (int64_t)blockIdx.x * kMlpWarps + warp; tile < ntiles; tile += (int64_t)gridDim.x * kMlpWarps) {
    const int64_t q = tile * kTile + lane;
    float f[16];
    float dsc = 0.f;
    T xv = T(0);
    if (q < nq) {
      const int i = (int)(q / K), k = (int)(q % K);
      // every slot's index and residual are loaded without waiting for the valence (padding
      // slots hold the row itself), then the slots past it are zeroed
      int cj[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) cj[j] = j < W ? col[(size_t)i * W + j] : i;
      float rv[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) rv[j] = (float)r[po + (size_t)cj[j] * K + k];
      const float4 t0 = tab[2 * (size_t)i], t1 = tab[2 * (size_t)i + 1];
      const int nn = __float2int_rn(t1.w * 6.0f);
      const float ri = (float)r[po + q];
      float nb[6];
      float s = fabsf(ri);
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        nb[j] = j < nn ? rv[j] : 0.f;
        s = fmaxf(s, fabsf(nb[j]));
      }
      if (s == 0.0f) s = 1.0f;
      const float inv = 1.0f / s;
      f[0] = ri * inv;
#pragma unroll
      for (int j = 0; j < 6; ++j) f[1 + j] = nb[j] * inv;
      f[7] = t0.x;
      f[8] = t0.y;
      f[9] = t0.z;
      f[10] = t0.w;
      f[11] = t1.x;
      f[12] = t1.y;
      f[13] = t1.z;
      f[14] = t1.w;
      f[15] = 0.0f;
      dsc = s / (float)diag[i];
      if (!zero_x) xv = x[po + q];
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    store_row(xs[warp], lane, f);
    __syncwarp();
    const float yv = mlp_tile32(sm, xs[warp]);
    if (q < nq) out[po + q] = xv + (T)(dsc * yv);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// tcgen05 inference (sm_100a).  One persistent CTA of 1024 threads per SM runs eight independent
// tile chains, one per warpgroup.  A warpgroup takes 128 samples at a time (one per thread and
// TMEM lane) through
//   features -> A1 (128 x 16, shared)   MMA1: D = A1 W1ᵀ           (the warpgroup's 64 TMEM columns)
//   D + b1, ReLU, BF16 -> A2 (128 x 64)  MMA2: D = Σ_s A2_s W2_sᵀ   (the same columns)
//   y = b3 + Σ_j w3_j ReLU(D_j + b2_j)   (FP32, per thread; even and odd j in two lanes)
// with its own shared-memory stages, mbarrier and named barrier, so eight chains are in flight
// per SM (the whole 512-column TMEM) and one chain's gathers and epilogues overlap another's
// MMAs.  W1 and W2 are staged once per CTA; b1, b2, w3 and b3 come by value in the kernel
// parameters, so the epilogues take them as constant operands (shared-memory broadcast loads of
// them had kept the load/store pipe 72% busy).  The epilogues use packed FP32 pairs.  The operands are BF16 in the canonical
// K-major layout without swizzle (8-row groups of 16-byte core rows: byte (r / 8) * SBO +
// (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, SBO = K / 8 * 128); one elected thread of the
// warpgroup issues tcgen05.mma.cta_group::1.kind::f16 (FP32 accumulation) and commits to the
// warpgroup's mbarrier; every thread reads its own TMEM lane in 16-column chunks, the next
// chunk's load in flight while the current one is used.
// Every mbarrier wait is bounded: on time-out the warpgroup agrees (bar.red.and), waits once more
// (bounded) for its MMA in flight, sets *err and leaves its loop; the CTA then frees its TMEM and
// returns.
// ---------------------------------------------------------------------------------------------
constexpr int kTcRows = 128;                     // samples per tile: one warpgroup
constexpr int kTcGroups = 8;                     // tile chains per CTA
constexpr int kTcThreads = kTcRows * kTcGroups;  // 1024
constexpr uint32_t kTcCols = 64 * kTcGroups;     // TMEM columns of the CTA

struct __align__(128) TcGroup {
  __nv_bfloat16 a1[kTcRows * kMlpIn];  // 4 KB
  __nv_bfloat16 a2[kTcRows * kMlpH];   // 16 KB
};
struct __align__(128) TcSmem {
  __nv_bfloat16 w1[kMlpH * kMlpIn];
  __nv_bfloat16 w2[kMlpH * kMlpH];
  // The biases as an MMA: ones (128 x 16, columns 0..2 one, the rest zero) times bb1 / bb2 (64 x 16,
  // row j = the exact three-part BF16 split hi + mid + lo of b1_j / b2_j) puts b into the
  // accumulator before the layer's products add onto it.
  __nv_bfloat16 ones[kTcRows * kMlpIn];
  __nv_bfloat16 bb1[kMlpH * kMlpIn];
  __nv_bfloat16 bb2[kMlpH * kMlpIn];
  uint32_t tmem;
  uint64_t mbar[kTcGroups];
  TcGroup g[kTcGroups];
};
// dynamic shared memory per CTA (one CTA per SM), with slack to align the struct to 128 bytes
constexpr size_t kTcSmemBytes = sizeof(TcSmem) + 128;

__device__ __forceinline__ TcSmem& tc_smem(unsigned char* raw) {
  return *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127));
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// byte offset of element (r, k) of a K-major no-swizzle operand with K columns
__device__ __forceinline__ uint32_t kmaj(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// shared-memory matrix descriptor: start >> 4, LBO >> 4 at 16, SBO >> 4 at 32, version 1 at 46,
// no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: F32 accumulator, BF16 A and B, both K-major, N = 64, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(64 >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(acc));
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (int it = 0; it < (1 << 20); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// 16 consecutive TMEM columns of this thread's lane; the registers are valid after tc_wait16
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// waits for this thread's TMEM loads; the registers are operands, so no use of them moves above it
__device__ __forceinline__ void tc_wait16(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// the warpgroup's named barrier (ids 1..8; 0 is __syncthreads)
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool group_all(int id, bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"((uint32_t)v), "r"(id)
      : "memory");
  return out != 0;
}

// Writes one sample's 16 features (row r of A1).
__device__ __forceinline__ void tc_store_features(__nv_bfloat16* a1, int r, const float (&f)[16]) {
  uint4 lo, hi;
  lo.x = pack_bf16(f[0], f[1]);
  lo.y = pack_bf16(f[2], f[3]);
  lo.z = pack_bf16(f[4], f[5]);
  lo.w = pack_bf16(f[6], f[7]);
  hi.x = pack_bf16(f[8], f[9]);
  hi.y = pack_bf16(f[10], f[11]);
  hi.z = pack_bf16(f[12], f[13]);
  hi.w = pack_bf16(f[14], f[15]);
  char* base = reinterpret_cast<char*>(a1);
  *reinterpret_cast<uint4*>(base + kmaj(r, 0, kMlpIn)) = lo;
  *reinterpret_cast<uint4*>(base + kmaj(r, 8, kMlpIn)) = hi;
}

// b = hi + mid + lo exactly (each part the round-to-nearest BF16 of what the previous ones leave:
// 8 of FP32's 24 significant bits per part), part k of value v.
__device__ __forceinline__ __nv_bfloat16 bf16_part(float v, int k) {
  const __nv_bfloat16 hi = __float2bfloat16_rn(v);
  if (k == 0) return hi;
  const float r1 = v - __bfloat162float(hi);
  const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
  if (k == 1) return mid;
  return __float2bfloat16_rn(r1 - __bfloat162float(mid));
}

__device__ void tc_setup(TcSmem& sm, const MlpWeights& w) {
  char* w1 = reinterpret_cast<char*>(sm.w1);
  char* w2 = reinterpret_cast<char*>(sm.w2);
  char* ones = reinterpret_cast<char*>(sm.ones);
  char* bb1 = reinterpret_cast<char*>(sm.bb1);
  char* bb2 = reinterpret_cast<char*>(sm.bb2);
  for (int i = threadIdx.x; i < kTcRows * kMlpIn; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16*>(ones + kmaj(i / kMlpIn, i % kMlpIn, kMlpIn)) =
        __float2bfloat16_rn(i % kMlpIn < 3 ? 1.f : 0.f);
  for (int i = threadIdx.x; i < kMlpH * kMlpIn; i += blockDim.x) {
    const int j = i / kMlpIn, k = i % kMlpIn;
    *reinterpret_cast<__nv_bfloat16*>(bb1 + kmaj(j, k, kMlpIn)) =
        k < 3 ? bf16_part(w.hs.b1[j], k) : __float2bfloat16_rn(0.f);
    *reinterpret_cast<__nv_bfloat16*>(bb2 + kmaj(j, k, kMlpIn)) =
        k < 3 ? bf16_part(w.hs.b2[j], k) : __float2bfloat16_rn(0.f);
  }
  for (int i = threadIdx.x; i < kMlpH * kMlpIn; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16*>(w1 + kmaj(i / kMlpIn, i % kMlpIn, kMlpIn)) = w.w1[i];
  for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16*>(w2 + kmaj(i / kMlpH, i % kMlpH, kMlpH)) = w.w2[i];
  if (threadIdx.x == 0) {
    for (int g = 0; g < kTcGroups; ++g)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.mbar[g])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {  // warp 0 allocates the accumulator columns of all eight chains
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ void tc_teardown(TcSmem& sm) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem), "r"(kTcCols));
}

// Packed FP32 pairs (.f32x2, two IEEE round-to-nearest lanes per instruction).
__device__ __forceinline__ uint64_t f2(uint32_t lo, uint32_t hi) { return ((uint64_t)hi << 32) | lo; }
__device__ __forceinline__ uint64_t f2(float lo, float hi) { return f2(__float_as_uint(lo), __float_as_uint(hi)); }
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ float lo_of(uint64_t v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float hi_of(uint64_t v) { return __uint_as_float((uint32_t)(v >> 32)); }

// Layer-1 epilogue of one 16-column chunk: A2[r, c0 .. c0+15] = bf16(ReLU(D)), D = b1 + A1 W1ᵀ (the
// bias is in the accumulator), the ReLU and the round-to-nearest BF16 pair in one conversion (a NaN
// stays NaN there, where max(x, 0) gave 0).
__device__ __forceinline__ void tc_epi1(char* a2, int r, int c0, const uint32_t (&z)[16]) {
  uint32_t pk[8];
#pragma unroll
  for (int j = 0; j < 8; ++j)
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;"
        : "=r"(pk[j])
        : "f"(__uint_as_float(z[2 * j + 1])), "f"(__uint_as_float(z[2 * j])));
  *reinterpret_cast<uint4*>(a2 + kmaj(r, c0, kMlpH)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  *reinterpret_cast<uint4*>(a2 + kmaj(r, c0 + 8, kMlpH)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
}
// Layer-3 partial sums of one chunk, two lanes: acc.lo += w3_j ReLU(D_j) over even j, acc.hi over
// odd j, D = b2 + A2 W2ᵀ.
__device__ __forceinline__ void tc_epi2(const MlpSmall& hs, int c0, const uint32_t (&z)[16], uint64_t& acc) {
#pragma unroll
  for (int j = 0; j < 16; j += 2) {
    const uint64_t h = f2(fmaxf(__uint_as_float(z[j]), 0.f), fmaxf(__uint_as_float(z[j + 1]), 0.f));
    acc = fma2(f2(hs.w3[c0 + j], hs.w3[c0 + j + 1]), h, acc);
  }
}

// The MLP on warpgroup g's tile (A1 written by every thread of the group): y of this thread's row,
// or false on time-out.
__device__ __forceinline__ bool tc_tile(TcSmem& sm, const MlpSmall& hs, int g, int r, uint32_t& phase, float& y) {
  const int bar = 1 + g;
  const uint32_t mbar = smem_u32(&sm.mbar[g]);
  const uint32_t dcol = sm.tmem + 64u * g;
  const uint32_t lane = dcol + ((uint32_t)(r & ~31) << 16);
  TcGroup& G = sm.g[g];
  fence_async_smem();
  tc_fence_before();
  group_sync(bar);
  if (r == 0) {
    tc_fence_after();
    tc_mma(dcol, smem_desc(smem_u32(sm.ones), 128, 256), smem_desc(smem_u32(sm.bb1), 128, 256), 0);
    tc_mma(dcol, smem_desc(smem_u32(G.a1), 128, 256), smem_desc(smem_u32(sm.w1), 128, 256), 1);
    tc_commit(mbar);
  }
  // one thread polls the MMA's mbarrier; the others block on the named barrier, which hands them its
  // result and orders their TMEM reads after the wait (tcgen05.fence::after_thread_sync below)
  bool ok = group_all(bar, r == 0 ? mbar_wait(mbar, phase) : true);
  if (!ok) {  // one more bounded wait for the MMA in flight before the TMEM is freed
    if (r == 0) mbar_wait(mbar, phase);
    return false;
  }
  phase ^= 1;
  tc_fence_after();
  char* a2 = reinterpret_cast<char*>(G.a2);
  uint32_t za[16], zb[16];
  tc_ld16(lane, za);
  tc_wait16(za);
  tc_ld16(lane + 16, zb);
  tc_epi1(a2, r, 0, za);
  tc_wait16(zb);
  tc_ld16(lane + 32, za);
  tc_epi1(a2, r, 16, zb);
  tc_wait16(za);
  tc_ld16(lane + 48, zb);
  tc_epi1(a2, r, 32, za);
  tc_wait16(zb);
  tc_epi1(a2, r, 48, zb);
  fence_async_smem();
  tc_fence_before();
  group_sync(bar);  // every lane has read D1 and written its A2 row
  if (r == 0) {
    tc_fence_after();
    tc_mma(dcol, smem_desc(smem_u32(sm.ones), 128, 256), smem_desc(smem_u32(sm.bb2), 128, 256), 0);
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
      tc_mma(dcol, smem_desc(smem_u32(G.a2) + 256 * ks, 128, 1024), smem_desc(smem_u32(sm.w2) + 256 * ks, 128, 1024),
             1u);
    tc_commit(mbar);
  }
  ok = group_all(bar, r == 0 ? mbar_wait(mbar, phase) : true);
  if (!ok) {
    if (r == 0) mbar_wait(mbar, phase);
    return false;
  }
  phase ^= 1;
  tc_fence_after();
  uint64_t acc = 0;  // two FP32 zeros
  tc_ld16(lane, za);
  tc_wait16(za);
  tc_ld16(lane + 16, zb);
  tc_epi2(hs, 0, za, acc);
  tc_wait16(zb);
  tc_ld16(lane + 32, za);
  tc_epi2(hs, 16, zb, acc);
  tc_wait16(za);
  tc_ld16(lane + 48, zb);
  tc_epi2(hs, 32, za, acc);
  tc_wait16(zb);
  tc_epi2(hs, 48, zb, acc);
  y = hs.b3 + (lo_of(acc) + hi_of(acc));
  return true;
}

// y = MLP(x) for n samples of 16 FP32 features (tcgen05).
__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_eval_tcg(int64_t n, const float* __restrict__ x,
                                                              float* __restrict__ y, MlpWeights w, int* err) {
  extern __shared__ unsigned char tc_raw[];
  TcSmem& sm = tc_smem(tc_raw);
  tc_setup(sm, w);
  const int g = threadIdx.x / kTcRows, rr = threadIdx.x % kTcRows;
  uint32_t phase = 0;
  const int64_t ntiles = (n + kTcRows - 1) / kTcRows;
  for (int64_t tile = (int64_t)blockIdx.x * kTcGroups + g; tile < ntiles; tile += (int64_t)gridDim.x * kTcGroups) {
    const int64_t q = tile * kTcRows + rr;
    float f[16];
    if (q < n) {
      const float4* src = reinterpret_cast<const float4*>(x + q * 16);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float4 t4 = src[v];
        f[4 * v] = t4.x;
        f[4 * v + 1] = t4.y;
        f[4 * v + 2] = t4.z;
        f[4 * v + 3] = t4.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    tc_store_features(sm.g[g].a1, rr, f);
    float yv;
    if (!tc_tile(sm, w.hs, g, rr, phase, yv)) {
      if (rr == 0) atomicExch(err, 1);
      break;
    }
    if (q < n) y[q] = yv;
  }
  tc_teardown(sm);
}

// Learned smoothing step with the tcgen05 MLP (same features and update as k_mlp_smooth).
template <class T, int K>
__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_smooth_tcg(MlpWeights w, int n, int W,
                                                                const int32_t* __restrict__ col,
                                                                const float4* __restrict__ tab,
                                                                const T* __restrict__ diag, const T* __restrict__ r,
                                                                const T* __restrict__ x, int zero_x,
                                                                T* __restrict__ out, size_t pstride, int np,
                                                                int* err) {
  extern __shared__ unsigned char tc_raw[];
  TcSmem& sm = tc_smem(tc_raw);
  tc_setup(sm, w);
  const int g = threadIdx.x / kTcRows, rr = threadIdx.x % kTcRows;
  uint32_t phase = 0;
  const int64_t nq = (int64_t)n * K;
  // 32-bit tile arithmetic (the launch checks that the tiles fit): one panel / offset division per
  // tile instead of a 64-bit one
  const uint32_t tiles_per_panel = (uint32_t)((nq + kTcRows - 1) / kTcRows);
  const uint32_t ntiles = tiles_per_panel * (uint32_t)np;
  for (uint32_t tile = blockIdx.x * kTcGroups + g; tile < ntiles; tile += gridDim.x * kTcGroups) {
    const uint32_t panel = tile / tiles_per_panel;
    const size_t po = (size_t)panel * pstride;
    const int64_t q = (int64_t)(tile - panel * tiles_per_panel) * kTcRows + rr;
    float f[16];
    float dsc = 0.f;
    T xv = T(0);
    if (q < nq) {
      const int i = (int)(q / K), k = (int)(q % K);
      // every slot's index and residual are loaded without waiting for the valence (padding
      // slots hold the row itself), then the slots past it are zeroed
      int cj[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) cj[j] = j < W ? col[(size_t)i * W + j] : i;
      float rv[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) rv[j] = (float)r[po + (size_t)cj[j] * K + k];
      const float4 t0 = tab[2 * (size_t)i], t1 = tab[2 * (size_t)i + 1];
      const int nn = __float2int_rn(t1.w * 6.0f);
      const float ri = (float)r[po + q];
      float nb[6];
      float s = fabsf(ri);
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        nb[j] = j < nn ? rv[j] : 0.f;
        s = fmaxf(s, fabsf(nb[j]));
      }
      if (s == 0.0f) s = 1.0f;
      const float inv = 1.0f / s;
      f[0] = ri * inv;
#pragma unroll
      for (int j = 0; j < 6; ++j) f[1 + j] = nb[j] * inv;
      f[7] = t0.x;
      f[8] = t0.y;
      f[9] = t0.z;
      f[10] = t0.w;
      f[11] = t1.x;
      f[12] = t1.y;
      f[13] = t1.z;
      f[14] = t1.w;
      f[15] = 0.0f;
      dsc = s / (float)diag[i];
      if (!zero_x) xv = x[po + q];
    } else {
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) f[k2] = 0.f;
    }
    tc_store_features(sm.g[g].a1, rr, f);
    float yv;
    if (!tc_tile(sm, w.hs, g, rr, phase, yv)) {
      if (rr == 0) atomicExch(err, 1);
      break;
    }
    if (q < nq) out[po + q] = xv + (T)(dsc * yv);
  }
  tc_teardown(sm);
}

static unsigned tc_grid(long long tiles) {
  const long long ctas = (tiles + kTcGroups - 1) / kTcGroups;
  return (unsigned)std::max<long long>(1, std::min<long long>(ctas, (long long)num_sms()));
}

// The tcgen05 kernels' shared memory exceeds 48 KB, which needs each kernel's opt-in.
template <class F>
static void tc_opt_in(F* kernel) {
  DEC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemBytes));
}

template <class T, int K>
void launch_mlp_smooth(const MlpWeights& w, int n, int W, const int32_t* col, const float4* tab, const T* diag,
                       const T* r, const T* x, int zero_x, T* out, int np, cudaStream_t s) {
  if (w.engine == 1) {
    const long long tiles = ((long long)n * K + kTcRows - 1) / kTcRows * np;
    require(tiles < (1LL << 31), "mlp: too many sample tiles for one launch");
    k_mlp_smooth_tcg<T, K><<<tc_grid(tiles), kTcThreads, kTcSmemBytes, s>>>(w, n, W, col, tab, diag, r, x, zero_x,
                                                                          out, (size_t)n * K, np, w.err);
    DEC_CHECK_LAUNCH();
    return;
  }
  const long long tiles = ((long long)n * K + kTile - 1) / kTile;
  const long long want = (tiles + kMlpWarps - 1) / kMlpWarps;
  const long long cap = std::max<long long>(1, (long long)num_sms() * 4 / std::max(1, np));
  dim3 grid((unsigned)std::max<long long>(1, std::min(want, cap)), np);
  k_mlp_smooth<T, K><<<grid, kMlpThreads, 0, s>>>(w, n, W, col, tab, diag, r, x, zero_x, out, (size_t)n * K);
  DEC_CHECK_LAUNCH();
}

// Opts every tcgen05 kernel into its shared memory on the current device.
void tc_opt_in_all() {
  tc_opt_in(k_mlp_eval_tcg);
#define DEC_OPT(T, K) tc_opt_in(k_mlp_smooth_tcg<T, K>);
  DEC_OPT(float, 1) DEC_OPT(float, 2) DEC_OPT(float, 4) DEC_OPT(float, 8) DEC_OPT(float, 16) DEC_OPT(float, 32)
  DEC_OPT(double, 1) DEC_OPT(double, 2) DEC_OPT(double, 4) DEC_OPT(double, 8) DEC_OPT(double, 16)
  DEC_OPT(double, 32)
#undef DEC_OPT
}

#define DEC_INST(T, K)                                                                                             \
  template void launch_mlp_smooth<T, K>(const MlpWeights&, int, int, const int32_t*, const float4*, const T*, \
                                        const T*, const T*, int, T*, int, cudaStream_t);
DEC_INST(float, 1) DEC_INST(float, 2) DEC_INST(float, 4) DEC_INST(float, 8) DEC_INST(float, 16) DEC_INST(float, 32)
DEC_INST(double, 1) DEC_INST(double, 2) DEC_INST(double, 4) DEC_INST(double, 8) DEC_INST(double, 16)
DEC_INST(double, 32)
#undef DEC_INST

// ---------------------------------------------------------------------------------------------
// CUDA-core forward (FP32, the inference roundings) and the training kernels
// ---------------------------------------------------------------------------------------------
__device__ float mlp_forward_cc(const float* f, const __nv_bfloat16* __restrict__ w1b,
                                const __nv_bfloat16* __restrict__ w2b, const float* __restrict__ p) {
  float x0[kMlpIn], h1[kMlpH];
  for (int k = 0; k < kMlpIn; ++k) x0[k] = __bfloat162float(__float2bfloat16_rn(f[k]));
  for (int j = 0; j < kMlpH; ++j) {
    float s = p[kOffB1 + j];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) s += __bfloat162float(w1b[j * kMlpIn + k]) * x0[k];
    h1[j] = __bfloat162float(__float2bfloat16_rn(fmaxf(s, 0.f)));
  }
  float y = p[kOffB3];
  for (int j = 0; j < kMlpH; ++j) {
    float s = p[kOffB2 + j];
    for (int i = 0; i < kMlpH; ++i) s += __bfloat162float(w2b[j * kMlpH + i]) * h1[i];
    y += p[kOffW3 + j] * fmaxf(s, 0.f);
  }
  return y;
}

__global__ void k_mlp_eval_cc(int64_t n, const float* __restrict__ x, float* __restrict__ y,
                              const __nv_bfloat16* __restrict__ w1b, const __nv_bfloat16* __restrict__ w2b,
                              const float* __restrict__ p) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    y[q] = mlp_forward_cc(x + q * 16, w1b, w2b, p);
}

// Activations of the backward batch, structure of arrays [row][batch]: x0 (16 rows),
// h1 = bf16(relu(z1)) (64), relu(z2) (64), dz1 (64), dz2 (64).
constexpr int kActX0 = 0, kActH1 = 16, kActR2 = 80, kActDz1 = 144, kActDz2 = 208, kActRows = 272;

// (a, b) as BF16 pairs hi (round to nearest) and lo (the remainders rounded): hi + lo keeps 16 of
// FP32's 24 significant bits.
__device__ __forceinline__ void split_pair(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = pack_bf16(a - __low2float(h), b - __high2float(h));
}

// ---- backward on the tensor cores -----------------------------------------------------------
// A warp takes 32 samples (rows of its feature tile xs, lane L's sample in row L, dL/dy d in lane L)
// through the forward of mlp_tile32 (mma.sync m16n8k16, the inference roundings: x0 and h1 BF16,
// FP32 accumulation), keeping the ReLU masks as bits, and the backward
//   dz2 = d w3 [z2 > 0],  dh1 = W2ᵀ dz2 (mma.sync: dz2 as hi + lo BF16 A fragments against W2ᵀ),
//   dz1 = dh1 [z1 > 0],
// and stores the batch columns jbase .. jbase + 31 of the activations x0, h1, relu(z2), dz1, dz2
// (structure of arrays [row][B], the layout of the gradient contractions) and dy.
struct MlpBwdSmem {
  MlpSmem f;                                              // W1, W2, b1, b2, w3, b3
  __align__(16) __nv_bfloat16 w2t[kMlpH * kW2Stride];    // W2ᵀ: row i = column i of W2
};

__device__ void load_bwd_weights(MlpBwdSmem& sm, const MlpWeights& w) {
  for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x)
    sm.w2t[(i % kMlpH) * kW2Stride + i / kMlpH] = w.w2[i];  // w2[j][i] -> w2t[i][j]
  load_weights(sm.f, w);  // ends with __syncthreads
}

__device__ __noinline__ void bwd_tile_tc(const MlpBwdSmem& sm, const __nv_bfloat16* xs, float d, float* __restrict__ act,
                                            float* __restrict__ dyb, int64_t jbase, int64_t B, int64_t valid) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t* X = reinterpret_cast<const uint32_t*>(xs);
  const uint32_t* W1 = reinterpret_cast<const uint32_t*>(sm.f.w1);
  const uint32_t* W2 = reinterpret_cast<const uint32_t*>(sm.f.w2);
  const uint32_t* W2T = reinterpret_cast<const uint32_t*>(sm.w2t);
  constexpr int XW = kXsStride / 2, W1W = kW1Stride / 2, W2W = kW2Stride / 2;
  // column jbase + s of the activation rows; samples past `valid` are not stored
  auto put = [&](int row, int smp, float v) {
    if (smp < valid) act[(size_t)row * B + jbase + smp] = v;
  };
  {  // x0 = bf16(features) and dy, one sample per lane
    const uint4* xr = reinterpret_cast<const uint4*>(xs + lane * kXsStride);
    const uint4 lo = xr[0], hi = xr[1];
    const uint32_t wv[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      put(kActX0 + 2 * k, lane, __uint_as_float(wv[k] << 16));
      put(kActX0 + 2 * k + 1, lane, __uint_as_float(wv[k] & 0xffff0000u));
    }
    if (lane < valid) dyb[jbase + lane] = d;
  }
  // dL/dy of the rows this thread's fragments hold: 16 m + g (+ 8)
  float dr[2][2];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int h = 0; h < 2; ++h) dr[m][h] = __shfl_sync(0xffffffffu, d, 16 * m + 8 * h + g);
  uint32_t a[2][4];
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int r0 = 16 * m + g;
    a[m][0] = X[r0 * XW + t];
    a[m][1] = X[(r0 + 8) * XW + t];
    a[m][2] = X[r0 * XW + t + 4];
    a[m][3] = X[(r0 + 8) * XW + t + 4];
  }
  // layer 1: h1 = bf16(relu(b1 + x W1ᵀ)) as layer-2 A fragments; mask bit (m, j, e) = z1 > 0
  uint32_t a2[2][4][4];
  uint64_t mask1 = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t b0 = W1[(8 * j + g) * W1W + t], b1 = W1[(8 * j + g) * W1W + t + 4];
    const float bb0 = sm.f.b1[8 * j + 2 * t], bb1 = sm.f.b1[8 * j + 2 * t + 1];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      float c[4] = {bb0, bb1, bb0, bb1};
      mma16816(c, a[m], b0, b1);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (c[e] > 0.f) mask1 |= 1ull << (m * 32 + j * 4 + e);
      const uint32_t lo = pack_bf16(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f));
      const uint32_t hi = pack_bf16(fmaxf(c[2], 0.f), fmaxf(c[3], 0.f));
      const int col = 8 * j + 2 * t, s0 = 16 * m + g;
      put(kActH1 + col, s0, __uint_as_float(lo << 16));
      put(kActH1 + col + 1, s0, __uint_as_float(lo & 0xffff0000u));
      put(kActH1 + col, s0 + 8, __uint_as_float(hi << 16));
      put(kActH1 + col + 1, s0 + 8, __uint_as_float(hi & 0xffff0000u));
      if ((j & 1) == 0) {
        a2[m][j >> 1][0] = lo;
        a2[m][j >> 1][1] = hi;
      } else {
        a2[m][j >> 1][2] = lo;
        a2[m][j >> 1][3] = hi;
      }
    }
  }
  // layer 2 and dz2 = d w3 [z2 > 0], packed as the A fragments (hi, lo) of dh1 = dz2 W2
  uint32_t dh[2][4][4], dl[2][4][4];
#pragma unroll
  for (int jt = 0; jt < 8; ++jt) {
    const float bb0 = sm.f.b2[8 * jt + 2 * t], bb1 = sm.f.b2[8 * jt + 2 * t + 1];
    const float w0 = sm.f.w3[8 * jt + 2 * t], w1 = sm.f.w3[8 * jt + 2 * t + 1];
    float c[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      c[m][0] = bb0;
      c[m][1] = bb1;
      c[m][2] = bb0;
      c[m][3] = bb1;
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint32_t b0 = W2[(8 * jt + g) * W2W + 8 * kk + t], b1 = W2[(8 * jt + g) * W2W + 8 * kk + t + 4];
#pragma unroll
      for (int m = 0; m < 2; ++m) mma16816(c[m], a2[m][kk], b0, b1);
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int col = 8 * jt + 2 * t, s0 = 16 * m + g;
      const float z[4] = {c[m][0], c[m][1], c[m][2], c[m][3]};
      const float dd[4] = {z[0] > 0.f ? dr[m][0] * w0 : 0.f, z[1] > 0.f ? dr[m][0] * w1 : 0.f,
                           z[2] > 0.f ? dr[m][1] * w0 : 0.f, z[3] > 0.f ? dr[m][1] * w1 : 0.f};
      put(kActR2 + col, s0, fmaxf(z[0], 0.f));
      put(kActR2 + col + 1, s0, fmaxf(z[1], 0.f));
      put(kActR2 + col, s0 + 8, fmaxf(z[2], 0.f));
      put(kActR2 + col + 1, s0 + 8, fmaxf(z[3], 0.f));
      put(kActDz2 + col, s0, dd[0]);
      put(kActDz2 + col + 1, s0, dd[1]);
      put(kActDz2 + col, s0 + 8, dd[2]);
      put(kActDz2 + col + 1, s0 + 8, dd[3]);
      uint32_t h01, l01, h23, l23;
      split_pair(dd[0], dd[1], h01, l01);
      split_pair(dd[2], dd[3], h23, l23);
      const int kk = jt >> 1, e = (jt & 1) * 2;
      dh[m][kk][e] = h01;
      dl[m][kk][e] = l01;
      dh[m][kk][e + 1] = h23;
      dl[m][kk][e + 1] = l23;
    }
  }
  // dh1 = dz2 W2 (K = the 64 units of layer 2), then dz1 = dh1 [z1 > 0]
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    float c[2][4] = {};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint32_t b0 = W2T[(8 * it + g) * W2W + 8 * kk + t], b1 = W2T[(8 * it + g) * W2W + 8 * kk + t + 4];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        mma16816(c[m], dh[m][kk], b0, b1);
        mma16816(c[m], dl[m][kk], b0, b1);
      }
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int col = 8 * it + 2 * t, s0 = 16 * m + g;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool on = (mask1 >> (m * 32 + it * 4 + e)) & 1ull;
        put(kActDz1 + col + (e & 1), s0 + 8 * (e >> 1), on ? c[m][e] : 0.f);
      }
    }
  }
}

// Backward of n given feature rows with given dL/dy (the gradient check entry point).
__global__ void __launch_bounds__(kMlpThreads) k_bwd_direct_tc(int64_t n, const float* __restrict__ x,
                                                               const float* __restrict__ dy, MlpWeights w,
                                                               float* __restrict__ act, float* __restrict__ dyb) {
  __shared__ MlpBwdSmem sm;
  __shared__ __align__(16) __nv_bfloat16 xs[kMlpWarps][kTile * kXsStride];
  load_bwd_weights(sm, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  for (int64_t tile = (int64_t)blockIdx.x * kMlpWarps + warp; tile < ntiles; tile += (int64_t)gridDim.x * kMlpWarps) {
    const int64_t q = tile * kTile + lane;
    float f[16], d = 0.f;
    if (q < n) {
      const float4* src = reinterpret_cast<const float4*>(x + q * 16);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float4 t4 = src[v];
        f[4 * v] = t4.x;
        f[4 * v + 1] = t4.y;
        f[4 * v + 2] = t4.z;
        f[4 * v + 3] = t4.w;
      }
      d = dy[q];
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    store_row(xs[warp], lane, f);
    __syncwarp();
    bwd_tile_tc(sm, xs[warp], d, act, dyb, tile * kTile, n, n - tile * kTile);
    __syncwarp();
  }
}

// Features of sample (vertex i, field rs) on a reference-ordered Laplacian / Helmholtz operator of
// n rows (slot-major ELL, columns sorted, the diagonal inside, padding column -1).
__device__ void op_features(int i, int n, int Wf, const int32_t* __restrict__ col, const double* __restrict__ val,
                            const double* __restrict__ rs, float* f, float* dsc) {
  double di = 0.0;
  for (int q = 0; q < Wf; ++q)
    if (col[(size_t)q * n + i] == i) di += val[(size_t)q * n + i];
  float nb[6], cp[6], sabs = 0.f;
  int nn = 0;
  const float dif = (float)di;
  for (int q = 0; q < Wf; ++q) {
    const int c = col[(size_t)q * n + i];
    if (c < 0 || c == i) continue;
    const float o = (float)val[(size_t)q * n + i];
    sabs += fabsf(o);
    if (nn < 6) {
      nb[nn] = (float)rs[c];
      cp[nn] = o / dif;
      ++nn;
    }
  }
  float scale;
  mlp_features((float)rs[i], nb, cp, nn, 1.f - sabs / dif, f, &scale);
  *dsc = scale / dif;
}

// The features alone, out of line: the backward tile that follows keeps its registers for the MMA
// fragments.
__device__ __noinline__ void op_features_only(int i, int n, int Wf, const int32_t* __restrict__ col,
                                              const double* __restrict__ val, const double* __restrict__ rs,
                                              float* f) {
  float dsc;
  op_features(i, n, Wf, col, val, rs, f, &dsc);
}

__global__ void k_op_features(int n, int S, int Wf, const int32_t* __restrict__ col, const double* __restrict__ val,
                              const double* __restrict__ r, float* __restrict__ feat, float* __restrict__ dscale) {
  const int64_t N = (int64_t)n * S;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(q / n), i = (int)(q % n);
    float f[16], dsc;
    op_features(i, n, Wf, col, val, r + (size_t)s * n, f, &dsc);
    for (int k = 0; k < 16; ++k) feat[q * 16 + k] = f[k];
    dscale[q] = dsc;
  }
}

// δ = dscale · MLP(features) for all n·S samples (tensor cores, the inference kernel's numerics).
__global__ void __launch_bounds__(kMlpThreads) k_train_fwd(int n, int S, int Wf, const int32_t* __restrict__ col,
                                                           const double* __restrict__ val, const double* __restrict__ r,
                                                           MlpWeights w, double* __restrict__ delta,
                                                           float* __restrict__ dscale) {
  __shared__ MlpSmem sm;
  __shared__ __align__(16) __nv_bfloat16 xs[kMlpWarps][kTile * kXsStride];
  load_weights(sm, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t N = (int64_t)n * S;
  const int64_t ntiles = (N + kTile - 1) / kTile;
  for (int64_t tile = (int64_t)blockIdx.x * kMlpWarps + warp; tile < ntiles; tile += (int64_t)gridDim.x * kMlpWarps) {
    const int64_t q = tile * kTile + lane;
    float f[16], dsc = 0.f;
    if (q < N) {
      const int s = (int)(q / n), i = (int)(q % n);
      op_features(i, n, Wf, col, val, r + (size_t)s * n, f, &dsc);
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    store_row(xs[warp], lane, f);
    __syncwarp();
    const float yv = mlp_tile32(sm, xs[warp]);
    if (q < N) {
      delta[q] = (double)(dsc * yv);
      dscale[q] = dsc;
    }
    __syncwarp();
  }
}

// n_s = Σ_i ⋆0_i r_si² / a_ii per field: kNormBlocks CTAs per field write partial sums over strided
// rows (lpart[s * kNormBlocks + b]), then one CTA per field adds them in block order.
constexpr int kNormBlocks = 64;
__global__ void __launch_bounds__(256) k_train_norm_parts(int n, int Wf, const int32_t* __restrict__ col,
                                                          const double* __restrict__ val,
                                                          const double* __restrict__ star0,
                                                          const double* __restrict__ r, double* __restrict__ part) {
  const double* rs = r + (size_t)blockIdx.y * n;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double di = 0.0;
    for (int q = 0; q < Wf; ++q)
      if (col[(size_t)q * n + i] == i) di += val[(size_t)q * n + i];
    acc += star0[i] * rs[i] * rs[i] / di;
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)blockIdx.y * kNormBlocks + blockIdx.x] = sh[0];
}

__global__ void k_train_norm_sum(const double* __restrict__ part, double* __restrict__ nrm) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < kNormBlocks; ++b) s += part[(size_t)blockIdx.x * kNormBlocks + b];
  nrm[blockIdx.x] = s > 0 ? s : 1.0;
}

static void train_norms(dec_mlp& m, const dec_op* op, const double* r, int S, cudaStream_t s) {
  if (m.npart.n < (size_t)S * kNormBlocks) m.npart.alloc((size_t)S * kNormBlocks);
  const int n = op->m->nv;
  k_train_norm_parts<<<dim3(kNormBlocks, S), 256, 0, s>>>(n, op->W, op->col.p, op->val64.p, op->m->star0.p, r,
                                                          m.npart.p);
  k_train_norm_sum<<<S, 32, 0, s>>>(m.npart.p, m.nrm.p);
  DEC_CHECK_LAUNCH();
}

// dL/dδ = 2 w (A δ - r), w = ⋆0_i / (S n_s); dy = dL/dδ · dscale; loss partials Σ w δ (A δ - 2 r).
constexpr int kLossBlocks = 512;
__global__ void __launch_bounds__(256) k_train_loss(int n, int S, const double* __restrict__ r,
                                                    const double* __restrict__ aq, const double* __restrict__ delta,
                                                    const double* __restrict__ star0, const double* __restrict__ nrm,
                                                    const float* __restrict__ dscale, double* __restrict__ dy,
                                                    double* __restrict__ lpart) {
  const int64_t N = (int64_t)n * S;
  double acc = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(k / n), i = (int)(k % n);
    const double w = star0[i] / (nrm[s] * S);
    dy[k] = 2.0 * w * (aq[k] - r[k]) * (double)dscale[k];
    acc += w * delta[k] * (aq[k] - 2.0 * r[k]);
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) lpart[blockIdx.x] = sh[0];
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Backward over the batch: column j is sample j when the fields hold at most B samples, else a
// sample drawn uniformly with replacement from (seed, step, j); dL/dy is scaled by N / B so the
// batch gradient estimates the full one.
__global__ void __launch_bounds__(kMlpThreads) k_train_bwd_tc(int n, int S, int64_t B, uint64_t seed, int64_t step,
                                                              int Wf, const int32_t* __restrict__ col,
                                                              const double* __restrict__ val,
                                                              const double* __restrict__ r, MlpWeights w,
                                                              const double* __restrict__ dy, float* __restrict__ act,
                                                              float* __restrict__ dyb) {
  __shared__ MlpBwdSmem sm;
  __shared__ __align__(16) __nv_bfloat16 xs[kMlpWarps][kTile * kXsStride];
  load_bwd_weights(sm, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t N = (int64_t)n * S;
  const bool sample = N > B;
  const int64_t Bn = sample ? B : N;
  const double scale = sample ? (double)N / (double)B : 1.0;
  const int64_t ntiles = (Bn + kTile - 1) / kTile;
  for (int64_t tile = (int64_t)blockIdx.x * kMlpWarps + warp; tile < ntiles; tile += (int64_t)gridDim.x * kMlpWarps) {
    const int64_t j = tile * kTile + lane;
    float f[16], d = 0.f;
    if (j < Bn) {
      int64_t q = j;
      if (sample) {
        const uint64_t h = mix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(step + 1) + 0xD1B54A32D192ED03ull * (uint64_t)j);
        q = (int64_t)(h % (uint64_t)N);
      }
      const int s = (int)(q / n), i = (int)(q % n);
      op_features_only(i, n, Wf, col, val, r + (size_t)s * n, f);
      d = (float)(dy[q] * scale);
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    store_row(xs[warp], lane, f);
    __syncwarp();
    bwd_tile_tc(sm, xs[warp], d, act, dyb, tile * kTile, Bn, Bn - tile * kTile);
    __syncwarp();
  }
}

static unsigned bwd_grid(int64_t samples) {
  const long long tiles = (samples + kTile - 1) / kTile;
  return (unsigned)std::max<long long>(1, std::min<long long>((tiles + kMlpWarps - 1) / kMlpWarps, num_sms() * 4LL));
}

// Parameter gradient partials over one chunk of batch columns per CTA, in a fixed order:
// dW1 = Σ dz1 x0ᵀ, db1 = Σ dz1, dW2 = Σ dz2 h1ᵀ, db2 = Σ dz2, dw3 = Σ dy relu(z2), db3 = Σ dy.
constexpr int kGradThreads = 256, kGradChunk = 256, kMaxChunks = 1024;

// The two contractions run on the tensor cores (mma.sync m16n8k16, BF16 operands,
// FP32 accumulation): dW2 = Σ_s dz2_s h1_sᵀ and dW1 = Σ_s dz1_s x0_sᵀ over the batch, K = the batch
// samples.  x0 and h1 are BF16 values already; dz1 and dz2 enter as hi + lo BF16 pairs (hi = the
// round-to-nearest BF16, lo = that of the remainder), so each product carries 16 of FP32's 24 bits
// of dz.  A CTA stages 32 samples of every activation row in shared memory at a time; warp w owns
// the output tiles dW2 rows 16 (w / 2) .. +15, columns 32 (w % 2) .. +31 (four n8 tiles) and dW1
// rows 16 (w / 2) .., columns 8 (w % 2) .. +7.  db1, db2, dw3 and db3 are sums on the CUDA cores.
constexpr int kGradStage = 32;

__global__ void __launch_bounds__(kGradThreads) k_train_grad_tc(int64_t B, int64_t chunk,
                                                                const float* __restrict__ act,
                                                                const float* __restrict__ dyb,
                                                                float* __restrict__ gpart) {
  // rows of the staged batch slice: the activation rows then dy, kGradStage samples each (+1 pad)
  constexpr int kRows = kActRows + 1, kLd = kGradStage + 1;
  __shared__ float sa[kRows * kLd];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int mt = warp >> 1, nh = warp & 1;
  float c2[4][4] = {}, c1[4] = {};
  float sacc = 0.f;  // this thread's bias / w3 sum (threads 0 .. 192)
  const int64_t lo = blockIdx.x * chunk, hi = min(B, lo + chunk);
  for (int64_t b0 = lo; b0 < hi; b0 += kGradStage) {
    // the slice arrives by asynchronous copies, all in flight before the one wait (a load and a
    // store per element serialised the staging on the load latency)
    for (int e = threadIdx.x; e < kRows * kGradStage; e += kGradThreads) {
      const int row = e / kGradStage, c = e % kGradStage;
      const int64_t q = b0 + c;
      float* dst = sa + row * kLd + c;
      if (q < hi) {
        const float* src = row < kActRows ? act + (size_t)row * B + q : dyb + q;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                     "l"(src)
                     : "memory");
      } else {
        *dst = 0.f;
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kGradStage; ks += 16) {
      // A fragments of dz2 rows 16 mt .. (and dz1 for dW1), hi and lo parts
      auto afrag = [&](int base, uint32_t (&ah)[4], uint32_t (&al)[4]) {
        const float* r0 = sa + (base + 16 * mt + g) * kLd + ks;
        const float* r8 = r0 + 8 * kLd;
        split_pair(r0[2 * t], r0[2 * t + 1], ah[0], al[0]);
        split_pair(r8[2 * t], r8[2 * t + 1], ah[1], al[1]);
        split_pair(r0[2 * t + 8], r0[2 * t + 9], ah[2], al[2]);
        split_pair(r8[2 * t + 8], r8[2 * t + 9], ah[3], al[3]);
      };
      uint32_t ah[4], al[4];
      afrag(kActDz2, ah, al);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float* h = sa + (kActH1 + 32 * nh + 8 * u + g) * kLd + ks;
        const uint32_t b0r = pack_bf16(h[2 * t], h[2 * t + 1]), b1r = pack_bf16(h[2 * t + 8], h[2 * t + 9]);
        mma16816(c2[u], ah, b0r, b1r);
        mma16816(c2[u], al, b0r, b1r);
      }
      afrag(kActDz1, ah, al);
      {
        const float* x = sa + (kActX0 + 8 * nh + g) * kLd + ks;
        const uint32_t b0r = pack_bf16(x[2 * t], x[2 * t + 1]), b1r = pack_bf16(x[2 * t + 8], x[2 * t + 9]);
        mma16816(c1, ah, b0r, b1r);
        mma16816(c1, al, b0r, b1r);
      }
    }
    // db1 (threads 0..63), db2 (64..127), dw3 = Σ dy relu(z2) (128..191), db3 = Σ dy (192)
    if (threadIdx.x < 3 * kMlpH + 1) {
      const int p = threadIdx.x;
      const float* row = p < kMlpH         ? sa + (kActDz1 + p) * kLd
                         : p < 2 * kMlpH   ? sa + (kActDz2 + p - kMlpH) * kLd
                         : p < 3 * kMlpH   ? sa + (kActR2 + p - 2 * kMlpH) * kLd
                                           : sa + kActRows * kLd;
      const float* dy = sa + kActRows * kLd;
      float s = 0.f;
      if (p >= 2 * kMlpH && p < 3 * kMlpH) {
        for (int c = 0; c < kGradStage; ++c) s += dy[c] * row[c];
      } else {
        for (int c = 0; c < kGradStage; ++c) s += row[c];
      }
      sacc += s;
    }
    __syncthreads();
  }
  float* out = gpart + (size_t)blockIdx.x * kMlpNParam;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int j = 16 * mt + g, i = 32 * nh + 8 * u + 2 * t;
    out[kOffW2 + j * kMlpH + i] = c2[u][0];
    out[kOffW2 + j * kMlpH + i + 1] = c2[u][1];
    out[kOffW2 + (j + 8) * kMlpH + i] = c2[u][2];
    out[kOffW2 + (j + 8) * kMlpH + i + 1] = c2[u][3];
  }
  {
    const int j = 16 * mt + g, k = 8 * nh + 2 * t;
    out[kOffW1 + j * kMlpIn + k] = c1[0];
    out[kOffW1 + j * kMlpIn + k + 1] = c1[1];
    out[kOffW1 + (j + 8) * kMlpIn + k] = c1[2];
    out[kOffW1 + (j + 8) * kMlpIn + k + 1] = c1[3];
  }
  if (threadIdx.x < kMlpH) out[kOffB1 + threadIdx.x] = sacc;
  else if (threadIdx.x < 2 * kMlpH) out[kOffB2 + threadIdx.x - kMlpH] = sacc;
  else if (threadIdx.x < 3 * kMlpH) out[kOffW3 + threadIdx.x - 2 * kMlpH] = sacc;
  else if (threadIdx.x == 3 * kMlpH) out[kOffB3] = sacc;
}

// The chunk partials summed in a fixed order, in two levels: group g of kReduceGroups adds chunks
// g, g + G, g + 2G, ... (in increasing order) into red[g]; then the groups are added in order.
constexpr int kReduceGroups = 16;
__global__ void k_grad_reduce(int nchunks, const float* __restrict__ gpart, float* __restrict__ red) {
  const int g = blockIdx.y;
  for (int pi = blockIdx.x * blockDim.x + threadIdx.x; pi < kMlpNParam; pi += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = g; c < nchunks; c += kReduceGroups) s += gpart[(size_t)c * kMlpNParam + pi];
    red[(size_t)g * kMlpNParam + pi] = s;
  }
}

__global__ void k_grad_reduce2(const float* __restrict__ red, float* __restrict__ grad) {
  for (int pi = blockIdx.x * blockDim.x + threadIdx.x; pi < kMlpNParam; pi += gridDim.x * blockDim.x) {
    float s = 0.f;
#pragma unroll
    for (int g = 0; g < kReduceGroups; ++g) s += red[(size_t)g * kMlpNParam + pi];
    grad[pi] = s;
  }
}

__global__ void k_refresh_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ w1b,
                               __nv_bfloat16* __restrict__ w2b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpH * kMlpH; i += gridDim.x * blockDim.x) {
    if (i < kMlpH * kMlpIn) w1b[i] = __float2bfloat16_rn(p[kOffW1 + i]);
    w2b[i] = __float2bfloat16_rn(p[kOffW2 + i]);
  }
}

// Adam (β1 = 0.9, β2 = 0.999, ε = 1e-8, bias-corrected) on the FP32 masters.
__global__ void k_adam(int64_t t, float lr, const float* __restrict__ g, float* __restrict__ p, float* __restrict__ m,
                       float* __restrict__ v) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpNParam; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static unsigned eval_grid(long long samples) {
  const long long tiles = (samples + kTile - 1) / kTile;
  return (unsigned)std::max<long long>(1, std::min<long long>((tiles + kMlpWarps - 1) / kMlpWarps, num_sms() * 4LL));
}

static void ensure_scratch(dec_mlp& m, size_t N, size_t B, int S) {
  if (m.cap_n < N) {
    m.delta.alloc(N);
    m.q.alloc(N);
    m.dy.alloc(N);
    m.dsc.alloc(N);
    m.cap_n = N;
  }
  if (m.cap_b < B) {
    m.act.alloc((size_t)kActRows * B);
    m.dyb.alloc(B);
    m.cap_b = B;
  }
  if (m.nrm.n < (size_t)S) m.nrm.alloc(std::max<size_t>(S, 64));
  if (m.lpart.n < (size_t)kLossBlocks) m.lpart.alloc(kLossBlocks);
  if (m.gpart.n < (size_t)(kMaxChunks + kReduceGroups) * kMlpNParam)
    m.gpart.alloc((size_t)(kMaxChunks + kReduceGroups) * kMlpNParam);
}

static int grad_chunks(int64_t B, int64_t* chunk) {
  int nch = (int)std::min<int64_t>(kMaxChunks, std::max<int64_t>(1, (B + kGradChunk - 1) / kGradChunk));
  *chunk = (B + nch - 1) / nch;
  return nch;
}

static void reduce_grad(dec_mlp& m, int64_t B, float* grad, cudaStream_t s) {
  int64_t chunk;
  const int nch = grad_chunks(B, &chunk);
  k_train_grad_tc<<<nch, kGradThreads, 0, s>>>(B, chunk, m.act.p, m.dyb.p, m.gpart.p);
  float* red = m.gpart.p + (size_t)kMaxChunks * kMlpNParam;  // after the chunk partials
  k_grad_reduce<<<dim3((kMlpNParam + 255) / 256, kReduceGroups), 256, 0, s>>>(nch, m.gpart.p, red);
  k_grad_reduce2<<<(kMlpNParam + 255) / 256, 256, 0, s>>>(red, grad);
  DEC_CHECK_LAUNCH();
}

static void check_train_op(const dec_op* op) {
  require(op != nullptr, "mlp: null operator");
  require(op->kind == DEC_OP_LAPLACE0 || op->kind == DEC_OP_HELMHOLTZ0,
          "mlp: training needs a Laplacian / Helmholtz operator");
  require(op->dtype == DEC_F64, "mlp: training needs an FP64 operator");
}

// δ, A δ, dL/dy and the loss partials of S fields on the operator's mesh.
static void loss_and_dy(dec_mlp& m, dec_op* op, const double* r, int S, cudaStream_t s) {
  const int n = op->m->nv;
  const int64_t N = (int64_t)n * S;
  k_train_fwd<<<eval_grid(N), kMlpThreads, 0, s>>>(n, S, op->W, op->col.p, op->val64.p, r, m.view(), m.delta.p,
                                                   m.dsc.p);
  DEC_CHECK_LAUNCH();
  for (int j = 0; j < S; ++j) op_apply_impl(op, m.delta.p + (size_t)j * n, m.q.p + (size_t)j * n, 1.0, 0.0, s);
  k_train_loss<<<kLossBlocks, 256, 0, s>>>(n, S, r, m.q.p, m.delta.p, op->m->star0.p, m.nrm.p, m.dsc.p, m.dy.p,
                                           m.lpart.p);
  DEC_CHECK_LAUNCH();
}

static double host_loss(dec_mlp& m, cudaStream_t s) {
  std::vector<double> lp(kLossBlocks);
  DEC_CUDA(cudaMemcpyAsync(lp.data(), m.lpart.p, kLossBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaStreamSynchronize(s));
  double tot = 0;
  for (double v : lp) tot += v;
  return tot;
}

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320), bitwise.
static uint32_t crc32(const unsigned char* p, size_t n) {
  uint32_t c = 0xFFFFFFFFu;
  for (size_t i = 0; i < n; ++i) {
    c ^= p[i];
    for (int k = 0; k < 8; ++k) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
  }
  return ~c;
}

}  // namespace decb

using namespace decb;

// After every change of the parameters: the host copy of the per-unit vectors, and a new
// version (cycles captured with the old copy are captured again).
static void refresh_small(dec_mlp* m) {
  DEC_CUDA(cudaDeviceSynchronize());
  DEC_CUDA(cudaMemcpy(m->hsmall.b1, m->master.p + kOffB1, kMlpH * 4, cudaMemcpyDeviceToHost));
  DEC_CUDA(cudaMemcpy(m->hsmall.b2, m->master.p + kOffB2, kMlpH * 4, cudaMemcpyDeviceToHost));
  DEC_CUDA(cudaMemcpy(m->hsmall.w3, m->master.p + kOffW3, kMlpH * 4, cudaMemcpyDeviceToHost));
  DEC_CUDA(cudaMemcpy(&m->hsmall.b3, m->master.p + kOffB3, 4, cudaMemcpyDeviceToHost));
  ++m->version;
}

dec_mlp* mlp_create_impl(uint64_t seed) {
  auto* m = new dec_mlp();
  try {
    // Xavier (Glorot) uniform U(-a, a), a = sqrt(6 / (fan_in + fan_out)), from the splitmix64
    // stream of the seed; biases zero.
    std::vector<float> p(kMlpNParam, 0.f);
    uint64_t st = seed;
    auto fill = [&](int off, int cnt, int fin, int fout) {
      const double a = std::sqrt(6.0 / (fin + fout));
      for (int i = 0; i < cnt; ++i) {
        const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
        p[off + i] = (float)((2.0 * u - 1.0) * a);
      }
    };
    fill(kOffW1, kMlpH * kMlpIn, kMlpIn, kMlpH);
    fill(kOffW2, kMlpH * kMlpH, kMlpH, kMlpH);
    fill(kOffW3, kMlpH, kMlpH, 1);
    m->master.upload(p);
    m->adam_m.alloc(kMlpNParam);
    m->adam_v.alloc(kMlpNParam);
    DEC_CUDA(cudaMemset(m->adam_m.p, 0, m->adam_m.bytes()));
    DEC_CUDA(cudaMemset(m->adam_v.p, 0, m->adam_v.bytes()));
    m->grad.alloc(kMlpNParam);
    m->w1b.alloc(kMlpH * kMlpIn);
    m->w2b.alloc(kMlpH * kMlpH);
    m->err.alloc(1);
    DEC_CUDA(cudaMemset(m->err.p, 0, sizeof(int)));
    k_refresh_bf16<<<16, 256>>>(m->master.p, m->w1b.p, m->w2b.p);
    DEC_CHECK_LAUNCH();
    refresh_small(m);
    tc_opt_in_all();  // the default engine's kernels, outside any stream capture
  } catch (...) {
    delete m;
    throw;
  }
  return m;
}

void mlp_destroy_impl(dec_mlp* m) { delete m; }

void mlp_params_impl(dec_mlp* m, float* out, const float* in) {
  require(m != nullptr, "mlp: null handle");
  if (out) DEC_CUDA(cudaMemcpy(out, m->master.p, m->master.bytes(), cudaMemcpyDeviceToHost));
  if (in) {
    DEC_CUDA(cudaMemcpy(m->master.p, in, m->master.bytes(), cudaMemcpyHostToDevice));
    k_refresh_bf16<<<16, 256>>>(m->master.p, m->w1b.p, m->w2b.p);
    DEC_CHECK_LAUNCH();
    refresh_small(m);
  }
}

int64_t mlp_step_impl(const dec_mlp* m) {
  require(m != nullptr, "mlp: null handle");
  return m->step;
}

MlpWeights mlp_weights(const dec_mlp* m) {
  require(m != nullptr, "mlp: null handle");
  return m->view();
}

// Reads and clears the tcgen05 kernels' error flag (synchronises the stream).
void mlp_check_error(const dec_mlp* m, cudaStream_t s) {
  int h = 0;
  DEC_CUDA(cudaMemcpyAsync(&h, m->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaStreamSynchronize(s));
  if (h) {
    DEC_CUDA(cudaMemsetAsync(m->err.p, 0, sizeof(int), s));
    throw Error(DEC_ERR_TIMEOUT, "mlp: a tcgen05 kernel timed out waiting for its MMA");
  }
}

void mlp_set_engine_impl(dec_mlp* m, int engine) {
  require(m != nullptr, "mlp: null handle");
  require(engine == 0 || engine == 1, "mlp: engine must be 0 (mma.sync) or 1 (tcgen05)");
  if (engine == 1) tc_opt_in_all();  // outside any stream capture
  m->engine = engine;
}

void mlp_eval_impl(dec_mlp* m, const float* x, int64_t n, float* y, int tensor_cores, void* stream) {
  require(m != nullptr && n >= 0 && (n == 0 || (x != nullptr && y != nullptr)), "mlp: bad eval arguments");
  require((reinterpret_cast<uintptr_t>(x) & 15) == 0, "mlp: features must be 16-byte aligned");
  if (n == 0) return;
  cudaStream_t s = as_stream(stream);
  if (tensor_cores == 2) {
    tc_opt_in(k_mlp_eval_tcg);
    k_mlp_eval_tcg<<<tc_grid((n + kTcRows - 1) / kTcRows), kTcThreads, kTcSmemBytes, s>>>(n, x, y, m->view(),
                                                                                        m->err.p);
    DEC_CHECK_LAUNCH();
    mlp_check_error(m, s);
    return;
  }
  if (tensor_cores) k_mlp_eval_tc<<<eval_grid(n), kMlpThreads, 0, s>>>(n, x, y, m->view());
  else k_mlp_eval_cc<<<grid_for(n, 128), 128, 0, s>>>(n, x, y, m->w1b.p, m->w2b.p, m->master.p);
  DEC_CHECK_LAUNCH();
}

void mlp_grad_impl(dec_mlp* m, const float* x, const float* dy, int64_t n, float* grad, void* stream) {
  require(m != nullptr && x != nullptr && dy != nullptr && grad != nullptr && n > 0, "mlp: bad grad arguments");
  cudaStream_t s = as_stream(stream);
  ensure_scratch(*m, 1, (size_t)n, 1);
  k_bwd_direct_tc<<<bwd_grid(n), kMlpThreads, 0, s>>>(n, x, dy, mlp_weights(m), m->act.p, m->dyb.p);
  DEC_CHECK_LAUNCH();
  reduce_grad(*m, n, grad, s);
}

void mlp_features_impl(const dec_op* op, const double* r, int S, float* feat, float* dscale, void* stream) {
  check_train_op(op);
  require(r != nullptr && feat != nullptr && dscale != nullptr && S >= 1, "mlp: bad feature arguments");
  const int n = op->m->nv;
  k_op_features<<<grid_for((long long)n * S, 128), 128, 0, as_stream(stream)>>>(n, S, op->W, op->col.p, op->val64.p, r,
                                                                                 feat, dscale);
  DEC_CHECK_LAUNCH();
}

void mlp_loss_grad_impl(dec_mlp* m, dec_op* op, const double* r, int S, double* loss, float* grad, void* stream) {
  require(m != nullptr && r != nullptr && S >= 1, "mlp: bad loss arguments");
  check_train_op(op);
  cudaStream_t s = as_stream(stream);
  const int n = op->m->nv;
  const int64_t N = (int64_t)n * S;
  ensure_scratch(*m, (size_t)N, (size_t)N, S);
  train_norms(*m, op, r, S, s);
  loss_and_dy(*m, op, r, S, s);
  if (grad) {
    k_train_bwd_tc<<<bwd_grid(N), kMlpThreads, 0, s>>>(n, S, N, 0, 0, op->W, op->col.p, op->val64.p, r,
                                                         mlp_weights(m), m->dy.p, m->act.p, m->dyb.p);
    DEC_CHECK_LAUNCH();
    reduce_grad(*m, N, grad, s);
  }
  if (loss) *loss = host_loss(*m, s);
}

void mlp_train_impl(dec_mlp* m, dec_op* op, const double* r, int S, int steps, double lr, int64_t batch,
                    uint64_t seed, double* losses, void* stream) {
  require(m != nullptr && r != nullptr && S >= 1 && steps >= 0 && batch >= 1 && lr > 0, "mlp: bad train arguments");
  check_train_op(op);
  cudaStream_t s = as_stream(stream);
  const int n = op->m->nv;
  const int64_t N = (int64_t)n * S;
  const int64_t Bn = std::min<int64_t>(batch, N);
  ensure_scratch(*m, (size_t)N, (size_t)Bn, S);
  train_norms(*m, op, r, S, s);
  for (int it = 0; it < steps; ++it) {
    loss_and_dy(*m, op, r, S, s);
    k_train_bwd_tc<<<bwd_grid(Bn), kMlpThreads, 0, s>>>(n, S, batch, seed, m->step, op->W, op->col.p, op->val64.p,
                                                          r, mlp_weights(m), m->dy.p, m->act.p, m->dyb.p);
    DEC_CHECK_LAUNCH();
    reduce_grad(*m, Bn, m->grad.p, s);
    ++m->step;
    k_adam<<<(kMlpNParam + 255) / 256, 256, 0, s>>>(m->step, (float)lr, m->grad.p, m->master.p, m->adam_m.p,
                                                    m->adam_v.p);
    k_refresh_bf16<<<16, 256, 0, s>>>(m->master.p, m->w1b.p, m->w2b.p);
    DEC_CHECK_LAUNCH();
    if (losses) losses[it] = host_loss(*m, s);  // the loss before this step's update
  }
  if (steps > 0) refresh_small(m);
}

// Checkpoint: "DECMLP01" | u32 version | u32 nparam | i64 step | f32 master, adam_m, adam_v
// (nparam each) | u32 CRC-32 of everything before it.
static constexpr char kMagic[8] = {'D', 'E', 'C', 'M', 'L', 'P', '0', '1'};

void mlp_save_impl(const dec_mlp* m, const char* path) {
  require(m != nullptr && path != nullptr, "mlp: bad save arguments");
  DEC_CUDA(cudaDeviceSynchronize());
  std::vector<unsigned char> buf;
  auto put = [&](const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    buf.insert(buf.end(), c, c + n);
  };
  const uint32_t version = 1, np = kMlpNParam;
  put(kMagic, 8);
  put(&version, 4);
  put(&np, 4);
  put(&m->step, 8);
  for (const DArr<float>* a : {&m->master, &m->adam_m, &m->adam_v}) {
    std::vector<float> h = a->download();
    put(h.data(), h.size() * 4);
  }
  const uint32_t crc = crc32(buf.data(), buf.size());
  put(&crc, 4);
  FILE* f = std::fopen(path, "wb");
  require(f != nullptr, std::string("mlp: cannot open ") + path + " for writing");
  const size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
  const int rc = std::fclose(f);
  require(w == buf.size() && rc == 0, std::string("mlp: short write to ") + path);
}

void mlp_load_impl(dec_mlp* m, const char* path) {
  require(m != nullptr && path != nullptr, "mlp: bad load arguments");
  FILE* f = std::fopen(path, "rb");
  require(f != nullptr, std::string("mlp: cannot open ") + path);
  std::vector<unsigned char> buf;
  unsigned char tmp[65536];
  size_t k;
  while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
  std::fclose(f);
  const size_t body = 8 + 4 + 4 + 8 + 3 * (size_t)kMlpNParam * 4;
  require(buf.size() == body + 4, "mlp: checkpoint has the wrong size");
  require(std::memcmp(buf.data(), kMagic, 8) == 0, "mlp: not a checkpoint");
  uint32_t version, np, crc;
  int64_t step;
  std::memcpy(&version, buf.data() + 8, 4);
  std::memcpy(&np, buf.data() + 12, 4);
  std::memcpy(&step, buf.data() + 16, 8);
  std::memcpy(&crc, buf.data() + body, 4);
  require(version == 1 && np == (uint32_t)kMlpNParam, "mlp: unsupported checkpoint version / shape");
  require(crc32(buf.data(), body) == crc, "mlp: checkpoint CRC mismatch");
  const unsigned char* p = buf.data() + 24;
  for (DArr<float>* a : {&m->master, &m->adam_m, &m->adam_v}) {
    DEC_CUDA(cudaMemcpy(a->p, p, (size_t)kMlpNParam * 4, cudaMemcpyHostToDevice));
    p += (size_t)kMlpNParam * 4;
  }
  m->step = step;
  k_refresh_bf16<<<16, 256>>>(m->master.p, m->w1b.p, m->w2b.p);
  DEC_CHECK_LAUNCH();
  refresh_small(m);
}
