// The learned smoother's per-vertex MLP (16 -> 64 -> 64 -> 1, ReLU): parameters, inference on
// the tensor cores and the training state.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace decb {

constexpr int kMlpIn = 16, kMlpH = 64;
constexpr int kMlpNParam = kMlpH * kMlpIn + kMlpH + kMlpH * kMlpH + kMlpH + kMlpH + 1;  // 5313
// flat layout: W1[64][16] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpH * kMlpIn, kOffW2 = kOffB1 + kMlpH, kOffB2 = kOffW2 + kMlpH * kMlpH,
              kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kMlpH;

// Device view of the inference weights: W1, W2 in BF16, the rest FP32.
// The network's per-unit vectors, passed by value (kernel parameter space) to the tcgen05
// kernels, whose epilogues then read them as constant operands instead of shared memory.
struct MlpSmall {
  float b1[kMlpH], b2[kMlpH], w3[kMlpH], b3;
};

struct MlpWeights {
  const __nv_bfloat16* w1;  // [64][16]
  const __nv_bfloat16* w2;  // [64][64]
  const float* b1;          // 64
  const float* b2;          // 64
  const float* w3;          // 64
  const float* b3;          // 1
  int engine;               // 0: mma.sync kernels, 1: tcgen05 / TMEM kernels
  int* err;                 // set by a kernel whose bounded wait timed out
  MlpSmall hs;              // b1, b2, w3, b3 as of the last parameter change (host copy)
};

// Features of one vertex sample from its residual and its 1-ring (used by inference and
// training alike).  nbr_r / cpl hold up to 6 neighbour residuals and couplings a_ij / a_ii in
// the operator row's column order; margin = 1 - Σ_j |a_ij| / a_ii.
//   f0 = r_i / s, f1..f6 = r_j / s, f7..f12 = a_ij / a_ii, f13 = margin, f14 = valence / 6,
//   f15 = 0, with s = max(|r_i|, |r_j|) (1 when all are zero).
__device__ __forceinline__ void mlp_features(float ri, const float* nbr_r, const float* cpl, int nn, float margin,
                                             float* f, float* scale) {
  float s = fabsf(ri);
  for (int q = 0; q < nn; ++q) s = fmaxf(s, fabsf(nbr_r[q]));
  if (s == 0.0f) s = 1.0f;
  const float inv = 1.0f / s;
  f[0] = ri * inv;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    f[1 + q] = q < nn ? nbr_r[q] * inv : 0.0f;
    f[7 + q] = q < nn ? cpl[q] : 0.0f;
  }
  f[13] = margin;
  f[14] = (float)nn * (1.0f / 6.0f);
  f[15] = 0.0f;
  *scale = s;
}

}  // namespace decb

struct dec_mlp {
  decb::DArr<float> master;   // FP32 master parameters (kMlpNParam)
  decb::DArr<float> adam_m, adam_v;
  decb::DArr<__nv_bfloat16> w1b, w2b;  // BF16 copies used by inference
  decb::DArr<float> grad;
  int64_t step = 0;
  // training scratch (sized on demand)
  size_t cap_n = 0, cap_b = 0;
  decb::DArr<float> act;      // per-sample activations of the backward batch, SoA
  decb::DArr<double> delta, q, dy;  // per sample: δ, A δ, dL/dy
  decb::DArr<float> dsc;            // per sample: s_i / a_ii
  decb::DArr<float> dyb;      // dL/dy of the backward batch
  decb::DArr<float> gpart;    // per-chunk gradient partials
  decb::DArr<double> lpart, nrm, npart;
  decb::DArr<int> err;        // device error flag of the tcgen05 kernels
  int engine = 1;             // tcgen05 (1) by default; mma.sync (0) on request
  decb::MlpSmall hsmall{};    // host copy of b1, b2, w3, b3 (refreshed with every parameter change)
  uint64_t version = 0;       // bumped with every parameter change (captured cycles hold hsmall)
  decb::MlpWeights view() const {
    return {w1b.p, w2b.p, master.p + decb::kOffB1, master.p + decb::kOffB2, master.p + decb::kOffW3,
            master.p + decb::kOffB3, engine, err.p, hsmall};
  }
};

namespace decb {
// Launches the learned smoothing step on a multigrid level (panel layout [panel][row][K]):
// out = x + (s_i / a_ii) MLP(features(r)) with x taken as zero when zero_x.
// T = float / double level arrays.  Defined in mlp.cu.
// tab: the level's per-row feature table (build_mlp_table).
template <class T, int K>
void launch_mlp_smooth(const MlpWeights& w, int n, int W, const int32_t* col, const float4* tab, const T* diag,
                       const T* r, const T* x, int zero_x, T* out, int np, cudaStream_t s);
// Per-row coupling features of a level's split operator (2 float4 per row).
void build_mlp_table(int n, int W, const int32_t* col, const double* off, const double* diag, DArr<float4>& tab);
}  // namespace decb
