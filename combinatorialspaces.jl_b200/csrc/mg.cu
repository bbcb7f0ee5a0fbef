// Geometric multigrid over binary-subdivision hierarchies (src/Multigrid.jl) on the GPU.
//
// Hierarchy (MultigridData(s, BinarySubdivision(), levels, op, steps), Multigrid.jl:698-797):
// refine / propagate_points / subdivision_matrix / make_restriction are restated here on the
// host (integer work, exact); every level's dual geometry and operator A = L + shift I is
// built on the GPU by the mesh / ops code.  The orientation that dualize's orient! would give
// a refined level is written down directly: binary refinement puts children 4t..4t+3 of
// triangle t at orientation (o_t, ¬o_t, o_t, ¬o_t) relative to the parent, and the first child
// of a component's first triangle is the DFS seed, so one flip per component at the first
// refinement reproduces orient!'s result exactly.
//
// Solve layout.  Each level is stored internally in a locality order (vertices sorted along a
// 3D Morton curve), so a row's neighbours sit close in memory and the gathers of the SpMV hit
// L2; rows keep the reference's column order, so sums are unchanged, and only the finest
// level's entry / exit kernels apply the permutation.  Right-hand sides are processed in
// panels of K (1..32) stored [panel][row][K]: a row's K values are contiguous, each lane moves
// V of them with one vector load (V = 4 FP32 / 2 FP64 values), and the K/V lanes of a row read
// the same matrix entries (one broadcast transaction).  A panel grid dimension processes all
// panels in one launch.  Smoothers: damped Jacobi or Chebyshev-Jacobi (bounds from a GPU power
// iteration); coarsest level: dense FP64 solve with the precomputed inverse.  Mixed precision
// runs the V-cycles in FP32 on the FP64 residual inside FP64 iterative refinement; the residual
// step and the V-cycle step are each one CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <numeric>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_fp16.h>

#include "mg.cuh"
#include "mlp.cuh"
#include "tune.cuh"

dec_op* op_create_impl(dec_mesh* mh, int kind, double shift, dec_dtype dt);
dec_op* op_from_csr_impl(dec_mesh* mh, int n, const std::vector<int32_t>& rowptr, const std::vector<int32_t>& colind,
                         const std::vector<double>& val);
void csc_to_csr(const dec_csc& a, std::vector<int32_t>& rp, std::vector<int32_t>& ci, std::vector<double>& vv);
decb::MlpWeights mlp_weights(const dec_mlp* m);
void mlp_check_error(const dec_mlp* m, cudaStream_t s);

namespace decb {

// ---------------------------------------------------------------------------------------------
// Host topology: the coarse mesh's orientation flips and GalerkinMode's sparse products
// (the refinement itself runs on the device, Mesh::refine_from)
// ---------------------------------------------------------------------------------------------
struct HostLevel {
  int nv = 0, ne = 0, nt = 0;
  std::vector<int32_t> ev0, ev1, te0, te1, te2;
  std::vector<int8_t> eo, to;
  std::vector<double> pts;
};

// Per coarse triangle: does its component's DFS seed (first triangle) carry `false`?  Then the
// fine level's orient! (seeded true at that triangle's first child) flips the component.
static std::vector<int8_t> component_flips(const HostLevel& c) {
  const int nt = c.nt, ne = c.ne;
  std::vector<int32_t> comp(nt, -1);
  std::vector<std::vector<int32_t>> etri(ne);
  for (int t = 0; t < nt; ++t) {
    etri[c.te0[t]].push_back(t);
    etri[c.te1[t]].push_back(t);
    etri[c.te2[t]].push_back(t);
  }
  std::vector<int8_t> flip(nt, 0);
  std::vector<int32_t> stack;
  for (int seed = 0; seed < nt; ++seed) {
    if (comp[seed] >= 0) continue;
    int8_t f = c.to[seed] ? 0 : 1;
    comp[seed] = seed;
    stack.assign(1, seed);
    while (!stack.empty()) {
      int x = stack.back();
      stack.pop_back();
      flip[x] = f;
      int es[3] = {c.te0[x], c.te1[x], c.te2[x]};
      for (int e : es)
        for (int y : etri[e])
          if (comp[y] < 0) {
            comp[y] = seed;
            stack.push_back(y);
          }
    }
  }
  return flip;
}

// The host topology of a mesh (downloaded once if the mesh was refined on the device).
static HostLevel host_level(const Mesh& m) {
  m.ensure_host();
  HostLevel h;
  h.nv = m.nv;
  h.ne = m.ne;
  h.nt = m.nt;
  h.ev0 = m.h_ev0;
  h.ev1 = m.h_ev1;
  h.te0 = m.h_te0;
  h.te1 = m.h_te1;
  h.te2 = m.h_te2;
  h.eo = m.h_eo;
  h.to = m.h_to;
  h.pts = m.h_pts;
  return h;
}

// Locality order: vertices sorted by the 3D Morton code of their (bounding-box normalised)
// position, 21 bits per axis (a stable sort, ties in vertex order).  Returns perm (new -> old).
__host__ __device__ inline uint64_t spread21(uint64_t x) {
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

__global__ void k_morton_keys(int n, const double* __restrict__ pts, double3 lo, double3 span,
                              uint64_t* __restrict__ key, int32_t* __restrict__ idx) {
  const double q = (double)((1 << 21) - 1);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double l[3] = {lo.x, lo.y, lo.z}, sp[3] = {span.x, span.y, span.z};
    uint64_t c[3];
    for (int k = 0; k < 3; ++k) {
      const double t = sp[k] > 0 ? (pts[3 * (size_t)i + k] - l[k]) / sp[k] : 0.0;
      c[k] = (uint64_t)llround(t * q);
    }
    key[i] = spread21(c[0]) | (spread21(c[1]) << 1) | (spread21(c[2]) << 2);
    idx[i] = i;
  }
}

// Bounding box of the points: per block the minima and maxima of x, y, z (part[6 b + k]).
__global__ void __launch_bounds__(256) k_bbox(int n, const double* __restrict__ pts, double* __restrict__ part) {
  __shared__ double sh[6][256];
  double v[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const double p = pts[3 * (size_t)i + k];
      v[k] = fmin(v[k], p);
      v[3 + k] = fmax(v[3 + k], p);
    }
  for (int k = 0; k < 6; ++k) sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 6; ++k)
        sh[k][threadIdx.x] = k < 3 ? fmin(sh[k][threadIdx.x], sh[k][threadIdx.x + st])
                                   : fmax(sh[k][threadIdx.x], sh[k][threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x < 6) part[6 * (size_t)blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

static std::vector<int32_t> morton_order(const double* d_pts, int n) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  {
    const int nb = (int)grid_for(n, 256, 4);
    DArr<double> part(6 * (size_t)nb);
    k_bbox<<<nb, 256>>>(n, d_pts, part.p);
    DEC_CHECK_LAUNCH();
    auto h = part.download();
    for (int b = 0; b < nb; ++b)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], h[6 * (size_t)b + k]);
        hi[k] = std::max(hi[k], h[6 * (size_t)b + 3 + k]);
      }
  }
  DArr<uint64_t> key(n), ks(n);
  DArr<int32_t> idx(n), is(n);
  k_morton_keys<<<grid_for(n, 256), 256>>>(n, d_pts, make_double3(lo[0], lo[1], lo[2]),
                                           make_double3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]), key.p, idx.p);
  DEC_CHECK_LAUNCH();
  size_t tmp_bytes = 0;
  DEC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.p, ks.p, idx.p, is.p, n, 0, 64));
  DArr<unsigned char> tmp(std::max<size_t>(1, tmp_bytes));
  DEC_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, key.p, ks.p, idx.p, is.p, n, 0, 64));
  return is.download();
}

// ---------------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------------
enum SweepMode { S_RESID = 0, S_JACOBI = 1, S_CHEB0 = 2, S_CHEBN = 3 };

template <class T>
struct SweepPrm {
  int mode;
  int zero_x;   // x is known to be zero: A x is skipped
  int d_is_x;   // Chebyshev: the previous iterate is zero (second step from zero), so it is not read
  T omega;      // Jacobi
  T inv_theta;  // Chebyshev first step
  T c1, c2;     // Chebyshev recurrence
};

// The coarse correction a fused sweep prolongs: fine row j's parents pa[j], pb[j] (equal for a kept
// vertex) and the coarse panels z.
template <class T>
struct ProlongSrc {
  const int32_t* pa;
  const int32_t* pb;
  const T* z;
  size_t cstride;
};

constexpr int TB = 256;

// State of the refinement loop that runs on the device (graph with a conditional WHILE node).
struct LoopState {
  int it;         // refinement steps run
  int conv;       // every right-hand side reached rtol
  int nrhs;       // right-hand sides in use (the rest of the panels is padding)
  int max_iters;
  double rtol;
  double worst;   // max_j ||b_j - A u_j|| / ||b_j|| at the last test
};


// Programmatic dependent launch: every kernel of a cycle is launched with the
// programmatic-serialization attribute and waits for its predecessor's results with
// griddepcontrol.wait before touching memory.  A kernel does not trigger its dependents early: the
// trigger is the implicit one as its blocks exit, so the next launch is prepared during the tail of
// the kernel before it without taking SM slots from the kernel's own blocks.
__device__ __forceinline__ void pdl_enter() {
#if __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// An L2 prefetch of the bytes [p, p + bytes) as one bulk request (cp.async.bulk.prefetch, no register
// held while it is in flight), trimmed inward to 16-byte boundaries so nothing outside the range is
// touched.  The row kernels issue it for the rows their CTA takes next, so those rows' streamed loads
// (b, the iterate, the operator rows) hit L2 instead of starting a DRAM round trip in front of the
// gathers that depend on them.
__device__ __forceinline__ void l2_prefetch(const void* p, size_t bytes) {
  size_t a = __cvta_generic_to_global(p), e = a + bytes;
  a = (a + 15) & ~size_t(15);
  e &= ~size_t(15);
  if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)));
}

// On unless DEC_B200_PDL=0.  Measured on B200 (same process, 10 L8 solves of 32 RHS; 20 L6
// single-RHS FP64 solves): without the attribute 10,440 solves/s and 0.928 ms; with dependents
// triggered at each kernel's start 10,250 and 0.891 ms (their blocks took SM slots from the large
// finest-level kernels); with the implicit trigger at exit 10,525 and 0.840 ms.
static bool pdl_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("DEC_B200_PDL");
    return !(v && v[0] == '0');
  }();
  return on;
}

template <class... KArgs, class... Args>
static void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  DEC_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
}

template <class... KArgs, class... Args>
static void launch_pdl_smem(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  DEC_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
}

// Storage type T of the panel vectors and the type C the kernels compute in: FP16 storage
// (precision 2) computes in FP32.
template <class T> struct Cmp { using t = T; };
template <> struct Cmp<__half> { using t = float; };
template <class T> using CT = typename Cmp<T>::t;

template <class T, int V> struct VecT;
template <> struct VecT<float, 1> { using t = float; };
template <> struct VecT<float, 2> { using t = float2; };
template <> struct VecT<float, 4> { using t = float4; };
template <> struct VecT<double, 1> { using t = double; };
template <> struct VecT<double, 2> { using t = double2; };
template <> struct VecT<__half, 1> { using t = unsigned short; };
template <> struct VecT<__half, 2> { using t = unsigned; };
template <> struct VecT<__half, 4> { using t = uint2; };
template <> struct VecT<__half, 8> { using t = uint4; };

// V consecutive values of storage type S as one vector load, converted to the compute type C.
template <class S, int V, class C>
__device__ __forceinline__ void ldv(const S* p, C (&r)[V]) {
  if constexpr (!std::is_same<S, __half>::value && sizeof(S) * V > 16) {  // several 16-byte loads
    constexpr int H = 16 / sizeof(S);
    static_assert(V % H == 0, "vector width");
#pragma unroll
    for (int c = 0; c < V / H; ++c) {
      S t[H];
      ldv<S, H>(p + c * H, t);
#pragma unroll
      for (int k = 0; k < H; ++k) r[c * H + k] = t[k];
    }
    return;
  } else {
  using VT = typename VecT<S, V>::t;
  VT t = *reinterpret_cast<const VT*>(p);
  if constexpr (std::is_same<S, __half>::value) {
    __half h[V];
    memcpy(h, &t, sizeof(VT));
#pragma unroll
    for (int q = 0; q < V; ++q) r[q] = __half2float(h[q]);
  } else {
    memcpy(r, &t, sizeof(VT));
  }
  }
}
template <class S, int V, class C>
__device__ __forceinline__ void stv(S* p, const C (&r)[V]) {
  if constexpr (!std::is_same<S, __half>::value && sizeof(S) * V > 16) {  // several 16-byte stores
    constexpr int H = 16 / sizeof(S);
    static_assert(V % H == 0, "vector width");
#pragma unroll
    for (int c = 0; c < V / H; ++c) {
      C t[H];
#pragma unroll
      for (int k = 0; k < H; ++k) t[k] = r[c * H + k];
      stv<S, H>(p + c * H, t);
    }
    return;
  } else {
  using VT = typename VecT<S, V>::t;
  VT t;
  if constexpr (std::is_same<S, __half>::value) {
    __half h[V];
#pragma unroll
    for (int q = 0; q < V; ++q) h[q] = __float2half_rn(r[q]);
    memcpy(&t, h, sizeof(VT));
  } else {
    memcpy(&t, r, sizeof(VT));
  }
  *reinterpret_cast<VT*>(p) = t;
  }
}
template <class T> __device__ __forceinline__ double to_d(T v) { return (double)v; }
template <> __device__ __forceinline__ double to_d<__half>(__half v) { return (double)__half2float(v); }
template <class T> __device__ __forceinline__ T from_d(double v) { return (T)v; }
template <> __device__ __forceinline__ __half from_d<__half>(double v) { return __float2half_rn((float)v); }

// Lanes per row: each lane moves one 16-byte vector (or the whole row when K is smaller).
// Algorithmic bytes of the kernels enqueued while a solve graph is captured (every streamed array
// read or written once, each gathered vector once, int32 indices; reduction partials of under a
// megabyte are not counted).  Set only around a capture, on the capturing thread.
static thread_local double* t_bytes = nullptr;
static inline void add_bytes(double b) {
  if (t_bytes) *t_bytes += b;
}

// The sweep's row arithmetic with each rounding pinned (no contraction choices left to the compiler),
// so the one-step sweeps and the two-step pair (k_cheb2) compute the same bits.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
// ½ za + ½ zb, one rounding (both halvings are exact): the prolongation's per-row term, shared by
// k_prolong and the sweeps that prolong on the fly so both give the same bits.
template <class C>
__device__ __forceinline__ C prolong_term(C za, C zb) {
  return fma_rn(C(0.5), zb, mul_rn(C(0.5), za));
}

// VV > 0 overrides the vector width (a tuned variant: VV = 2 on FP32 panels of K >= 8 puts twice the
// lanes on a row).
template <class T, int K, int VV = 0>
struct Lanes {
  static constexpr int V = VV > 0 ? VV
                           : std::is_same<T, float>::value  ? (K >= 4 ? 4 : K)
                           : std::is_same<T, __half>::value ? (K >= 8 ? 8 : K)
                                                            : (K >= 2 ? 2 : 1);
  static constexpr int LPR = K / V;        // lanes per row
  static constexpr int RPB = TB / LPR;     // rows per block
};

// The row kernels' FP32 forms of fixed width that do not add an iterate are compiled for 8 resident
// CTAs of 256 threads per SM (32 registers a thread: every warp slot holds a warp waiting on its loads),
// 6 for the shifted forms (SH, 40 registers), and, except the step that adds into the FP64 iterate (UPD)
// and a plain middle Chebyshev step, prefetch the rows their CTA takes next (l2_prefetch).  The other
// forms keep the code and the register counts they have without either: forced to 32 registers they
// spill, and with the prefetch alone their counts rose (FP64 panels 32-40 -> 70-124) and their occupancy
// fell.  Measured on B200 at icosphere L8 with 32 FP32 right-hand sides: k_sweep_ap 47.1 -> 44.0 us,
// the second step after the prolongation 67.4 -> 60.3 us (40 registers and 6 CTAs per SM before), the
// FP64 residual 103.5 -> 91.0 us, a middle Chebyshev step 64.6 -> 62.6 us (the bound alone; 69.7 us with
// the prefetch), the solve 10,525 -> 10,980 solves/s (10,715 with the UPD step prefetching too) with
// every iterate bit for bit; the batch of 512 shifted solves 57,900 -> 58,400-59,800 solves/s.
template <class T, bool KEEP, bool SHV = false>
constexpr int kRowCtas = (sizeof(T) == 4 && !KEEP) ? (SHV ? 6 : 8) : 0;  // 0: no bound given
template <class T, bool KEEP>
constexpr bool kRowPrefetch = sizeof(T) == 4 && !KEEP;

// One smoothing sweep / residual on all panels: r = b - A x, then
//   S_RESID : out = r
//   S_JACOBI: out = x + ω D⁻¹ r
//   S_CHEB0 : d = D⁻¹ r / θ; out = x + d
//   S_CHEBN : d = c1 (x - x_prev) + c2 D⁻¹ r; out = x + d, where x_prev, the iterate before x, is
//             what out holds on entry: the last direction is recomputed from the two iterates
//             (each row reads its own x_prev before writing over it), so no direction vector is
//             stored, a vector write less per step than keeping d in its own buffer
// SH: right-hand side j of panel p has its own operator A + cs[p*K + j] I (D likewise).
// UPD: the sweep's result is the refinement step's correction e, added straight to the FP64
// iterate (u += (double) e, the update pass's arithmetic) instead of being stored in out.
// PV (k_sweep_p, a Chebyshev step after the first): the previous iterate is formed from the coarse
// correction z as the prolongation would have stored it (prolong_term, same bits): 1: P z (the level's
// iterate was zero), 2: out + P z (out still holds the iterate before the correction); 3: P z, and the
// step's result is added to out (the iterate e the correction δ = the smoothed P z belongs to:
// out = e + δ, each row reading its e before writing; with UPD u += e + δ).
template <class T, int K, int W, bool SH, bool UPD = false, int VV = 0, int PV = 0>
__device__ __forceinline__ void sweep_rows(int n, int Wr, const int32_t* __restrict__ col,
                                           const CT<T>* __restrict__ off, const CT<T>* __restrict__ diag,
                                           const CT<T>* __restrict__ dinv, const T* __restrict__ b,
                                           const T* __restrict__ x, T* __restrict__ out, const SweepPrm<CT<T>>& prm,
                                           size_t pstride, const CT<T>* __restrict__ shf,
                                           double* __restrict__ u64 = nullptr, ProlongSrc<T> pz = {}) {
  using Ln = Lanes<T, K, VV>;
  using C = CT<T>;
  pdl_enter();
  constexpr int V = Ln::V;
  const int w = W > 0 ? W : Wr;
  const int lane = threadIdx.x % Ln::LPR;
  const size_t po = (size_t)blockIdx.y * pstride + (size_t)lane * V;
  C csv[V];
  if constexpr (SH) ldv<C, V>(shf + (size_t)blockIdx.y * K + (size_t)lane * V, csv);
  for (int i = blockIdx.x * Ln::RPB + threadIdx.x / Ln::LPR; i < n; i += gridDim.x * Ln::RPB) {
    const size_t ik = po + (size_t)i * K;
    // the CTA's next rows (i is their first row here), not in a plain middle Chebyshev step
    if (kRowPrefetch<T, W == 0 || UPD> && threadIdx.x == 0 && i + gridDim.x * Ln::RPB < n &&
        (PV != 0 || UPD || prm.mode != S_CHEBN)) {
      const int j = i + gridDim.x * Ln::RPB, m = min(Ln::RPB, n - j);
      const size_t pj = (size_t)blockIdx.y * pstride + (size_t)j * K, vb = (size_t)m * K * sizeof(T);
      l2_prefetch(b + pj, vb);
      if (!prm.zero_x) {
        l2_prefetch(x + pj, vb);
        l2_prefetch(col + (size_t)j * w, (size_t)m * w * sizeof(int32_t));
        l2_prefetch(off + (size_t)j * w, (size_t)m * w * sizeof(C));
        l2_prefetch(diag + j, (size_t)m * sizeof(C));
      }
      if (!SH && prm.mode != S_RESID) l2_prefetch(dinv + j, (size_t)m * sizeof(C));
      if ((PV == 0 || PV == 2) && prm.mode == S_CHEBN && !prm.d_is_x) l2_prefetch(out + pj, vb);
      if constexpr (PV == 3) l2_prefetch(out + pj, vb);
      if constexpr (PV != 0) {
        l2_prefetch(pz.pa + j, (size_t)m * sizeof(int32_t));
        l2_prefetch(pz.pb + j, (size_t)m * sizeof(int32_t));
      }
    }
    C r[V], xi[V];
    ldv<T, V>(b + ik, r);
    int pai = 0, pbi = 0;  // PV: the row's parents, loaded with the row's other indices
    if constexpr (PV != 0) {
      pai = __ldg(pz.pa + i);
      pbi = __ldg(pz.pb + i);
    }
    if (!prm.zero_x) {
      ldv<T, V>(x + ik, xi);
      const C dg = diag[i];
      C acc[V];
#pragma unroll
      for (int q = 0; q < V; ++q) {
        if constexpr (SH) acc[q] = mul_rn(add_rn(dg, csv[q]), xi[q]);
        else acc[q] = mul_rn(dg, xi[q]);
      }
      const int32_t* c = col + (size_t)i * w;
      const C* v = off + (size_t)i * w;
      if constexpr (W > 0) {
        int cs[W];
        C vs[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
          cs[s] = c[s];
          vs[s] = v[s];
        }
#pragma unroll
        for (int s = 0; s < W; ++s) {
          C nb[V];
          ldv<T, V>(x + po + (size_t)cs[s] * K, nb);
#pragma unroll
          for (int q = 0; q < V; ++q) acc[q] = fma_rn(vs[s], nb[q], acc[q]);
        }
      } else {
        for (int s = 0; s < w; ++s) {
          C nb[V];
          ldv<T, V>(x + po + (size_t)c[s] * K, nb);
          const C vv = v[s];
#pragma unroll
          for (int q = 0; q < V; ++q) acc[q] = fma_rn(vv, nb[q], acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < V; ++q) r[q] = sub_rn(r[q], acc[q]);
    } else {
#pragma unroll
      for (int q = 0; q < V; ++q) xi[q] = C(0);
    }
    if (prm.mode == S_RESID) {
      stv<T, V>(out + ik, r);
      continue;
    }
    C di[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      if constexpr (SH) di[q] = C(1) / (diag[i] + csv[q]);
      else di[q] = dinv[i];
    }
    C o[V];
    if (prm.mode == S_JACOBI) {
#pragma unroll
      for (int q = 0; q < V; ++q) o[q] = xi[q] + prm.omega * (di[q] * r[q]);
    } else if (prm.mode == S_CHEB0) {
      C dn[V];
#pragma unroll
      for (int q = 0; q < V; ++q) {
        dn[q] = mul_rn(mul_rn(di[q], r[q]), prm.inv_theta);
        o[q] = add_rn(xi[q], dn[q]);
      }
    } else {
      C dn[V];
      if (prm.d_is_x) {
#pragma unroll
        for (int q = 0; q < V; ++q) dn[q] = xi[q];
      } else {
        C xp[V];
        if constexpr (PV == 0 || PV == 2) ldv<T, V>(out + ik, xp);
        if constexpr (PV != 0) {  // + ½ z[pa_i] + ½ z[pb_i], k_prolong's arithmetic
          const T* zc = pz.z + (size_t)blockIdx.y * pz.cstride + (size_t)lane * V;
          C za[V], zb[V];
          ldv<T, V>(zc + (size_t)pai * K, za);
          ldv<T, V>(zc + (size_t)pbi * K, zb);
#pragma unroll
          for (int q = 0; q < V; ++q) xp[q] = add_rn(PV == 2 ? xp[q] : C(0), prolong_term(za[q], zb[q]));
        }
#pragma unroll
        for (int q = 0; q < V; ++q) dn[q] = sub_rn(xi[q], xp[q]);
      }
#pragma unroll
      for (int q = 0; q < V; ++q) {
        dn[q] = fma_rn(prm.c1, dn[q], mul_rn(prm.c2, mul_rn(di[q], r[q])));
        o[q] = add_rn(xi[q], dn[q]);
      }
    }
    if constexpr (PV == 3) {  // out = e + δ
      C ev[V];
      ldv<T, V>(out + ik, ev);
#pragma unroll
      for (int q = 0; q < V; ++q) o[q] = add_rn(ev[q], o[q]);
    }
    if constexpr (UPD) {
#pragma unroll
      for (int q = 0; q < V; ++q) u64[ik + q] += (double)(T)o[q];
    } else {
      stv<T, V>(out + ik, o);
    }
  }
}

template <class T, int K, int W, bool SH, int VV = 0>
__global__ void __launch_bounds__(TB, kRowCtas<T, W == 0, SH>)
    k_sweep(int n, int Wr, const int32_t* __restrict__ col,
                                              const CT<T>* __restrict__ off, const CT<T>* __restrict__ diag,
                                              const CT<T>* __restrict__ dinv, const T* __restrict__ b,
                                              const T* __restrict__ x, T* __restrict__ out,
                                              SweepPrm<CT<T>> prm, size_t pstride, const CT<T>* __restrict__ shf) {
  sweep_rows<T, K, W, SH, false, VV>(n, Wr, col, off, diag, dinv, b, x, out, prm, pstride, shf);
}

// The last sweep of a refinement step's V-cycles on the finest level with the step's update
// u += e fused in (FP32 / FP64 storage).
template <class T, int K, int W, bool SH, int VV = 0>
__global__ void __launch_bounds__(TB, kRowCtas<T, W == 0, SH>)
    k_sweep_u(int n, int Wr, const int32_t* __restrict__ col,
                                                const CT<T>* __restrict__ off, const CT<T>* __restrict__ diag,
                                                const CT<T>* __restrict__ dinv, const T* __restrict__ b,
                                                const T* __restrict__ x, T* __restrict__ out,
                                                SweepPrm<CT<T>> prm, size_t pstride, const CT<T>* __restrict__ shf,
                                                double* __restrict__ u64) {
  sweep_rows<T, K, W, SH, true, VV>(n, Wr, col, off, diag, dinv, b, x, out, prm, pstride, shf, u64);
}

// The second Chebyshev step after x (+)= P z with its previous iterate formed from z (PV = 1: P z,
// 2: out + P z), so the prolonged iterate is never read back.  UPD as k_sweep_u.
template <class T, int K, int W, bool SH, bool UPD, int PV, int VV = 0>
__global__ void __launch_bounds__(TB, kRowCtas<T, W == 0, SH>)
    k_sweep_p(int n, int Wr, const int32_t* __restrict__ col,
                                                const CT<T>* __restrict__ off, const CT<T>* __restrict__ diag,
                                                const CT<T>* __restrict__ dinv, const T* __restrict__ b,
                                                const T* __restrict__ x, T* __restrict__ out,
                                                SweepPrm<CT<T>> prm, size_t pstride, const CT<T>* __restrict__ shf,
                                                double* __restrict__ u64, ProlongSrc<T> pz) {
  sweep_rows<T, K, W, SH, UPD, VV, PV>(n, Wr, col, off, diag, dinv, b, x, out, prm, pstride, shf, u64, pz);
}

// Width of a level's A P rows (fine row -> coarse columns; at most 7 on binary-subdivision levels of
// rows with 6 off-diagonal slots: a kept vertex's own coarse copy and its neighbours', a midpoint's
// four coarse vertices), padded with weight 0.
constexpr int kApW = 8;

// The first Chebyshev step after the prolongation, from x0 = P z (ADD: x0 = e + P z, e the iterate
// before the correction), without x0 stored: r = b - A x0 with A x0 = (A P) z (+ A e), the product
// A P precomputed per level (apc / apv, kApW slots per row); out = x0 + D⁻¹ r / θ.  SH: A + cs I per
// right-hand side (A P then holds the unshifted product and cs x0 is added).
template <class T, int K, bool SH, bool ADD, int VV = 0>
__global__ void __launch_bounds__(TB, kRowCtas<T, ADD, SH>)
    k_sweep_ap(int n, const int32_t* __restrict__ col, const CT<T>* __restrict__ off,
                                                 const CT<T>* __restrict__ diag, const CT<T>* __restrict__ dinv,
                                                 const int32_t* __restrict__ apc, const CT<T>* __restrict__ apv,
                                                 const T* __restrict__ b, const T* __restrict__ e,
                                                 T* __restrict__ out, CT<T> inv_theta, size_t pstride,
                                                 const CT<T>* __restrict__ shf, ProlongSrc<T> pz) {
  using Ln = Lanes<T, K, VV>;
  using C = CT<T>;
  pdl_enter();
  constexpr int V = Ln::V;
  const int lane = threadIdx.x % Ln::LPR;
  const size_t po = (size_t)blockIdx.y * pstride + (size_t)lane * V;
  const T* zc = pz.z + (size_t)blockIdx.y * pz.cstride + (size_t)lane * V;
  C csv[V];
  if constexpr (SH) ldv<C, V>(shf + (size_t)blockIdx.y * K + (size_t)lane * V, csv);
  for (int i = blockIdx.x * Ln::RPB + threadIdx.x / Ln::LPR; i < n; i += gridDim.x * Ln::RPB) {
    const size_t ik = po + (size_t)i * K;
    if (kRowPrefetch<T, ADD> && threadIdx.x == 0 && i + gridDim.x * Ln::RPB < n) {  // the CTA's next rows
      const int j = i + gridDim.x * Ln::RPB, m = min(Ln::RPB, n - j);            // (i: their first)
      l2_prefetch(b + (size_t)blockIdx.y * pstride + (size_t)j * K, (size_t)m * K * sizeof(T));
      l2_prefetch(apc + (size_t)j * kApW, (size_t)m * kApW * sizeof(int32_t));
      l2_prefetch(apv + (size_t)j * kApW, (size_t)m * kApW * sizeof(C));
      if constexpr (!SH) l2_prefetch(dinv + j, (size_t)m * sizeof(C));
      if constexpr (ADD) l2_prefetch(e + (size_t)blockIdx.y * pstride + (size_t)j * K, (size_t)m * K * sizeof(T));
    }
    int pc[kApW];
    C pw[kApW];
#pragma unroll
    for (int k = 0; k < kApW; ++k) {
      pc[k] = apc[(size_t)i * kApW + k];
      pw[k] = apv[(size_t)i * kApW + k];
    }
    C r[V], pzi[V], x0[V], acc[V];
    ldv<T, V>(b + ik, r);
    // A P's slots 0 and 1 are the row's own parents, so P z at this row comes from the same gathers;
    // the padding slots (column -1: a midpoint row has four columns) are not gathered
    C zk[kApW][V];
#pragma unroll
    for (int k = 0; k < kApW; ++k) {
      if (k < 2 || pc[k] >= 0) {
        ldv<T, V>(zc + (size_t)pc[k] * K, zk[k]);
      } else {
#pragma unroll
        for (int q = 0; q < V; ++q) zk[k][q] = C(0);
      }
    }
#pragma unroll
    for (int q = 0; q < V; ++q) {
      pzi[q] = prolong_term(zk[0][q], zk[1][q]);  // P z at this row
      x0[q] = add_rn(C(0), pzi[q]);              // k_prolong's assignment (from +0)
    }
    if constexpr (ADD) {  // A e, as the sweep forms it
      C ei[V];
      ldv<T, V>(e + ik, ei);
      const C dg = diag[i];
#pragma unroll
      for (int q = 0; q < V; ++q) {
        if constexpr (SH) acc[q] = mul_rn(add_rn(dg, csv[q]), ei[q]);
        else acc[q] = mul_rn(dg, ei[q]);
      }
      int cs[6];
      C vs[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        cs[s] = col[(size_t)i * 6 + s];
        vs[s] = off[(size_t)i * 6 + s];
      }
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        C nb[V];
        ldv<T, V>(e + po + (size_t)cs[s] * K, nb);
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] = fma_rn(vs[s], nb[q], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < V; ++q) x0[q] = add_rn(ei[q], pzi[q]);
    } else {
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = C(0);
    }
#pragma unroll
    for (int k = 0; k < kApW; ++k)  // + (A P) z
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = fma_rn(pw[k], zk[k][q], acc[q]);
    if constexpr (SH) {  // + cs (P z) at this row (A e already carries its cs e)
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = fma_rn(csv[q], pzi[q], acc[q]);
    }
    C o[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      C di;
      if constexpr (SH) di = C(1) / (diag[i] + csv[q]);
      else di = dinv[i];
      const C rr = sub_rn(r[q], acc[q]);
      o[q] = add_rn(x0[q], mul_rn(mul_rn(di, rr), inv_theta));
    }
    stv<T, V>(out + ik, o);
  }
}

// Two Chebyshev steps in one pass (post-smoothing from a given iterate x0, FP32 panels): step 1
// (S_CHEB0) on the rows of a patch and of its 1-ring from x0 staged in shared memory with the 2-ring,
// then step 2 (S_CHEBN, x_prev = x0) on the patch rows from step 1's result, also in shared memory.
// x0 is read once with its halo, b once per step, and only the second step's result is written, where
// two sweeps move the operator twice and seven vectors.  A CTA takes one patch and KS of the panel's K
// right-hand sides (grid.y), four per lane.  The per-element arithmetic is sweep_rows', statement for
// statement with every rounding pinned (mul_rn / fma_rn ...), so the result is the two sweeps' bit for
// bit.  UPD: u += (double) x2 as k_sweep_u.
constexpr int kTwoStepRows = 512;  // the largest patch (the tuned value picks 128, 256 or 512)
template <int K, int KS, int W, bool UPD>
__global__ void __launch_bounds__(TB) k_cheb2(int n, int P, int max_local, const int32_t* __restrict__ hptr,
                                              const int32_t* __restrict__ h1n, const int32_t* __restrict__ halo,
                                              const int32_t* __restrict__ lptr, const uint16_t* __restrict__ lcol,
                                              const float* __restrict__ off, const float* __restrict__ diag,
                                              const float* __restrict__ dinv, const float* __restrict__ b,
                                              const float* __restrict__ x0, float* __restrict__ out, float inv_theta,
                                              float c1, float c2, size_t pstride, double* __restrict__ u64) {
  static_assert(KS % 4 == 0 && K % KS == 0, "slices of whole float4 lanes");
  constexpr int LPR = KS / 4, RPP = TB / LPR;
  extern __shared__ float4 tsm[];
  pdl_enter();
  const int patch = blockIdx.x;
  const int lane = threadIdx.x % LPR, sub = threadIdx.x / LPR;
  const size_t po = (size_t)blockIdx.z * pstride + (size_t)blockIdx.y * KS + (size_t)lane * 4;
  const int a = patch * P, pr = min(P, n - a);
  const int hb = hptr[patch], nh = hptr[patch + 1] - hb, n1 = h1n[patch];
  const int nloc = pr + nh, nl1 = pr + n1;
  float4* X0 = tsm;
  float4* X1 = tsm + (size_t)max_local * LPR;
  const uint16_t* lc = lcol + (size_t)lptr[patch] * W;
  for (int lr = sub; lr < nloc; lr += RPP) {  // x0 by asynchronous 16-byte copies, all in flight
    const int g = lr < pr ? a + lr : halo[hb + lr - pr];
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(X0 + lr * LPR + lane)),
                 "l"(x0 + po + (size_t)g * K)
                 : "memory");
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  for (int lr = sub; lr < nl1; lr += RPP) {  // step 1
    const int g = lr < pr ? a + lr : halo[hb + lr - pr];
    const float4 b4 = *reinterpret_cast<const float4*>(b + po + (size_t)g * K);
    const float4 x4 = X0[lr * LPR + lane];
    float r[4] = {b4.x, b4.y, b4.z, b4.w}, xi[4] = {x4.x, x4.y, x4.z, x4.w}, acc[4];
    const float dg = diag[g];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = mul_rn(dg, xi[q]);
    int cs[W];
    float vs[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      cs[k] = lc[lr * W + k];
      vs[k] = off[(size_t)g * W + k];
    }
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const float4 nb4 = X0[cs[k] * LPR + lane];
      const float nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma_rn(vs[k], nb[q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) r[q] = sub_rn(r[q], acc[q]);
    float di[4], o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) di[q] = dinv[g];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float dn = mul_rn(mul_rn(di[q], r[q]), inv_theta);
      o[q] = add_rn(xi[q], dn);
    }
    X1[lr * LPR + lane] = make_float4(o[0], o[1], o[2], o[3]);
  }
  __syncthreads();
  for (int lr = sub; lr < pr; lr += RPP) {  // step 2
    const int g = a + lr;
    const size_t ik = po + (size_t)g * K;
    const float4 b4 = *reinterpret_cast<const float4*>(b + ik);
    const float4 x4 = X1[lr * LPR + lane], p4 = X0[lr * LPR + lane];
    float r[4] = {b4.x, b4.y, b4.z, b4.w}, xi[4] = {x4.x, x4.y, x4.z, x4.w}, xp[4] = {p4.x, p4.y, p4.z, p4.w};
    float acc[4];
    const float dg = diag[g];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = mul_rn(dg, xi[q]);
    int cs[W];
    float vs[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      cs[k] = lc[lr * W + k];
      vs[k] = off[(size_t)g * W + k];
    }
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const float4 nb4 = X1[cs[k] * LPR + lane];
      const float nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma_rn(vs[k], nb[q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) r[q] = sub_rn(r[q], acc[q]);
    float di[4], o[4], dn[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) di[q] = dinv[g];
#pragma unroll
    for (int q = 0; q < 4; ++q) dn[q] = sub_rn(xi[q], xp[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dn[q] = fma_rn(c1, dn[q], mul_rn(c2, mul_rn(di[q], r[q])));
      o[q] = add_rn(xi[q], dn[q]);
    }
    if constexpr (UPD) {
#pragma unroll
      for (int q = 0; q < 4; ++q) u64[ik + q] += (double)(float)o[q];
    } else {
      *reinterpret_cast<float4*>(out + ik) = make_float4(o[0], o[1], o[2], o[3]);
    }
  }
}

// FP16-stored sweeps carry eight values per 16-byte access; unbounded they took 72 registers
// (3 blocks, 24 warps per SM).  Held to six 256-thread blocks per SM (40 registers, no spills;
// seven spilled) the L8 sweep went from 4.05 to 4.58 TB/s; the grid is sized to that residency.
constexpr int kSweepHalfBlocks = 6;

template <int K, int W, bool SH>
__global__ void __launch_bounds__(TB, kSweepHalfBlocks) k_sweep_h(
    int n, int Wr, const int32_t* __restrict__ col, const float* __restrict__ off, const float* __restrict__ diag,
    const float* __restrict__ dinv, const __half* __restrict__ b, const __half* __restrict__ x,
    __half* __restrict__ out, SweepPrm<float> prm, size_t pstride,
    const float* __restrict__ shf) {
  sweep_rows<__half, K, W, SH>(n, Wr, col, off, diag, dinv, b, x, out, prm, pstride, shf);
}

// Restriction R = row-normalised S (make_restriction, Multigrid.jl:595-612):
// rc[i] = (1/rs_i) rf[self_i] + Σ_e (0.5/rs_i) rf[mid_e], rs_i = 1 + deg_i / 2, terms in the
// reference's column order; the two weights per row come rounded to the compute type from setup
// (rw: (C)(1.0 / rs_i), (C)(0.5 / rs_i)).  A row's midpoints fill the front of its ridx slots (-1 after them).
// WQ > 0 (the slot count, known at compile time) loads every midpoint index first and issues all
// the row's gathers before the first sum, instead of one index -> gather -> sum chain per slot;
// the sums keep the same order, so the result is the same bit for bit.
template <class T, int K, int WQ = 0>
__global__ void __launch_bounds__(TB) k_restrict(int nc, int Wq, const int32_t* __restrict__ rself,
                                                 const int32_t* __restrict__ ridx, const CT<T>* __restrict__ rw,
                                                 const T* __restrict__ rf, T* __restrict__ rc, size_t fstride,
                                                 size_t cstride) {
  using Ln = Lanes<T, K>;
  using C = CT<T>;
  pdl_enter();
  constexpr int V = Ln::V;
  const int lane = threadIdx.x % Ln::LPR;
  const T* f = rf + (size_t)blockIdx.y * fstride + (size_t)lane * V;
  T* c = rc + (size_t)blockIdx.y * cstride + (size_t)lane * V;
  for (int i = blockIdx.x * Ln::RPB + threadIdx.x / Ln::LPR; i < nc; i += gridDim.x * Ln::RPB) {
    const C w1 = rw[2 * (size_t)i], wh = rw[2 * (size_t)i + 1];  // (C)(1 / rs_i), (C)(0.5 / rs_i)
    C acc[V], v[V];
    if constexpr (WQ > 0) {
      int m[WQ];
#pragma unroll
      for (int e = 0; e < WQ; ++e) m[e] = ridx[(size_t)i * WQ + e];
      C g[WQ][V];
      ldv<T, V>(f + (size_t)rself[i] * K, v);
#pragma unroll
      for (int e = 0; e < WQ; ++e) {
        if (m[e] >= 0) ldv<T, V>(f + (size_t)m[e] * K, g[e]);
      }
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = w1 * v[q];
#pragma unroll
      for (int e = 0; e < WQ; ++e) {
        if (m[e] >= 0) {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[q] += wh * g[e][q];
        }
      }
    } else {
      ldv<T, V>(f + (size_t)rself[i] * K, v);
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] = w1 * v[q];
      for (int e = 0; e < Wq; ++e) {
        int m = ridx[(size_t)i * Wq + e];
        if (m < 0) break;
        ldv<T, V>(f + (size_t)m * K, v);
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] += wh * v[q];
      }
    }
    stv<T, V>(c + (size_t)i * K, acc);
  }
}

// Prolongation and correction x_f += P z (P = Sᵀ, Multigrid.jl:774): every fine row takes
// ½ z[pa] + ½ z[pb] (pa = pb for a coarse vertex, which gives z exactly).  ASSIGN: x_f is known
// to be zero (a cycle started from x = 0 with no pre-smoothing), so it is neither read nor
// cleared first; the sum starts from +0 as the cleared buffer's did, which keeps every bit.
template <class T, int K, bool ASSIGN = false>
__global__ void __launch_bounds__(TB) k_prolong(int nf, const int32_t* __restrict__ pa, const int32_t* __restrict__ pb,
                                                const T* __restrict__ z, T* __restrict__ x, size_t fstride,
                                                size_t cstride) {
  using Ln = Lanes<T, K>;
  using C = CT<T>;
  pdl_enter();
  constexpr int V = Ln::V;
  const int lane = threadIdx.x % Ln::LPR;
  const T* zc = z + (size_t)blockIdx.y * cstride + (size_t)lane * V;
  T* xf = x + (size_t)blockIdx.y * fstride + (size_t)lane * V;
  for (int j = blockIdx.x * Ln::RPB + threadIdx.x / Ln::LPR; j < nf; j += gridDim.x * Ln::RPB) {
    C za[V], zb[V], xv[V];
    ldv<T, V>(zc + (size_t)pa[j] * K, za);
    ldv<T, V>(zc + (size_t)pb[j] * K, zb);
    if constexpr (ASSIGN) {
#pragma unroll
      for (int q = 0; q < V; ++q) xv[q] = C(0);
    } else {
      ldv<T, V>(xf + (size_t)j * K, xv);
    }
#pragma unroll
    for (int q = 0; q < V; ++q) xv[q] = add_rn(xv[q], prolong_term(za[q], zb[q]));
    stv<T, V>(xf + (size_t)j * K, xv);
  }
}

// General transfers (a hierarchy from caller matrices): dst (+)= M src on all panels, M row-major
// ELL with each row's columns increasing and -1 after the last, so a row's terms are added in the
// column order of SparseArrays' CSC product (from zero); ADD: the sum is then added to dst, as
// u += p * z adds the finished product.
template <class T, int K, bool ADD>
__global__ void __launch_bounds__(TB) k_transfer(int rows, int W, const int32_t* __restrict__ col,
                                                 const CT<T>* __restrict__ val, const T* __restrict__ src,
                                                 T* __restrict__ dst, size_t sstride, size_t dstride) {
  using Ln = Lanes<T, K>;
  using C = CT<T>;
  pdl_enter();
  constexpr int V = Ln::V;
  const int lane = threadIdx.x % Ln::LPR;
  const T* sp = src + (size_t)blockIdx.y * sstride + (size_t)lane * V;
  T* dp = dst + (size_t)blockIdx.y * dstride + (size_t)lane * V;
  for (int i = blockIdx.x * Ln::RPB + threadIdx.x / Ln::LPR; i < rows; i += gridDim.x * Ln::RPB) {
    C acc[V];
#pragma unroll
    for (int q = 0; q < V; ++q) acc[q] = C(0);
    for (int e = 0; e < W; ++e) {
      const int c = col[(size_t)i * W + e];
      if (c < 0) break;
      const C w = val[(size_t)i * W + e];
      C v[V];
      ldv<T, V>(sp + (size_t)c * K, v);
#pragma unroll
      for (int q = 0; q < V; ++q) acc[q] += w * v[q];
    }
    if constexpr (ADD) {
      C xv[V];
      ldv<T, V>(dp + (size_t)i * K, xv);
#pragma unroll
      for (int q = 0; q < V; ++q) xv[q] += acc[q];
      stv<T, V>(dp + (size_t)i * K, xv);
    } else {
      stv<T, V>(dp + (size_t)i * K, acc);
    }
  }
}

// Coarsest level: x = A⁻¹ b with the dense FP64 inverse.  One CTA per (row, panel): its TB threads
// are S = TB / K segments of the row's dot product for the K right-hand sides (segment g takes
// columns g, g + S, g + 2S, ... into two FP64 sums), and the segments' sums meet in a fixed-order
// tree in shared memory.  A thread per (row, right-hand side) running the whole row left a
// 162-vertex level's solve latency-bound at 21 CTAs.
template <class T, int K>
__global__ void __launch_bounds__(TB) k_coarse(int n, const double* __restrict__ ainv, const T* __restrict__ b,
                                               T* __restrict__ x, size_t pstride) {
  constexpr int S = TB / K;
  pdl_enter();
  const T* bb = b + (size_t)blockIdx.y * pstride;
  T* xx = x + (size_t)blockIdx.y * pstride;
  const int k = threadIdx.x % K, g = threadIdx.x / K;
  __shared__ double sh[TB];
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const double* a = ainv + (size_t)i * n;
    double s0 = 0.0, s1 = 0.0;
    int j = g;
    for (; j + S < n; j += 2 * S) {
      s0 += a[j] * to_d(bb[(size_t)j * K + k]);
      s1 += a[j + S] * to_d(bb[(size_t)(j + S) * K + k]);
    }
    if (j < n) s0 += a[j] * to_d(bb[(size_t)j * K + k]);
    sh[threadIdx.x] = s0 + s1;
    __syncthreads();
    for (int st = S / 2; st > 0; st >>= 1) {
      if (g < st) sh[threadIdx.x] += sh[threadIdx.x + st * K];
      __syncthreads();
    }
    if (g == 0) xx[(size_t)i * K + k] = from_d<T>(sh[k]);
    __syncthreads();
  }
}

// Coarsest-level solve for per-right-hand-side shifts c (coarse_solver 2): with
// L = M⁻¹ K (M = ⋆0, K symmetric) and M^{1/2} L M^{-1/2} = Q Λ Qᵀ,
// (L + c I)⁻¹ = E (Λ + c)⁻¹ F,  E = M^{-1/2} Q,  F = Qᵀ M^{1/2}.
// Phase 1: y = (Λ + c)⁻¹ F b (FP64 scratch); phase 2: x = E y.
template <class T, int K>
__global__ void __launch_bounds__(TB) k_coarse_eig1(int n, const double* __restrict__ F, const double* __restrict__ lam,
                                                    const double* __restrict__ cs, const T* __restrict__ b,
                                                    double* __restrict__ y, size_t pstride) {
  pdl_enter();
  const T* bb = b + (size_t)blockIdx.y * pstride;
  double* yy = y + (size_t)blockIdx.y * pstride;
  const int k = threadIdx.x % K;
  const double c = cs[(size_t)blockIdx.y * K + k];
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    const double* a = F + (size_t)i * n;
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += a[j] * to_d(bb[(size_t)j * K + k]);
    yy[(size_t)i * K + k] = s / (lam[i] + c);
  }
}

template <class T, int K>
__global__ void __launch_bounds__(TB) k_coarse_eig2(int n, const double* __restrict__ E, const double* __restrict__ y,
                                                    T* __restrict__ x, size_t pstride) {
  pdl_enter();
  const double* yy = y + (size_t)blockIdx.y * pstride;
  T* xx = x + (size_t)blockIdx.y * pstride;
  const int k = threadIdx.x % K;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    const double* a = E + (size_t)i * n;
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += a[j] * yy[(size_t)j * K + k];
    xx[(size_t)i * K + k] = from_d<T>(s);
  }
}

// Column-major RHS block (nrhs vectors of length n, reference vertex order) <-> panels of K in the
// level's internal order (iperm: reference -> internal).  A CTA moves a tile of kTile vertices x K
// right-hand sides of one panel through shared memory, so both sides move in whole runs: a panel
// row's K contiguous values, and kTile contiguous values of a vector.  (Element by element, one of
// the two sides was a scattered 8-byte access: 1.7 / 3.3 TB/s at L8 x 32.)  Padding right-hand
// sides (j >= nrhs) of the last panel are zero.
constexpr int kTile = 32;

template <int K>
__global__ void __launch_bounds__(256) k_vectors_to_panels(int n, int nrhs, const int32_t* __restrict__ iperm,
                                                           const double* __restrict__ src, double* __restrict__ dst) {
  __shared__ double t[kTile][K + 1];
  const int p = blockIdx.y;
  double* dp = dst + (size_t)p * n * K;
  for (int v0 = blockIdx.x * kTile; v0 < n; v0 += gridDim.x * kTile) {
    for (int e = threadIdx.x; e < kTile * K; e += blockDim.x) {
      const int k = e / kTile, dv = e % kTile, v = v0 + dv, j = p * K + k;
      t[dv][k] = (v < n && j < nrhs) ? src[(size_t)j * n + v] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * K; e += blockDim.x) {
      const int dv = e / K, k = e % K, v = v0 + dv;
      if (v < n) dp[(size_t)iperm[v] * K + k] = t[dv][k];
    }
    __syncthreads();
  }
}

template <int K>
__global__ void __launch_bounds__(256) k_panels_to_vectors(int n, int nrhs, const int32_t* __restrict__ iperm,
                                                           const double* __restrict__ src, double* __restrict__ dst) {
  __shared__ double t[kTile][K + 1];
  const int p = blockIdx.y;
  const double* sp = src + (size_t)p * n * K;
  for (int v0 = blockIdx.x * kTile; v0 < n; v0 += gridDim.x * kTile) {
    for (int e = threadIdx.x; e < kTile * K; e += blockDim.x) {
      const int dv = e / K, k = e % K, v = v0 + dv;
      if (v < n) t[dv][k] = sp[(size_t)iperm[v] * K + k];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * K; e += blockDim.x) {
      const int k = e / kTile, dv = e % kTile, v = v0 + dv, j = p * K + k;
      if (v < n && j < nrhs) dst[(size_t)j * n + v] = t[dv][k];
    }
    __syncthreads();
  }
}

// src (nrhs x n, reference order) -> dst panels; iperm: reference -> internal row.
static void to_panels(int n, int nrhs, int K, int np, const int32_t* iperm, const double* src, double* dst,
                      cudaStream_t s) {
  const dim3 g(grid_for(n, kTile, 16), np);
  switch (K) {
#define DEC_K(KK) \
  case KK: k_vectors_to_panels<KK><<<g, 256, 0, s>>>(n, nrhs, iperm, src, dst); break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
    default: throw Error(DEC_ERR_INVALID_ARG, "multigrid: bad panel width");
  }
}

// panels -> dst (nrhs x n, reference order).
static void from_panels(int n, int nrhs, int K, int np, const int32_t* iperm, const double* src, double* dst,
                        cudaStream_t s) {
  const dim3 g(grid_for(n, kTile, 16), np);
  switch (K) {
#define DEC_K(KK) \
  case KK: k_panels_to_vectors<KK><<<g, 256, 0, s>>>(n, nrhs, iperm, src, dst); break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
    default: throw Error(DEC_ERR_INVALID_ARG, "multigrid: bad panel width");
  }
}

// u += (double) z on the panels.
template <class T>
__global__ void k_axpy_update(size_t total, const T* __restrict__ z, double* __restrict__ u) {
  pdl_enter();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    u[q] += (double)z[q];
}

// FP16 storage: u += (double) z · escale[j] (z holds the correction of the scaled right-hand side).
template <int K>
__global__ void k_axpy_scaled(size_t total, size_t pstride, const __half* __restrict__ z,
                              const double* __restrict__ esc, double* __restrict__ u) {
  pdl_enter();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    u[q] += (double)__half2float(z[q]) * esc[(q / pstride) * K + q % K];
}

// FP16 storage: the finest right-hand side is the FP64 residual (rounded to FP32) over its RMS,
// b_j = r_j / rms_j, rms_j = sqrt(Σ r_j² / n) (1 for a zero residual), so the V-cycle works on
// values of order one; escale_j = rms_j undoes it in the next update.
template <int K>
__global__ void k_scale_half(int n, int np, const float* __restrict__ r, const double* __restrict__ norms,
                             __half* __restrict__ b, double* __restrict__ esc) {
  pdl_enter();
  auto rms_of = [&](int c) {
    const double v = sqrt(norms[c] / n);
    return (v > 0.0 && isfinite(v)) ? v : 1.0;
  };
  if (blockIdx.x == 0)
    for (int c = threadIdx.x; c < K * np; c += blockDim.x) esc[c] = rms_of(c);
  const size_t pstride = (size_t)n * K, total = pstride * np;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)((q / pstride) * K + q % K);
    b[q] = __float2half_rn((float)((double)r[q] / rms_of(c)));
  }
}

// FP64 residual r = b - A u on the panels, written in the inner precision T, with per-block
// partial sums of r² per right-hand side (deterministic two-stage reduction).
template <class T, int K, int W, bool SH>
__global__ void __launch_bounds__(TB, kRowCtas<T, W == 0, SH>)
    k_residual64(int n, int Wr, const int32_t* __restrict__ col,
                                                   const double* __restrict__ off, const double* __restrict__ diag,
                                                   const double* __restrict__ b, const double* __restrict__ u,
                                                   T* __restrict__ rT, double* __restrict__ partial, size_t pstride,
                                                   const double* __restrict__ cs) {
  using Ln = Lanes<double, K>;
  pdl_enter();
  constexpr int V = Ln::V;
  const int w = W > 0 ? W : Wr;
  const int lane = threadIdx.x % Ln::LPR;
  const size_t po = (size_t)blockIdx.y * pstride + (size_t)lane * V;
  double ss[V], csv[V];
#pragma unroll
  for (int q = 0; q < V; ++q) ss[q] = 0.0;
  if constexpr (SH) ldv<double, V>(cs + (size_t)blockIdx.y * K + (size_t)lane * V, csv);
  for (int i = blockIdx.x * Ln::RPB + threadIdx.x / Ln::LPR; i < n; i += gridDim.x * Ln::RPB) {
    const size_t ik = po + (size_t)i * K;
    if (kRowPrefetch<T, W == 0> && threadIdx.x == 0 && i + gridDim.x * Ln::RPB < n) {  // the CTA's next rows
      const int j = i + gridDim.x * Ln::RPB, m = min(Ln::RPB, n - j);            // (i: their first)
      const size_t pj = (size_t)blockIdx.y * pstride + (size_t)j * K, vb = (size_t)m * K * sizeof(double);
      l2_prefetch(u + pj, vb);
      l2_prefetch(b + pj, vb);
      l2_prefetch(col + (size_t)j * w, (size_t)m * w * sizeof(int32_t));
      l2_prefetch(off + (size_t)j * w, (size_t)m * w * sizeof(double));
      l2_prefetch(diag + j, (size_t)m * sizeof(double));
    }
    double ui[V], acc[V], bv[V];
    ldv<double, V>(u + ik, ui);
    ldv<double, V>(b + ik, bv);
    const double dg = diag[i];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      if constexpr (SH) acc[q] = (dg + csv[q]) * ui[q];
      else acc[q] = dg * ui[q];
    }
    const int32_t* c = col + (size_t)i * w;
    const double* v = off + (size_t)i * w;
    if constexpr (W > 0) {  // all index, value and neighbour loads before the products
      int cc[W];
      double vs[W], nb[W][V];
#pragma unroll
      for (int s = 0; s < W; ++s) {
        cc[s] = c[s];
        vs[s] = v[s];
      }
#pragma unroll
      for (int s = 0; s < W; ++s) ldv<double, V>(u + po + (size_t)cc[s] * K, nb[s]);
#pragma unroll
      for (int s = 0; s < W; ++s)
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] += vs[s] * nb[s][q];
    } else {
      for (int s = 0; s < w; ++s) {
        double nb[V];
        ldv<double, V>(u + po + (size_t)c[s] * K, nb);
        const double vv = v[s];
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] += vv * nb[q];
      }
    }
#pragma unroll
    for (int q = 0; q < V; ++q) {
      double r = bv[q] - acc[q];
      rT[ik + q] = (T)r;
      ss[q] += r * r;
    }
  }
  // reduce over the rows of this block per right-hand side (column lane*V + q)
  __shared__ double sh[TB * V];
#pragma unroll
  for (int q = 0; q < V; ++q) sh[threadIdx.x * V + q] = ss[q];
  __syncthreads();
  for (int stride = TB / 2; stride >= Ln::LPR; stride >>= 1) {
    if (threadIdx.x < stride)
#pragma unroll
      for (int q = 0; q < V; ++q) sh[threadIdx.x * V + q] += sh[(threadIdx.x + stride) * V + q];
    __syncthreads();
  }
  if (threadIdx.x < Ln::LPR)
#pragma unroll
    for (int q = 0; q < V; ++q)
      partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * K + threadIdx.x * V + q] = sh[threadIdx.x * V + q];
}

// Σ over blocks of the partial sums: out[p*K + k], one CTA per (panel, lane), tree-reduced in a
// fixed order (deterministic).
__global__ void __launch_bounds__(256) k_reduce_partials(int nblocks, int K, int npanels,
                                                         const double* __restrict__ partial,
                                                         double* __restrict__ out) {
  pdl_enter();
  const int q = blockIdx.x;
  const int p = q / K, k = q % K;
  double s = 0.0;
  for (int bq = threadIdx.x; bq < nblocks; bq += blockDim.x) s += partial[((size_t)p * nblocks + bq) * K + k];
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[q] = sh[0];
}

__global__ void k_loop_init(LoopState* st, int nrhs, int max_iters, double rtol) {
  st->it = 0;
  st->conv = 0;
  st->nrhs = nrhs;
  st->max_iters = max_iters;
  st->rtol = rtol;
  st->worst = 0.0;
}

// The refinement loop's test on the device: the worst relative residual over the right-hand
// sides (sqrt(r²) / sqrt(b²), sqrt(r²) where b = 0; a non-finite one counts as infinite), then
// the WHILE node's condition: another step when it is above rtol and max_iters is not reached.
__global__ void __launch_bounds__(256) k_ir_check(cudaGraphConditionalHandle h, const double* __restrict__ norms,
                                                  const double* __restrict__ bn2, LoopState* st) {
  const int nrhs = st->nrhs;
  double w = 0.0;
  int bad = 0;
  for (int j = threadIdx.x; j < nrhs; j += blockDim.x) {
    const double bn = sqrt(bn2[j]);
    const double rel = bn > 0 ? sqrt(norms[j]) / bn : sqrt(norms[j]);
    if (!isfinite(rel)) bad = 1;
    else w = fmax(w, rel);
  }
  __shared__ double sw[256];
  __shared__ int sb[256];
  sw[threadIdx.x] = w;
  sb[threadIdx.x] = bad;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) {
      sw[threadIdx.x] = fmax(sw[threadIdx.x], sw[threadIdx.x + k]);
      sb[threadIdx.x] |= sb[threadIdx.x + k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double worst = sb[0] ? HUGE_VAL : sw[0];
    st->worst = worst;
    const bool conv = worst <= st->rtol;
    st->conv = conv ? 1 : 0;
    const bool more = !conv && st->it < st->max_iters;
    if (more) ++st->it;
    cudaGraphSetConditional(h, more ? 1u : 0u);
  }
}

// Per-block partial sums of x² per right-hand side over the panels (same layout as k_residual64).
template <int K>
__global__ void __launch_bounds__(TB) k_panel_sumsq(int n, const double* __restrict__ x, double* __restrict__ partial,
                                                    size_t pstride) {
  const int k = threadIdx.x % K;
  const size_t po = (size_t)blockIdx.y * pstride;
  double ss = 0.0;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    double v = x[po + (size_t)i * K + k];
    ss += v * v;
  }
  __shared__ double sh[TB];
  sh[threadIdx.x] = ss;
  __syncthreads();
  for (int stride = TB / 2; stride >= K; stride >>= 1) {
    if (threadIdx.x < stride) sh[threadIdx.x] += sh[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < K) partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * K + threadIdx.x] = sh[threadIdx.x];
}

// k_panel_sumsq's partial sums of b², and the first refinement step's right-hand side from a zero
// initial guess: r = b - A·0 = b, rounded to the V-cycle's storage type as the residual kernel
// rounds it (so the step is the same bit for bit without the FP64 update and residual passes).
template <int K, class T>
__global__ void __launch_bounds__(TB) k_first_rhs(int n, const double* __restrict__ x, double* __restrict__ partial,
                                                  size_t pstride, T* __restrict__ r) {
  const int k = threadIdx.x % K;
  const size_t po = (size_t)blockIdx.y * pstride;
  double ss = 0.0;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    const size_t ik = po + (size_t)i * K + k;
    const double v = x[ik];
    r[ik] = (T)v;
    ss += v * v;
  }
  __shared__ double sh[TB];
  sh[threadIdx.x] = ss;
  __syncthreads();
  for (int stride = TB / 2; stride >= K; stride >>= 1) {
    if (threadIdx.x < stride) sh[threadIdx.x] += sh[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < K) partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * K + threadIdx.x] = sh[threadIdx.x];
}

// Power iteration for λmax(D⁻¹A): y = D⁻¹ A x (single vector, FP64).
__global__ void k_dinv_a(int n, int W, const int32_t* __restrict__ col, const double* __restrict__ off,
                         const double* __restrict__ diag, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double acc = diag[i] * x[i];
    for (int s = 0; s < W; ++s) acc += off[(size_t)i * W + s] * x[col[(size_t)i * W + s]];
    y[i] = acc / diag[i];
  }
}

// Start vector of the power iteration: a hash of each vertex's reference index.
__global__ void k_hash_init(int n, const int32_t* __restrict__ perm, double* x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint64_t z = (uint64_t)perm[i] * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    x[i] = 0.5 + (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
}

__global__ void k_sumsq_part(int n, const double* __restrict__ x, double* __restrict__ part) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += x[i] * x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_parts(int nb, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += part[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// x /= ||x|| with ||x||² read from the device
__global__ void k_scale_inv_norm(int n, const double* __restrict__ s2, double* x) {
  const double a = 1.0 / sqrt(*s2);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] *= a;
}

// Split layout of the level operator in the internal order: row i' (reference row perm[i'])
// gets its diagonal and W off-diagonal slots (reference column order kept, columns mapped
// through iperm; padding: own row, value 0).
__global__ void k_split(int n, int Wf, const int32_t* __restrict__ fcol, const double* __restrict__ fval, int W,
                        const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                        int32_t* __restrict__ col, double* __restrict__ off, double* __restrict__ diag,
                        double* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = perm[i];
    int q = 0;
    double dg = 0.0;
    for (int s = 0; s < Wf; ++s) {
      int c = fcol[(size_t)s * n + r];
      if (c < 0) continue;
      if (c == r) {
        dg += fval[(size_t)s * n + r];
      } else if (q < W) {
        col[(size_t)i * W + q] = iperm[c];
        off[(size_t)i * W + q] = fval[(size_t)s * n + r];
        ++q;
      }
    }
    for (; q < W; ++q) {
      col[(size_t)i * W + q] = i;
      off[(size_t)i * W + q] = 0.0;
    }
    diag[i] = dg;
    dinv[i] = 1.0 / dg;
  }
}


// ---------------------------------------------------------------------------------------------
// Krylov-CG smoother (the reference's smoother: Krylov.jl cg(A, b, u; itmax = steps) with warm
// start, atol = rtol = sqrt(eps), called at Multigrid.jl:860 / :871), FP64, one lane per
// right-hand side.  Every right-hand side j keeps its own scalars in scal[f * ntot + j]:
enum CgField { CG_GAMMA = 0, CG_PNORM2, CG_EPS, CG_ALPHA, CG_BETA, CG_ACTIVE, CG_UPDP, CG_ITER, CG_NFIELDS };
// and a kernel sequence per iteration: q = A p (+ p·q partials); reduce + decide α; Δx += α p,
// r -= α q (+ r·r partials); reduce + decide β; p = r + β p.

template <int K>
__device__ __forceinline__ void block_partials(double v, double* partial) {
  __shared__ double sh[TB];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int st = TB / 2; st >= K; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < K) partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * K + threadIdx.x] = sh[threadIdx.x];
}

// r = b - A x0 (x0 = 0 when zero_x), p = r, Δx = 0; partial r·r.
template <int K, int W>
__global__ void __launch_bounds__(TB) k_cg_init(int n, int Wr, const int32_t* __restrict__ col,
                                                const double* __restrict__ off, const double* __restrict__ diag,
                                                const double* __restrict__ b, const double* __restrict__ x0,
                                                int zero_x, double* __restrict__ r, double* __restrict__ p,
                                                double* __restrict__ dx, double* __restrict__ partial, size_t ps) {
  const int w = W > 0 ? W : Wr;
  const int k = threadIdx.x % K;
  const size_t po = (size_t)blockIdx.y * ps + k;
  double ss = 0.0;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    const size_t ik = po + (size_t)i * K;
    double rv = b[ik];
    if (!zero_x) {
      double acc = diag[i] * x0[ik];
      for (int s = 0; s < w; ++s) acc += off[(size_t)i * w + s] * x0[po + (size_t)col[(size_t)i * w + s] * K];
      rv = rv - acc;
    }
    r[ik] = rv;
    p[ik] = rv;
    dx[ik] = 0.0;
    ss += rv * rv;
  }
  block_partials<K>(ss, partial);
}

// q = A p for active right-hand sides; partial p·q.
template <int K, int W>
__global__ void __launch_bounds__(TB) k_cg_spmv(int n, int Wr, const int32_t* __restrict__ col,
                                                const double* __restrict__ off, const double* __restrict__ diag,
                                                const double* __restrict__ p, double* __restrict__ q,
                                                const double* __restrict__ scal, int ntot, double* __restrict__ partial,
                                                size_t ps) {
  const int w = W > 0 ? W : Wr;
  const int k = threadIdx.x % K;
  const int j = blockIdx.y * K + k;
  const bool active = scal[CG_ACTIVE * ntot + j] != 0.0;
  const size_t po = (size_t)blockIdx.y * ps + k;
  double ss = 0.0;
  if (active)
    for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
      const size_t ik = po + (size_t)i * K;
      double pi = p[ik];
      double acc = diag[i] * pi;
      for (int s = 0; s < w; ++s) acc += off[(size_t)i * w + s] * p[po + (size_t)col[(size_t)i * w + s] * K];
      q[ik] = acc;
      ss += pi * acc;
    }
  block_partials<K>(ss, partial);
}

// Δx += α p, r -= α q for active right-hand sides; partial r·r.
template <int K>
__global__ void __launch_bounds__(TB) k_cg_axpy(int n, const double* __restrict__ p, const double* __restrict__ q,
                                                double* __restrict__ dx, double* __restrict__ r,
                                                const double* __restrict__ scal, int ntot, double* __restrict__ partial,
                                                size_t ps) {
  const int k = threadIdx.x % K;
  const int j = blockIdx.y * K + k;
  const bool active = scal[CG_ACTIVE * ntot + j] != 0.0;
  const double a = scal[CG_ALPHA * ntot + j];
  const size_t po = (size_t)blockIdx.y * ps + k;
  double ss = 0.0;
  if (active)
    for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
      const size_t ik = po + (size_t)i * K;
      dx[ik] += a * p[ik];
      double rv = r[ik] + (-a) * q[ik];
      r[ik] = rv;
      ss += rv * rv;
    }
  block_partials<K>(ss, partial);
}

// p = r + β p where the right-hand side continues.
template <int K>
__global__ void __launch_bounds__(TB) k_cg_pupd(int n, const double* __restrict__ r, double* __restrict__ p,
                                                const double* __restrict__ scal, int ntot, size_t ps) {
  const int k = threadIdx.x % K;
  const int j = blockIdx.y * K + k;
  if (scal[CG_UPDP * ntot + j] == 0.0) return;
  const double bt = scal[CG_BETA * ntot + j];
  const size_t po = (size_t)blockIdx.y * ps + k;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    const size_t ik = po + (size_t)i * K;
    p[ik] = r[ik] + bt * p[ik];
  }
}

// x = Δx + x0 (Krylov adds the warm start back at the end).
template <int K>
__global__ void __launch_bounds__(TB) k_cg_finish(int n, const double* __restrict__ x0, int zero_x,
                                                  const double* __restrict__ dx, double* __restrict__ out, size_t ps) {
  const int k = threadIdx.x % K;
  const size_t po = (size_t)blockIdx.y * ps + k;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += gridDim.x * (TB / K)) {
    const size_t ik = po + (size_t)i * K;
    out[ik] = zero_x ? dx[ik] : dx[ik] + x0[ik];
  }
}

enum CgPhase { CG_PH_INIT = 0, CG_PH_ALPHA = 1, CG_PH_BETA = 2 };

// One CTA per right-hand side: sum the block partials (fixed tree order) and take the CG
// decisions of Krylov.jl's cg for that phase.
__global__ void __launch_bounds__(256) k_cg_scalar(int phase, int nb, int K, int ntot, int itmax,
                                                   const double* __restrict__ partial, double* __restrict__ scal) {
  const int j = blockIdx.x;
  const int pnl = j / K, k = j % K;
  double s = 0.0;
  for (int bq = threadIdx.x; bq < nb; bq += blockDim.x) s += partial[((size_t)pnl * nb + bq) * K + k];
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double v = sh[0];
  const double eps = 2.220446049250313e-16, rt = 1.4901161193847656e-08;  // eps(Float64), sqrt(eps)
  double* S = scal;
  auto F = [&](int f) -> double& { return S[(size_t)f * ntot + j]; };
  if (phase == CG_PH_INIT) {
    const double gamma = v;
    F(CG_GAMMA) = gamma;
    F(CG_ITER) = 0.0;
    F(CG_UPDP) = 0.0;
    F(CG_ALPHA) = 0.0;
    if (gamma == 0.0) {  // x0 is a zero-residual solution: return it
      F(CG_ACTIVE) = 0.0;
      return;
    }
    const double rnorm = sqrt(gamma);
    F(CG_EPS) = rt + rt * rnorm;
    F(CG_PNORM2) = gamma;
    const bool solved = rnorm <= F(CG_EPS);
    F(CG_ACTIVE) = (!solved && itmax > 0) ? 1.0 : 0.0;
  } else if (phase == CG_PH_ALPHA) {
    if (F(CG_ACTIVE) == 0.0) return;
    const double pAp = v, pn2 = F(CG_PNORM2);
    if (pAp <= eps * pn2 && fabs(pAp) <= eps * pn2) {  // zero curvature
      F(CG_ACTIVE) = 0.0;
      F(CG_ALPHA) = 0.0;
      return;
    }
    F(CG_ALPHA) = F(CG_GAMMA) / pAp;
  } else {
    F(CG_UPDP) = 0.0;
    if (F(CG_ACTIVE) == 0.0) return;
    const double gnext = v;
    const double rnorm = sqrt(gnext);
    const bool solved = (rnorm <= F(CG_EPS)) || (rnorm + 1.0 <= 1.0);
    const double iter = F(CG_ITER) + 1.0;
    F(CG_ITER) = iter;
    if (!solved) {
      const double beta = gnext / F(CG_GAMMA);
      F(CG_BETA) = beta;
      F(CG_PNORM2) = gnext + beta * beta * F(CG_PNORM2);
      F(CG_GAMMA) = gnext;
    }
    const bool more = !solved && iter < (double)itmax;
    F(CG_UPDP) = more ? 1.0 : 0.0;
    F(CG_ACTIVE) = more ? 1.0 : 0.0;
  }
}

// ---------------------------------------------------------------------------------------------
// Hierarchy
// ---------------------------------------------------------------------------------------------
struct Level {
  std::unique_ptr<dec_mesh> mesh;
  std::unique_ptr<dec_op> op;  // A = L + shift I (reference order, sorted ELL, FP64): exports, parity
  int n = 0, W = 0;
  std::vector<int32_t> perm, iperm;  // internal -> reference, reference -> internal
  DArr<int32_t> dperm, diperm;
  DArr<int32_t> col;
  DArr<double> off64, diag64, dinv64;
  DArr<float> off32, diag32, dinv32;
  DArr<float4> mtab;  // learned smoother: per-row coupling features
  double lmax = 0.0;
  // transfer to the next coarser level (internal numbering on both sides)
  int nc = 0, Wq = 0;
  DArr<int32_t> rself, ridx, pa, pb;
  DArr<double> rs;
  DArr<double> rw64;  // per coarse row (1 / rs, 0.5 / rs), FP64 and rounded to FP32
  DArr<float> rw32;
  // A P (kApW coarse columns per fine row) for the first sweep after a prolongation (k_sweep_ap);
  // built for binary-subdivision levels with rows of 6 off-diagonal slots
  bool ap_ok = false;
  DArr<int32_t> apc;
  DArr<double> apv64;
  DArr<float> apv32;
  // a hierarchy from caller matrices: general R (nc x n) and P (n x nc) as row-major ELL
  bool gen = false;
  int Wr = 0, Wp = 0;
  DArr<int32_t> rcol, pcol;
  DArr<double> rval64, pval64;
  DArr<float> rval32, pval32;
  // tuned FP32 sweep variant per panel width 8 / 16 / 32 (index 3 / 4 / 5), cached per table version
  mutable unsigned sweep_tuned_at[6] = {0, 0, 0, 0, 0, 0};
  mutable int sweep_vv[6] = {0, 0, 0, 0, 0, 0};
  // The two-step Chebyshev pair (k_cheb2): patches of P consecutive internal rows, each with its
  // 1-ring halo H1 then its 2-ring halo H2 (internal row ids in halo[hptr[p] ..], |H1| = h1n[p]), and
  // the local column of every slot of the patch and H1 rows (lcol, rows from lptr[p]; local numbering:
  // patch rows, then H1, then H2).  Built on the host the first time it is used.
  struct TwoStep {
    int P = 0, npatch = 0, max_local = 0, max_l1 = 0;
    double sum_local = 0, sum_l1 = 0;
    DArr<int32_t> hptr, h1n, halo, lptr;
    DArr<uint16_t> lcol;
  } ts;
};

template <class T>
struct LevelBufs {
  DArr<T> x, y, b, d;  // x / y ping-pong, b right-hand side, d the learned sweep's residual / CG direction
  DArr<T> q, e;        // CG smoother: A p and the accumulated correction Δx (CG mode only)
  const CT<T>* cs = nullptr;  // per-RHS shifts (coarse_solver 2), K * npanels, shared by all levels
};

struct Workspace {
  int K = 0, npanels = 0, prec = 0;
  std::vector<LevelBufs<float>> f32;
  std::vector<LevelBufs<double>> f64;
  std::vector<LevelBufs<__half>> f16;  // precision 2: FP16 panels, FP32 arithmetic
  DArr<float> r32;                     // precision 2: the FP64 residual rounded to FP32
  DArr<double> escale;                 // precision 2: per-RHS scale of the FP16 right-hand side
  DArr<double> B64, U64;      // finest FP64 panels
  DArr<double> partial, norms;
  DArr<double> scal;          // CG smoother: per-right-hand-side scalars (CgField x K*npanels)
  DArr<double> ucm, bcm;      // column-major device copies for host-buffer solves
  DArr<double> pu[3], pb[3];  // staging slots of pipelined host-buffer solves
  DArr<double> bn2;           // ||b_j||² (device refinement loop)
  DArr<LoopState> loop;       // device refinement loop state
  // the whole refinement loop (Jacobi / Chebyshev): [0] from a given initial guess, [1] from zero
  cudaGraphExec_t solve_graph[2] = {nullptr, nullptr};
  int64_t solve_pre[2] = {0, 0}, solve_body = 0;  // kernel nodes before / inside its loop
  double solve_pre_bytes[2] = {0.0, 0.0}, solve_body_bytes = 0.0;  // their algorithmic bytes
  int nblocks = 0;
  DArr<double> Ubak;          // learned smoother: the iterate before a refinement step
  DArr<double> cs64;          // coarse_solver 2: per-RHS total shifts (K * npanels)
  DArr<float> cs32;
  DArr<double> ceig;          // coarse_solver 2: FP64 scratch of the coarsest solve
  std::vector<double> hcs64;  // host staging of the shifts
  std::vector<float> hcs32;
  cudaGraphExec_t graph[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // GraphKind
  int64_t launches[5] = {0, 0, 0, 0, 0};                                     // kernel nodes per graph
  void drop_graphs() {
    for (auto& g : graph) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
    for (auto& g : solve_graph) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
  }
  ~Workspace() { drop_graphs(); }
};

}  // namespace decb

struct dec_mg {
  dec_mg_options opt{};
  std::vector<decb::Level> lv;  // 0 = finest
  std::vector<int> steps;       // per-level smoother steps before and after the coarse correction
                                // (MultigridData.steps); empty: opt.pre / opt.post everywhere
  int pre_at(int l) const { return steps.empty() ? opt.pre : steps[l]; }
  int post_at(int l) const { return steps.empty() ? opt.post : steps[l]; }
  decb::DArr<double> ainv;      // dense inverse of level lc (FP64, internal order)
  decb::DArr<double> eigE, eigF, eigL;  // coarse_solver 2: (L + c I)⁻¹ = E (Λ + c)⁻¹ F on level lc
  int lc = 0;                   // level at which cycles solve directly
  std::map<long long, std::unique_ptr<decb::Workspace>> ws;
  std::map<long long, int> tuned;  // (nrhs, precision) -> panel width chosen by the autotuner
  cudaStream_t cap = nullptr;      // capture stream
  const dec_mlp* mlp = nullptr;    // learned smoother network (not owned)
  uint64_t epoch = 0;              // bumped whenever workspaces or their graphs are dropped
  bool force_plain = false;        // set while capturing the plain-smoother fallback cycle
  int mlp_engine = -1;             // kernel engine of the network when the graphs were captured
  uint64_t mlp_version = 0;        // its parameter version then (the tcgen05 kernels take b1 .. b3 by value)
  // Pipelined host-buffer solves (submit / wait): copy-in, compute and copy-out streams, per
  // staging slot the events start, copied in, computed, copied out, and the loop state read back.
  static constexpr int kSlots = 3;
  cudaStream_t pipe[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t pev[kSlots][4] = {};
  decb::LoopState* hstate = nullptr;  // pinned, one per slot
  struct Pending {
    bool active = false;
    uint64_t ticket = 0;
    decb::Workspace* w = nullptr;
    int nrhs = 0;
    bool guess = false;
  } pend[kSlots];
  uint64_t next_ticket = 1;
  ~dec_mg() {
    for (cudaStream_t p : pipe)
      if (p) cudaStreamSynchronize(p);
    ws.clear();
    for (auto& sl : pev)
      for (cudaEvent_t e : sl)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t p : pipe)
      if (p) cudaStreamDestroy(p);
    if (hstate) cudaFreeHost(hstate);
    if (cap) cudaStreamDestroy(cap);
  }
};

namespace decb {

void mg_default_options(dec_mg_options& o) {
  o = dec_mg_options{};
  o.levels = 1;
  o.center = DEC_CIRCUMCENTER;
  o.project_radius = 0.0;
  o.shift = 0.0;
  o.smoother = DEC_SMOOTH_CHEBYSHEV;
  o.pre = 3;
  o.post = 3;
  o.omega = 0.8;
  o.cheb_ratio = 4.0;
  o.coarse_solver = 0;
  o.precision = 0;
  o.rhs_block = 0;
  o.mu = 1;
  o.inner_cycles = 1;
  o.reorder = 1;
  o.coarse_max = 0;
  o.fallback_rho = 0.5;
  o.device_loop = 1;
}

// λmax(D⁻¹A) of a level: 30 power steps from a hashed start vector, all on the device (the norm
// never leaves it until the end).
static double power_lmax(const Level& L) {
  if (L.n < 2) return 1.0;
  const int T = 256;
  const int nb = (int)std::min<long long>(4LL * num_sms(), ((long long)L.n + T - 1) / T);
  DArr<double> x(L.n), y(L.n), part(nb), s(1);
  k_hash_init<<<grid_for(L.n, T), T>>>(L.n, L.dperm.p, x.p);
  for (int it = 0; it < 30; ++it) {
    k_sumsq_part<<<nb, T>>>(L.n, x.p, part.p);
    k_sum_parts<<<1, T>>>(nb, part.p, s.p);
    k_scale_inv_norm<<<grid_for(L.n, T), T>>>(L.n, s.p, x.p);
    k_dinv_a<<<grid_for(L.n, T), T>>>(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, x.p, y.p);
    std::swap(x.p, y.p);
  }
  k_sumsq_part<<<nb, T>>>(L.n, x.p, part.p);
  k_sum_parts<<<1, T>>>(nb, part.p, s.p);
  DEC_CHECK_LAUNCH();
  const double lam = std::sqrt(s.download()[0]);
  return lam * 1.05;  // power iteration approaches λmax from below
}

// Dense inverse of the coarsest operator (Gauss-Jordan, partial pivoting), reference order.
static std::vector<double> dense_inverse(const dec_op& op, int n) {
  auto c = op.col.download();
  auto vv = op.val64.download();
  std::vector<double> A((size_t)n * n, 0.0), Ainv((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int q = 0; q < op.W; ++q) {
      int j = c[(size_t)q * n + i];
      if (j >= 0) A[(size_t)i * n + j] += vv[(size_t)q * n + i];
    }
  for (int i = 0; i < n; ++i) Ainv[(size_t)i * n + i] = 1.0;
  double amax = 0.0;
  for (double a : A) amax = std::max(amax, std::fabs(a));
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[(size_t)i * n + k]) > std::fabs(A[(size_t)p * n + k])) p = i;
    if (std::fabs(A[(size_t)p * n + k]) <= 1e-13 * amax)
      throw Error(DEC_ERR_INVALID_ARG,
                  "multigrid: the coarsest operator is singular; use a positive shift or coarse_solver = 1");
    if (p != k)
      for (int j = 0; j < n; ++j) {
        std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
        std::swap(Ainv[(size_t)k * n + j], Ainv[(size_t)p * n + j]);
      }
    double piv = A[(size_t)k * n + k];
    for (int j = 0; j < n; ++j) {
      A[(size_t)k * n + j] /= piv;
      Ainv[(size_t)k * n + j] /= piv;
    }
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      double f = A[(size_t)i * n + k];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        A[(size_t)i * n + j] -= f * A[(size_t)k * n + j];
        Ainv[(size_t)i * n + j] -= f * Ainv[(size_t)k * n + j];
      }
    }
  }
  return Ainv;
}

// Eigendecomposition of a symmetric matrix (row-major n x n, overwritten) by the cyclic Jacobi
// method: rotations zero each off-diagonal entry in turn until the off-diagonal mass is below
// 1e-30 of the total.  Returns the eigenvalues; Q (row-major) holds the eigenvectors as columns.
static std::vector<double> symmetric_eigen(std::vector<double>& A, int n, std::vector<double>& Q) {
  Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
  auto at = [&](int i, int j) -> double& { return A[(size_t)i * n + j]; };
  double total = 0.0;
  for (double a : A) total += a * a;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double offm = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) offm += 2.0 * at(i, j) * at(i, j);
    if (offm <= 1e-30 * total) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = at(p, q);
        if (apq == 0.0) continue;
        const double theta = (at(q, q) - at(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A J (columns p, q)
          const double akp = at(k, p), akq = at(k, q);
          at(k, p) = c * akp - sn * akq;
          at(k, q) = sn * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- Jᵀ A (rows p, q)
          const double apk = at(p, k), aqk = at(q, k);
          at(p, k) = c * apk - sn * aqk;
          at(q, k) = sn * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {  // Q <- Q J
          const double qkp = Q[(size_t)k * n + p], qkq = Q[(size_t)k * n + q];
          Q[(size_t)k * n + p] = c * qkp - sn * qkq;
          Q[(size_t)k * n + q] = sn * qkp + c * qkq;
        }
      }
  }
  std::vector<double> lam(n);
  for (int i = 0; i < n; ++i) lam[i] = at(i, i);
  return lam;
}

// Coarse solver 2: with M = ⋆0 of the level and S = M^{1/2} L M^{-1/2} = Q Λ Qᵀ (symmetrised),
// E = M^{-1/2} Q and F = Qᵀ M^{1/2}, permuted to the level's internal order.
static void build_eigen_coarse(dec_mg& mg, const Level& C) {
  const int n = C.n;
  auto c = C.op->col.download();
  auto vv = C.op->val64.download();
  auto m0 = C.mesh->m.star0.download();
  std::vector<double> S((size_t)n * n, 0.0), Q;
  for (int i = 0; i < n; ++i)
    for (int q = 0; q < C.op->W; ++q) {
      const int j = c[(size_t)q * n + i];
      if (j >= 0) S[(size_t)i * n + j] += std::sqrt(m0[i]) * vv[(size_t)q * n + i] / std::sqrt(m0[j]);
    }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double a = 0.5 * (S[(size_t)i * n + j] + S[(size_t)j * n + i]);
      S[(size_t)i * n + j] = S[(size_t)j * n + i] = a;
    }
  std::vector<double> lam = symmetric_eigen(S, n, Q);
  std::vector<double> E((size_t)n * n), F((size_t)n * n);
  for (int ii = 0; ii < n; ++ii) {  // internal row / column ii <-> reference perm[ii]
    const int r = C.perm[ii];
    for (int k = 0; k < n; ++k) {
      E[(size_t)ii * n + k] = Q[(size_t)r * n + k] / std::sqrt(m0[r]);
      F[(size_t)k * n + ii] = Q[(size_t)r * n + k] * std::sqrt(m0[r]);
    }
  }
  mg.eigE.upload(E);
  mg.eigF.upload(F);
  mg.eigL.upload(lam);
}

// ---- GalerkinMode (Multigrid.jl:740-748): A_{k+1} = R_k A_k P_k on the host ------------------
struct HostCSC {
  int m = 0, n = 0;
  std::vector<int32_t> cp, ri;
  std::vector<double> v;
};

// C = X Y column by column, as SparseArrays' spmatmul: C[i, j] = Σ_k X[i, k] Y[k, j] summed over
// the stored entries of Y[:, j] in row order; each column's rows sorted.
static HostCSC csc_mul(const HostCSC& X, const HostCSC& Y) {
  require(X.n == Y.m, "multigrid: Galerkin product dimension mismatch");
  HostCSC C;
  C.m = X.m;
  C.n = Y.n;
  C.cp.assign(Y.n + 1, 0);
  std::vector<double> acc(X.m, 0.0);
  std::vector<int32_t> stamp(X.m, -1), rows;
  for (int j = 0; j < Y.n; ++j) {
    rows.clear();
    for (int q = Y.cp[j]; q < Y.cp[j + 1]; ++q) {
      const int k = Y.ri[q];
      const double y = Y.v[q];
      for (int p = X.cp[k]; p < X.cp[k + 1]; ++p) {
        const int i = X.ri[p];
        const double prod = X.v[p] * y;
        if (stamp[i] != j) {
          stamp[i] = j;
          rows.push_back(i);
          acc[i] = prod;
        } else {
          acc[i] += prod;
        }
      }
    }
    std::sort(rows.begin(), rows.end());
    for (int i : rows) {
      C.ri.push_back(i);
      C.v.push_back(acc[i]);
    }
    C.cp[j + 1] = (int32_t)C.ri.size();
  }
  return C;
}

static HostCSC csc_transpose(const HostCSC& A) {
  HostCSC T;
  T.m = A.n;
  T.n = A.m;
  T.cp.assign(A.m + 1, 0);
  for (int r : A.ri) T.cp[r + 1]++;
  for (int i = 0; i < A.m; ++i) T.cp[i + 1] += T.cp[i];
  T.ri.resize(A.ri.size());
  T.v.resize(A.v.size());
  std::vector<int32_t> pos(T.cp.begin(), T.cp.end() - 1);
  for (int j = 0; j < A.n; ++j)
    for (int p = A.cp[j]; p < A.cp[j + 1]; ++p) {
      const int q = pos[A.ri[p]]++;
      T.ri[q] = j;
      T.v[q] = A.v[p];
    }
  return T;
}

// The level operator (reference numbering, sorted ELL) as a CSC.
static HostCSC csc_of_op(const dec_op& op) {
  const int n = (int)op.rows;
  auto c = op.col.download();
  auto v = op.val64.download();
  HostCSC R;  // CSR of the rows first (as a CSC of the transpose), then transposed
  R.m = n;
  R.n = n;
  R.cp.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    for (int q = 0; q < op.W; ++q)
      if (c[(size_t)q * n + i] >= 0) {
        R.ri.push_back(c[(size_t)q * n + i]);
        R.v.push_back(v[(size_t)q * n + i]);
      }
    R.cp[i + 1] = (int32_t)R.ri.size();
  }
  return csc_transpose(R);
}

// subdivision_matrix(BinarySubdivision(), topo) (Multigrid.jl:191-219) of coarse topology c:
// nv_c x (nv_c + ne_c), identity then ½ at min(∂v0, ∂v1) and max for each edge's midpoint.
static HostCSC subdivision_csc(const HostLevel& c) {
  HostCSC S;
  S.m = c.nv;
  S.n = c.nv + c.ne;
  S.cp.assign(S.n + 1, 0);
  for (int i = 0; i < c.nv; ++i) {
    S.ri.push_back(i);
    S.v.push_back(1.0);
    S.cp[i + 1] = (int32_t)S.ri.size();
  }
  for (int e = 0; e < c.ne; ++e) {
    const int a = std::min(c.ev0[e], c.ev1[e]), b = std::max(c.ev0[e], c.ev1[e]);
    S.ri.push_back(a);
    S.v.push_back(0.5);
    S.ri.push_back(b);
    S.v.push_back(0.5);
    S.cp[c.nv + e + 1] = (int32_t)S.ri.size();
  }
  return S;
}

// A_coarse = R A P with R = make_restriction(S) (each S entry over its row's sum, Multigrid.jl:
// 595-612) and P = Sᵀ, in the reference's evaluation order (R * A) * P; returned as a CSR.
static void galerkin_product(const dec_op& A, const HostLevel& c, std::vector<int32_t>& rp,
                             std::vector<int32_t>& ci, std::vector<double>& vv) {
  HostCSC S = subdivision_csc(c);
  std::vector<double> rs(S.m, 0.0);
  for (size_t k = 0; k < S.v.size(); ++k) rs[S.ri[k]] += S.v[k];
  HostCSC Rm = S;
  for (size_t k = 0; k < Rm.v.size(); ++k) Rm.v[k] = S.v[k] / rs[S.ri[k]];
  HostCSC P = csc_transpose(S);
  HostCSC Ac = csc_mul(csc_mul(Rm, csc_of_op(A)), P);
  HostCSC T = csc_transpose(Ac);  // rows of Ac, columns sorted
  rp = T.cp;
  ci = T.ri;
  vv = T.v;
}

static void build_level_operator(Level& L, double shift, bool reorder, dec_op* given = nullptr) {
  if (given) L.op.reset(given);
  else L.op.reset(op_create_impl(L.mesh.get(), DEC_OP_HELMHOLTZ0, shift, DEC_F64));
  L.n = L.mesh ? L.mesh->m.nv : (int)L.op->rows;
  if (reorder && L.mesh) {
    L.perm = morton_order(L.mesh->m.pts.p, L.n);
  } else {
    L.perm.resize(L.n);
    std::iota(L.perm.begin(), L.perm.end(), 0);
  }
  L.iperm.resize(L.n);
  for (int i = 0; i < L.n; ++i) L.iperm[L.perm[i]] = i;
  L.dperm.upload(L.perm);
  L.diperm.upload(L.iperm);
  // off-diagonal slots: the maximum vertex degree (a Galerkin operator: its widest row)
  L.W = given || !L.mesh ? std::max(1, L.op->W) : std::max(1, L.mesh->m.max_v2e);
  L.col.alloc((size_t)L.n * L.W);
  L.off64.alloc((size_t)L.n * L.W);
  L.diag64.alloc(L.n);
  L.dinv64.alloc(L.n);
  k_split<<<grid_for(L.n, 256), 256>>>(L.n, L.op->W, L.op->col.p, L.op->val64.p, L.W, L.dperm.p, L.diperm.p,
                                       L.col.p, L.off64.p, L.diag64.p, L.dinv64.p);
  DEC_CHECK_LAUNCH();
  cast_array(L.off64, L.off32);
  cast_array(L.diag64, L.diag32);
  cast_array(L.dinv64, L.dinv32);
}

// Restriction lists, on the device: per internal coarse row ic (reference vertex i = cperm[ic])
// its copy on the fine level, the fine midpoints of its incident edges in increasing edge order
// (the coarse mesh's d0ᵀ rows, sorted by edge; -1 after them in the Wq slots) and the row sum of S
// (1.0, then 0.5 per edge, in column order).
__global__ void k_restrict_lists(int nc, int Wq, const int32_t* __restrict__ cperm, const int32_t* __restrict__ fiperm,
                                 const int32_t* __restrict__ v2e_ptr, const int32_t* __restrict__ v2e,
                                 int32_t* __restrict__ rself, int32_t* __restrict__ ridx, double* __restrict__ rs) {
  for (int ic = blockIdx.x * blockDim.x + threadIdx.x; ic < nc; ic += gridDim.x * blockDim.x) {
    const int i = cperm[ic];
    rself[ic] = fiperm[i];
    double s = 1.0;
    int q = 0;
    for (int p = v2e_ptr[i]; p < v2e_ptr[i + 1] && q < Wq; ++p, ++q) {
      const int e = abs(v2e[p]) - 1;
      ridx[(size_t)ic * Wq + q] = fiperm[nc + e];
      s += 0.5;
    }
    for (; q < Wq; ++q) ridx[(size_t)ic * Wq + q] = -1;
    rs[ic] = s;
  }
}

// Prolongation lists: fine row jf (reference vertex j = fperm[jf]) takes ½ z[pa] + ½ z[pb], pa = pb
// = the coarse vertex itself for j < nc, else the endpoints of coarse edge j - nc, lower first.
__global__ void k_prolong_lists(int nf, int nc, const int32_t* __restrict__ fperm, const int32_t* __restrict__ ciperm,
                                const int32_t* __restrict__ cev0, const int32_t* __restrict__ cev1,
                                int32_t* __restrict__ pa, int32_t* __restrict__ pb) {
  for (int jf = blockIdx.x * blockDim.x + threadIdx.x; jf < nf; jf += gridDim.x * blockDim.x) {
    const int j = fperm[jf];
    if (j < nc) {
      pa[jf] = pb[jf] = ciperm[j];
    } else {
      const int e = j - nc;
      pa[jf] = ciperm[min(cev0[e], cev1[e])];
      pb[jf] = ciperm[max(cev0[e], cev1[e])];
    }
  }
}

// The restriction's two weights per coarse row, (1 / rs, 0.5 / rs), in FP64 and rounded to FP32.
__global__ void k_restrict_weights(int nc, const double* __restrict__ rs, double* __restrict__ w64,
                                   float* __restrict__ w32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
    const double a = 1.0 / rs[i], h = 0.5 / rs[i];
    w64[2 * (size_t)i] = a;
    w64[2 * (size_t)i + 1] = h;
    w32[2 * (size_t)i] = (float)a;
    w32[2 * (size_t)i + 1] = (float)h;
  }
}

// Transfers between fine level F and its coarse level C, in the internal numbering of both, from
// the coarse mesh's device topology (a simplicial complex: no edge has ∂v0 = ∂v1).
static void build_transfers(Level& F, const Level& C) {
  const Mesh& c = C.mesh->m;
  F.nc = c.nv;
  F.Wq = std::max(1, c.max_v2e);
  F.rself.alloc(c.nv);
  F.ridx.alloc((size_t)c.nv * F.Wq);
  F.rs.alloc(c.nv);
  F.pa.alloc(F.n);
  F.pb.alloc(F.n);
  const int T = 256;
  k_restrict_lists<<<grid_for(c.nv, T), T>>>(c.nv, F.Wq, C.dperm.p, F.diperm.p, c.v2e_ptr.p, c.v2e.p, F.rself.p,
                                             F.ridx.p, F.rs.p);
  F.rw64.alloc(2 * (size_t)c.nv);
  F.rw32.alloc(2 * (size_t)c.nv);
  k_restrict_weights<<<grid_for(c.nv, T), T>>>(c.nv, F.rs.p, F.rw64.p, F.rw32.p);
  k_prolong_lists<<<grid_for(F.n, T), T>>>(F.n, c.nv, F.dperm.p, C.diperm.p, c.ev0.p, c.ev1.p, F.pa.p, F.pb.p);
  DEC_CHECK_LAUNCH();
}

// Row i of A P (A the level operator, P the prolongation from the next coarser level): slots 0 and 1
// are the row's own parents pa_i, pb_i (for a kept vertex pa_i twice, the second at weight 0, so a
// sweep reads P z at the row from slots 0 and 1), then the parents of its six neighbours; equal coarse
// columns merged into their first slot (FP64 sums of ½ a_ij); kApW slots, padded with column -1 at
// weight 0.  *bad = 1 if a row has more than kApW slots.
__global__ void k_ap_build(int n, const int32_t* __restrict__ col, const double* __restrict__ off,
                           const double* __restrict__ diag, const int32_t* __restrict__ pa,
                           const int32_t* __restrict__ pb, int32_t* __restrict__ apc, double* __restrict__ apv,
                           int* __restrict__ bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c[16];
    double w[16];
    c[0] = pa[i];
    c[1] = pb[i];
    w[0] = w[1] = 0.0;
    int m = 2;
    auto put = [&](int p, double v) {
      for (int k = 0; k < m; ++k)
        if (c[k] == p) {
          w[k] += v;
          return;
        }
      c[m] = p;
      w[m] = v;
      ++m;
    };
    const double h = 0.5 * diag[i];
    put(pa[i], h);
    put(pb[i], h);
    for (int s = 0; s < 6; ++s) {
      const int j = col[(size_t)i * 6 + s];
      const double hj = 0.5 * off[(size_t)i * 6 + s];
      put(pa[j], hj);
      put(pb[j], hj);
    }
    if (m > kApW) {
      atomicExch(bad, 1);
      m = kApW;
    }
    for (int k = 0; k < kApW; ++k) {
      apc[(size_t)i * kApW + k] = k < m ? c[k] : -1;
      apv[(size_t)i * kApW + k] = k < m ? w[k] : 0.0;
    }
  }
}

static void build_ap(Level& L) {
  L.ap_ok = false;
  if (L.W != 6 || L.gen || !L.pa.p) return;
  L.apc.alloc((size_t)L.n * kApW);
  L.apv64.alloc((size_t)L.n * kApW);
  DArr<int> bad(1);
  DEC_CUDA(cudaMemset(bad.p, 0, sizeof(int)));
  k_ap_build<<<grid_for(L.n, 256), 256>>>(L.n, L.col.p, L.off64.p, L.diag64.p, L.pa.p, L.pb.p, L.apc.p, L.apv64.p,
                                          bad.p);
  DEC_CHECK_LAUNCH();
  if (bad.download()[0]) {  // wider rows than the slots: this level keeps the stored prolongation
    L.apc.release();
    L.apv64.release();
    return;
  }
  cast_array(L.apv64, L.apv32);
  L.ap_ok = true;
}

dec_mg* mg_create(const dec_mesh_desc& cd, const dec_mg_options& o) {
  require(o.levels >= 0 && o.levels <= 12, "multigrid: levels must be in [0, 12]");
  require(o.smoother >= 0 && o.smoother <= 3, "multigrid: unknown smoother");
  require(o.smoother != DEC_SMOOTH_LEARNED || (o.fallback_rho > 0 && o.fallback_rho <= 1),
          "multigrid: fallback_rho must be in (0, 1]");
  require(o.smoother != DEC_SMOOTH_CG || o.precision == 0, "multigrid: the CG smoother runs in FP64 (precision 0)");
  require(o.pre >= 0 && o.post >= 0 && o.pre <= 16 && o.post <= 16, "multigrid: sweeps must be in [0, 16]");
  require(o.mu == 1 || o.mu == 2, "multigrid: mu must be 1 (V) or 2 (W)");
  require(o.precision >= 0 && o.precision <= 2, "multigrid: precision must be 0, 1 or 2");
  require(o.precision != 2 || o.smoother == DEC_SMOOTH_JACOBI || o.smoother == DEC_SMOOTH_CHEBYSHEV,
          "multigrid: FP16 storage (precision 2) needs the Jacobi or Chebyshev smoother");
  require(o.cheb_ratio > 1.0, "multigrid: cheb_ratio must exceed 1");
  require(o.inner_cycles >= 1 && o.inner_cycles <= 8, "multigrid: inner_cycles must be in [1, 8]");
  require(o.coarse_max >= 0 && o.coarse_max <= 1024, "multigrid: coarse_max must be in [0, 1024]");
  require(o.coarse_solver >= 0 && o.coarse_solver <= 2, "multigrid: coarse_solver must be 0, 1 or 2");
  require(o.coarse_solver != 2 || (o.smoother == DEC_SMOOTH_JACOBI || o.smoother == DEC_SMOOTH_CHEBYSHEV),
          "multigrid: per-RHS shifts (coarse_solver 2) need the Jacobi or Chebyshev smoother");
  require(o.galerkin == 0 || o.galerkin == 1, "multigrid: galerkin must be 0 or 1");
  require(o.device_loop == 0 || o.device_loop == 1, "multigrid: device_loop must be 0 or 1");
  require(!(o.galerkin && o.coarse_solver == 2),
          "multigrid: per-RHS shifts (coarse_solver 2) need every level's own Laplacian (not GalerkinMode)");
  auto mg = std::make_unique<dec_mg>();
  mg->opt = o;
  {
    auto m = std::make_unique<dec_mesh>();
    dec_mesh_desc d = cd;
    d.center = o.center;
    m->m.build(d);
    mg->lv.resize(o.levels + 1);
    mg->lv[o.levels].mesh = std::move(m);
  }
  // every finer level is the binary subdivision of the one below it, refined on the device; the
  // first refinement carries the coarse mesh's orientation flips (orient!'s seeds)
  DArr<int8_t> dflip;
  if (o.levels >= 1) dflip.upload(component_flips(host_level(mg->lv[o.levels].mesh->m)));
  for (int l = 1; l <= o.levels; ++l) {
    auto fm = std::make_unique<dec_mesh>();
    fm->m.refine_from(mg->lv[o.levels - l + 1].mesh->m, o.project_radius, l == 1 ? dflip.p : nullptr, o.center);
    mg->lv[o.levels - l].mesh = std::move(fm);
  }
  // coarse_solver 2 keeps every level's operator the Laplacian; the shifts come per RHS
  for (int l = 0; l <= o.levels; ++l) {
    if (o.galerkin && l > 0) {  // A_l = R A_{l-1} P over the coarse topology of level l
      std::vector<int32_t> rp, ci;
      std::vector<double> vv;
      const HostLevel hc = host_level(mg->lv[l].mesh->m);
      galerkin_product(*mg->lv[l - 1].op, hc, rp, ci, vv);
      dec_op* A = op_from_csr_impl(mg->lv[l].mesh.get(), hc.nv, rp, ci, vv);
      build_level_operator(mg->lv[l], 0.0, o.reorder != 0, A);
    } else {
      build_level_operator(mg->lv[l], o.coarse_solver == 2 ? 0.0 : o.shift, o.reorder != 0);
    }
  }
  for (int l = 0; l <= o.levels; ++l) {
    Level& L = mg->lv[l];
    if (l < o.levels) {
      build_transfers(L, mg->lv[l + 1]);
      build_ap(L);
    }
    L.lmax = power_lmax(L);
  }
  mg->lc = o.levels;
  if (o.coarse_max > 0)
    for (int l = 0; l <= o.levels; ++l)
      if (mg->lv[l].n <= o.coarse_max) {
        mg->lc = l;
        break;
      }
  if (o.smoother == DEC_SMOOTH_CG) mg->lc = o.levels;  // the reference runs CG on its coarsest level
  const Level& C = mg->lv[mg->lc];
  if (o.coarse_solver == 2) {
    require(C.n <= 640, "multigrid: coarse_solver 2 needs a coarsest level of at most 640 vertices (coarse_max)");
    build_eigen_coarse(*mg, C);
  }
  if (o.coarse_solver == 0 && o.smoother != DEC_SMOOTH_CG) {
    auto ai = dense_inverse(*C.op, C.n);
    std::vector<double> ap((size_t)C.n * C.n);
    for (int i = 0; i < C.n; ++i)
      for (int j = 0; j < C.n; ++j) ap[(size_t)i * C.n + j] = ai[(size_t)C.perm[i] * C.n + C.perm[j]];
    mg->ainv.upload(ap);
  }
  DEC_CUDA(cudaStreamCreateWithFlags(&mg->cap, cudaStreamNonBlocking));
  DEC_CUDA(cudaDeviceSynchronize());
  return mg.release();
}

// Row-major ELL (rows x W, -1 padding) of a CSR, for the general transfers.
static int ell_rows(const std::vector<int32_t>& rp, const std::vector<int32_t>& ci, const std::vector<double>& vv,
                    DArr<int32_t>& col, DArr<double>& val64, DArr<float>& val32) {
  const int rows = (int)rp.size() - 1;
  int W = 1;
  for (int i = 0; i < rows; ++i) W = std::max(W, rp[i + 1] - rp[i]);
  std::vector<int32_t> c((size_t)rows * W, -1);
  std::vector<double> v((size_t)rows * W, 0.0);
  for (int i = 0; i < rows; ++i)
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      c[(size_t)i * W + (q - rp[i])] = ci[q];
      v[(size_t)i * W + (q - rp[i])] = vv[q];
    }
  col.upload(c);
  val64.upload(v);
  cast_array(val64, val32);
  return W;
}

// MultigridData(g, r, p, s) (Multigrid.jl:538-546): levels from the caller's operators,
// restrictions and prolongations, in the caller's numbering (no locality order: there are no points).
dec_mg* mg_create_from_csc(int nl, const dec_csc* ops, const dec_csc* rs, const dec_csc* ps, const int* steps,
                           const dec_mg_options& o) {
  require(nl >= 1 && nl <= 32, "multigrid: the number of levels must be in [1, 32]");
  require(ops != nullptr && (nl == 1 || (rs != nullptr && ps != nullptr)),
          "multigrid: null operators / restrictions / prolongations");
  require(o.smoother == DEC_SMOOTH_JACOBI || o.smoother == DEC_SMOOTH_CHEBYSHEV || o.smoother == DEC_SMOOTH_CG,
          "multigrid: a hierarchy from matrices takes the CG, Jacobi or Chebyshev smoother");
  require(o.smoother != DEC_SMOOTH_CG || o.precision == 0, "multigrid: the CG smoother runs in FP64 (precision 0)");
  require(o.pre >= 0 && o.post >= 0 && o.pre <= 16 && o.post <= 16, "multigrid: sweeps must be in [0, 16]");
  require(o.mu == 1 || o.mu == 2, "multigrid: mu must be 1 (V) or 2 (W)");
  require(o.precision >= 0 && o.precision <= 2, "multigrid: precision must be 0, 1 or 2");
  require(o.precision != 2 || o.smoother != DEC_SMOOTH_CG,
          "multigrid: FP16 storage (precision 2) needs the Jacobi or Chebyshev smoother");
  require(o.cheb_ratio > 1.0, "multigrid: cheb_ratio must exceed 1");
  require(o.inner_cycles >= 1 && o.inner_cycles <= 8, "multigrid: inner_cycles must be in [1, 8]");
  require(o.coarse_max >= 0 && o.coarse_max <= 1024, "multigrid: coarse_max must be in [0, 1024]");
  require(o.coarse_solver == 0 || o.coarse_solver == 1,
          "multigrid: a hierarchy from matrices takes coarse_solver 0 (dense) or 1 (the smoother)");
  require(o.device_loop == 0 || o.device_loop == 1, "multigrid: device_loop must be 0 or 1");
  if (steps)
    for (int k = 0; k < nl; ++k) require(steps[k] >= 0 && steps[k] <= 16, "multigrid: steps must be in [0, 16]");
  for (int k = 0; k < nl; ++k) require(ops[k].m == ops[k].n && ops[k].m >= 1, "multigrid: operators must be square");
  for (int k = 0; k + 1 < nl; ++k) {
    require(rs[k].m == ops[k + 1].m && rs[k].n == ops[k].m,
            "multigrid: restriction k must be (size of level k+1) x (size of level k)");
    require(ps[k].m == ops[k].m && ps[k].n == ops[k + 1].m,
            "multigrid: prolongation k must be (size of level k) x (size of level k+1)");
  }
  auto mg = std::make_unique<dec_mg>();
  mg->opt = o;
  mg->opt.levels = nl - 1;
  mg->opt.reorder = 0;
  mg->opt.galerkin = 0;
  mg->lv.resize(nl);
  if (steps) mg->steps.assign(steps, steps + nl);
  for (int k = 0; k < nl; ++k) {
    std::vector<int32_t> rp, ci;
    std::vector<double> vv;
    csc_to_csr(ops[k], rp, ci, vv);
    dec_op* A = op_from_csr_impl(nullptr, ops[k].m, rp, ci, vv);
    A->kind = DEC_OP_GENERAL;
    build_level_operator(mg->lv[k], 0.0, false, A);
    if (o.smoother != DEC_SMOOTH_CG) {
      for (double d : mg->lv[k].diag64.download())
        require(d != 0.0 && std::isfinite(d),
                "multigrid: the Jacobi / Chebyshev smoothers need a nonzero diagonal on every level");
    }
  }
  for (int k = 0; k + 1 < nl; ++k) {
    Level& L = mg->lv[k];
    L.gen = true;
    L.nc = mg->lv[k + 1].n;
    std::vector<int32_t> rp, ci;
    std::vector<double> vv;
    csc_to_csr(rs[k], rp, ci, vv);
    L.Wr = ell_rows(rp, ci, vv, L.rcol, L.rval64, L.rval32);
    csc_to_csr(ps[k], rp, ci, vv);
    L.Wp = ell_rows(rp, ci, vv, L.pcol, L.pval64, L.pval32);
  }
  for (Level& L : mg->lv) L.lmax = power_lmax(L);
  mg->lc = nl - 1;
  if (o.coarse_max > 0)
    for (int l = 0; l < nl; ++l)
      if (mg->lv[l].n <= o.coarse_max) {
        mg->lc = l;
        break;
      }
  if (o.smoother == DEC_SMOOTH_CG) mg->lc = nl - 1;
  const Level& C = mg->lv[mg->lc];
  if (o.coarse_solver == 0 && o.smoother != DEC_SMOOTH_CG) {
    require(C.n <= 8192, "multigrid: the dense coarsest solve takes at most 8192 unknowns (coarse_max)");
    mg->ainv.upload(dense_inverse(*C.op, C.n));  // identity order: internal = caller numbering
  }
  DEC_CUDA(cudaStreamCreateWithFlags(&mg->cap, cudaStreamNonBlocking));
  DEC_CUDA(cudaDeviceSynchronize());
  return mg.release();
}

void mg_destroy(dec_mg* mg) { delete mg; }

static const Level& level_at(const dec_mg* mg, int level) {
  require(mg != nullptr, "multigrid: null handle");
  require(level >= 0 && level < (int)mg->lv.size(), "multigrid: level out of range");
  return mg->lv[level];
}

void mg_level_info(const dec_mg* mg, int level, int64_t* nv, int64_t* ne, int64_t* nt, double* lmax) {
  const Level& L = level_at(mg, level);
  if (nv) *nv = L.n;
  if (ne) *ne = L.mesh ? L.mesh->m.ne : 0;
  if (nt) *nt = L.mesh ? L.mesh->m.nt : 0;
  if (lmax) *lmax = L.lmax;
}

const dec_mesh* mg_level_mesh(const dec_mg* mg, int level) {
  const Level& L = level_at(mg, level);
  require(L.mesh != nullptr, "multigrid: a hierarchy built from matrices has no level meshes");
  return L.mesh.get();
}
const dec_op* mg_level_op(const dec_mg* mg, int level) { return level_at(mg, level).op.get(); }

// ---------------------------------------------------------------------------------------------
// Cycle enqueue
// ---------------------------------------------------------------------------------------------
// The level's operator arrays in the compute type of storage type T (FP32 for FP16 storage).
template <class T>
static const CT<T>* pick(const DArr<double>& a64, const DArr<float>& a32) {
  if constexpr (std::is_same<T, double>::value) return a64.p;
  else return a32.p;
}

template <class T, int K>
static dim3 row_grid(int n, int np) {
  return dim3(grid_for((long long)n, Lanes<T, K>::RPB, 8), np);
}

// CTAs of k_restrict<T, K, WQ> resident per SM (queried once): its grid stays within one wave, so
// no partial second wave of grid-stride CTAs trails the rest.
template <class T, int K, int WQ>
static int restrict_ctas() {
  static const int ctas = [] {
    int o = 0;
    DEC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_restrict<T, K, WQ>, TB, 0));
    return std::max(1, o);
  }();
  return ctas;
}

// R r_f into the coarse level's panels; the unrolled kernel where a coarse vertex has at most six
// midpoints (every level of the refined icosphere and of the triangulated grids).
template <class T, int K>
static void launch_restrict(const Level& L, const Level& Cl, const T* r, T* bc, int np, cudaStream_t s,
                            bool pdl = true) {
  if (L.gen) {
    const dim3 g = row_grid<T, K>(Cl.n, np);
    const size_t fs = (size_t)L.n * K, cs = (size_t)Cl.n * K;
    add_bytes((double)Cl.n * L.Wr * (4.0 + sizeof(CT<T>)) + (double)(fs + cs) * np * sizeof(T));
    const CT<T>* v = pick<T>(L.rval64, L.rval32);
    if (pdl)
      launch_pdl(k_transfer<T, K, false>, g, dim3(TB), s, Cl.n, L.Wr, (const int32_t*)L.rcol.p, v, r, bc, fs, cs);
    else
      k_transfer<T, K, false><<<g, TB, 0, s>>>(Cl.n, L.Wr, L.rcol.p, v, r, bc, fs, cs);
    return;
  }
  auto kern = L.Wq == 6 ? k_restrict<T, K, 6> : k_restrict<T, K>;
  dim3 g = row_grid<T, K>(Cl.n, np);
  const int ctas = L.Wq == 6 ? restrict_ctas<T, K, 6>() : restrict_ctas<T, K, 0>();
  g.x = std::min<unsigned>(g.x, (unsigned)(ctas * num_sms()));
  const size_t fs = (size_t)L.n * K, cs = (size_t)Cl.n * K;
  add_bytes((double)Cl.n * ((L.Wq + 1) * 4.0 + 2 * sizeof(CT<T>)) + (double)(fs + cs) * np * sizeof(T));
  const CT<T>* rw = pick<T>(L.rw64, L.rw32);
  if (pdl)
    launch_pdl(kern, g, dim3(TB), s, L.nc, L.Wq, (const int32_t*)L.rself.p, (const int32_t*)L.ridx.p, rw, r, bc,
               fs, cs);
  else
    kern<<<g, TB, 0, s>>>(L.nc, L.Wq, L.rself.p, L.ridx.p, rw, r, bc, fs, cs);
}

// x_f (+)= P z on all panels; assign when x_f is known to be zero (no clear, no read of x_f).
template <class T, int K>
static void launch_prolong(const Level& L, const Level& Cl, const T* z, T* x, bool assign, int np, cudaStream_t s,
                           bool pdl = true) {
  if (L.gen) {
    const dim3 g = row_grid<T, K>(L.n, np);
    const size_t fs = (size_t)L.n * K, cs = (size_t)Cl.n * K;
    add_bytes((double)L.n * L.Wp * (4.0 + sizeof(CT<T>)) + (double)(cs + (assign ? 1 : 2) * fs) * np * sizeof(T));
    const CT<T>* v = pick<T>(L.pval64, L.pval32);
    auto kern = assign ? k_transfer<T, K, false> : k_transfer<T, K, true>;
    if (pdl)
      launch_pdl(kern, g, dim3(TB), s, L.n, L.Wp, (const int32_t*)L.pcol.p, v, z, x, cs, fs);
    else
      kern<<<g, TB, 0, s>>>(L.n, L.Wp, L.pcol.p, v, z, x, cs, fs);
    return;
  }
  auto kern = assign ? k_prolong<T, K, true> : k_prolong<T, K, false>;
  const dim3 g = row_grid<T, K>(L.n, np);
  const size_t fs = (size_t)L.n * K, cs = (size_t)Cl.n * K;
  add_bytes((double)L.n * 8.0 + (double)(cs + (assign ? 1 : 2) * fs) * np * sizeof(T));
  if (pdl)
    launch_pdl(kern, g, dim3(TB), s, L.n, (const int32_t*)L.pa.p, (const int32_t*)L.pb.p, z, x, fs, cs);
  else
    kern<<<g, TB, 0, s>>>(L.n, L.pa.p, L.pb.p, z, x, fs, cs);
}

// Tuning key of the FP32 sweep's lanes per row (panel widths of 8 or more: vector width 4, the
// default, or 2, twice the lanes on a row), per panel width, row width and size bucket.
static std::string sweep_key(int K, int W, int n) {
  return "sweep/f32/K" + std::to_string(K) + "/W" + std::to_string(W) + "/n" + std::to_string(size_bucket(n));
}

// The tuned vector width override of level L's FP32 sweep at panel width K (0: the default),
// looked up once per change of the tuning table.
template <int K>
static int sweep_variant(const Level& L) {
  constexpr int k = K >= 32 ? 5 : K >= 16 ? 4 : 3;
  if (L.sweep_tuned_at[k] != tune_version()) {
    L.sweep_tuned_at[k] = tune_version();
    const int v = tune_get(sweep_key(K, L.W, L.n), 4);
    L.sweep_vv[k] = v == 2 ? 2 : 0;
  }
  return L.sweep_vv[k];
}

template <class T, int K, int VV>
static void launch_sweep_fp(const Level& L, const T* b, const T* x, T* out, SweepPrm<CT<T>> prm, int np,
                            cudaStream_t s, const CT<T>* cs, double* upd) {
  size_t ps = (size_t)L.n * K;
  const dim3 grid(grid_for((long long)L.n, Lanes<T, K, VV>::RPB, 8), np);
  const CT<T>* off = pick<T>(L.off64, L.off32);
  const CT<T>* dg = pick<T>(L.diag64, L.diag32);
  const CT<T>* di = pick<T>(L.dinv64, L.dinv32);
  if (upd) {  // u += (this sweep's result); out is not written
    auto go = [&](auto kern) {
      launch_pdl(kern, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs, upd);
    };
    if (cs) {
      if (L.W == 6) go(k_sweep_u<T, K, 6, true, VV>);
      else go(k_sweep_u<T, K, 0, true, VV>);
    } else if (L.W == 6) {
      go(k_sweep_u<T, K, 6, false, VV>);
    } else {
      go(k_sweep_u<T, K, 0, false, VV>);
    }
  } else {
    auto go = [&](auto kern) {
      launch_pdl(kern, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs);
    };
    if (cs) {
      if (L.W == 6) go(k_sweep<T, K, 6, true, VV>);
      else go(k_sweep<T, K, 0, true, VV>);
    } else if (L.W == 6) {
      go(k_sweep<T, K, 6, false, VV>);
    } else {
      go(k_sweep<T, K, 0, false, VV>);
    }
  }
}

template <class T, int K>
static void launch_sweep(const Level& L, const T* b, const T* x, T* out, SweepPrm<CT<T>> prm, int np,
                         cudaStream_t s, const CT<T>* cs, double* upd = nullptr) {
  size_t ps = (size_t)L.n * K;
  dim3 grid = row_grid<T, K>(L.n, np);
  {
    const double c = sizeof(CT<T>), v = (double)ps * np * sizeof(T);
    double by = v;                                                       // b
    if (!prm.zero_x) by += (double)L.n * (L.W * (4.0 + c) + c) + v;      // operator row, x
    if (prm.mode != S_RESID && !cs) by += (double)L.n * c;               // 1/diagonal
    if (prm.mode == S_CHEBN && !prm.d_is_x) by += v;                     // previous iterate
    by += upd ? 2.0 * (double)ps * np * sizeof(double) : v;              // out, or u read + written
    add_bytes(by);
  }
  if constexpr (std::is_same<T, __half>::value) {
    grid.x = std::min<unsigned>(grid.x, (unsigned)(kSweepHalfBlocks * num_sms()));
    const float* off = L.off32.p;
    const float* dg = L.diag32.p;
    const float* di = L.dinv32.p;
    if (cs) {
      if (L.W == 6) launch_pdl(k_sweep_h<K, 6, true>, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs);
      else launch_pdl(k_sweep_h<K, 0, true>, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs);
    } else if (L.W == 6) {
      launch_pdl(k_sweep_h<K, 6, false>, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs);
    } else {
      launch_pdl(k_sweep_h<K, 0, false>, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs);
    }
  } else {
    if constexpr (std::is_same<T, float>::value && K >= 8) {
      if (sweep_variant<K>(L) == 2) {
        launch_sweep_fp<T, K, 2>(L, b, x, out, prm, np, s, cs, upd);
        return;
      }
    }
    launch_sweep_fp<T, K, 0>(L, b, x, out, prm, np, s, cs, upd);
  }
}

// ---- sweeps fused with the prolongation ----------------------------------------------------------
// CTAs of a kernel instance resident per SM (queried once per instance; the tag types keep the
// instances' counters apart): the grid-stride grids stay within one wave.
template <class Tag, class F>
static int resident_ctas(F* kern) {
  static const int ctas = [kern] {
    int o = 0;
    DEC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, TB, 0));
    return std::min(8, std::max(1, o));
  }();
  return ctas;
}
template <class T, int K, bool SH, bool UPD, int PV, int VV>
struct SweepPTag {};
template <class T, int K, bool SH, bool ADD, int VV>
struct SweepApTag {};

// The second Chebyshev step after x (+)= P z with its previous iterate P z (PV 1) or out + P z (PV 2)
// formed from the coarse panels z of level Cl.
template <class T, int K, int PV, int VV>
static void launch_sweep_p_vv(const Level& L, const Level& Cl, const T* b, const T* x, T* out, SweepPrm<CT<T>> prm,
                              const T* z, int np, cudaStream_t s, const CT<T>* cs, double* upd) {
  const size_t ps = (size_t)L.n * K;
  const CT<T>* off = pick<T>(L.off64, L.off32);
  const CT<T>* dg = pick<T>(L.diag64, L.diag32);
  const CT<T>* di = pick<T>(L.dinv64, L.dinv32);
  const ProlongSrc<T> pz{L.pa.p, L.pb.p, z, (size_t)Cl.n * K};
  auto go = [&](auto kern, int per_sm) {
    const dim3 grid(grid_for((long long)L.n, Lanes<T, K, VV>::RPB, per_sm), np);
    launch_pdl(kern, grid, dim3(TB), s, L.n, L.W, L.col.p, off, dg, di, b, x, out, prm, ps, cs, upd, pz);
  };
#define DEC_GO(SHV, UPDV) \
  go(k_sweep_p<T, K, 6, SHV, UPDV, PV, VV>, \
     resident_ctas<SweepPTag<T, K, SHV, UPDV, PV, VV>>(k_sweep_p<T, K, 6, SHV, UPDV, PV, VV>))
  if (cs) {
    if (upd) DEC_GO(true, true);
    else DEC_GO(true, false);
  } else {
    if (upd) DEC_GO(false, true);
    else DEC_GO(false, false);
  }
#undef DEC_GO
}

template <class T, int K>
static void launch_sweep_p(const Level& L, const Level& Cl, const T* b, const T* x, T* out, SweepPrm<CT<T>> prm,
                           int pv, const T* z, int np, cudaStream_t s, const CT<T>* cs, double* upd) {
  {
    const size_t ps = (size_t)L.n * K;
    const double c = sizeof(CT<T>), v = (double)ps * np * sizeof(T), vc = (double)Cl.n * K * np * sizeof(T);
    double by = 2.0 * v + (double)L.n * (L.W * (4.0 + c) + c);        // b, x, operator row
    by += vc + (double)L.n * 8.0;                                      // coarse correction, parent indices
    if (!cs) by += (double)L.n * c;                                    // 1/diagonal
    if (pv >= 2) by += v;                                              // the iterate before the correction
    by += upd ? 2.0 * (double)ps * np * sizeof(double) : v;            // out, or u read + written
    add_bytes(by);
  }
  auto run = [&](auto vv) {
    constexpr int VV = decltype(vv)::value;
    if (pv == 1) launch_sweep_p_vv<T, K, 1, VV>(L, Cl, b, x, out, prm, z, np, s, cs, upd);
    else if (pv == 2) launch_sweep_p_vv<T, K, 2, VV>(L, Cl, b, x, out, prm, z, np, s, cs, upd);
    else launch_sweep_p_vv<T, K, 3, VV>(L, Cl, b, x, out, prm, z, np, s, cs, upd);
  };
  if constexpr (std::is_same<T, float>::value && K >= 8) {
    if (sweep_variant<K>(L) == 2) {
      run(std::integral_constant<int, 2>());
      return;
    }
  }
  run(std::integral_constant<int, 0>());
}

// The first Chebyshev step after the prolongation (k_sweep_ap): out = x0 + D⁻¹ (b - A x0) / θ with
// x0 = P z (add: e + P z, e in x) from the coarse panels z of level Cl and A P precomputed.
template <class T, int K>
static void launch_sweep_ap(const Level& L, const Level& Cl, const T* b, const T* x, T* out, double inv_theta,
                            bool add, const T* z, int np, cudaStream_t s, const CT<T>* cs) {
  const size_t ps = (size_t)L.n * K;
  {
    const double c = sizeof(CT<T>), v = (double)ps * np * sizeof(T), vc = (double)Cl.n * K * np * sizeof(T);
    double by = 2.0 * v + (double)L.n * kApW * (4.0 + c);              // b, out, A P rows
    by += vc;                                                          // the coarse correction
    by += cs ? (double)L.n * c : (double)L.n * c;                      // diagonal or 1/diagonal
    if (add) by += v + (double)L.n * L.W * (4.0 + c);                  // e, the operator's off-diagonals
    add_bytes(by);
  }
  const CT<T>* off = pick<T>(L.off64, L.off32);
  const CT<T>* dg = pick<T>(L.diag64, L.diag32);
  const CT<T>* di = pick<T>(L.dinv64, L.dinv32);
  const CT<T>* apv = pick<T>(L.apv64, L.apv32);
  const ProlongSrc<T> pz{L.pa.p, L.pb.p, z, (size_t)Cl.n * K};
  auto run = [&](auto vv) {
    constexpr int VV = decltype(vv)::value;
    auto go = [&](auto kern, int per_sm) {
      const dim3 grid(grid_for((long long)L.n, Lanes<T, K, VV>::RPB, per_sm), np);
      launch_pdl(kern, grid, dim3(TB), s, L.n, (const int32_t*)L.col.p, off, dg, di, (const int32_t*)L.apc.p, apv,
                 b, x, out, (CT<T>)inv_theta, ps, cs, pz);
    };
#define DEC_GO(SHV, ADDV) \
  go(k_sweep_ap<T, K, SHV, ADDV, VV>, resident_ctas<SweepApTag<T, K, SHV, ADDV, VV>>(k_sweep_ap<T, K, SHV, ADDV, VV>))
    if (cs) {
      if (add) DEC_GO(true, true);
      else DEC_GO(true, false);
    } else {
      if (add) DEC_GO(false, true);
      else DEC_GO(false, false);
    }
#undef DEC_GO
  };
  if constexpr (std::is_same<T, float>::value && K >= 8) {
    if (sweep_variant<K>(L) == 2) {
      run(std::integral_constant<int, 2>());
      return;
    }
  }
  run(std::integral_constant<int, 0>());
}

// ---- the two-step Chebyshev pair ----------------------------------------------------------------
// Tuning key: P > 0 = the post-smoothing pair of this level runs as k_cheb2 over patches of P rows
// (128, 256 or 512), 0 (default) = two sweeps.
static std::string cheb2_key(int K, int W, int n) {
  return "cheb2/f32/K" + std::to_string(K) + "/W" + std::to_string(W) + "/n" + std::to_string(size_bucket(n));
}
constexpr int kCheb2MinRows = 1 << 14;  // smaller levels stay with the sweeps (launch-bound)

// The patches of P rows and their halos of level L (host, from the internal operator columns).
static void build_two_step(Level& L, int P) {
  require(P >= 32 && P <= kTwoStepRows, "multigrid: two-step patches of 32 to 512 rows");
  const int n = L.n, W = L.W;
  const std::vector<int32_t> col = L.col.download();
  const int npatch = (n + P - 1) / P;
  std::vector<int32_t> hptr(npatch + 1, 0), h1n(npatch, 0), lptr(npatch + 1, 0), halo, loc(n, 0), stamp(n, -1);
  std::vector<uint16_t> lcol;
  halo.reserve((size_t)n);
  lcol.reserve((size_t)n * W * 5 / 4);
  int max_local = 0, max_l1 = 0;
  double sum_local = 0, sum_l1 = 0;
  for (int p = 0; p < npatch; ++p) {
    const int a = p * P, e = std::min(n, a + P), pr = e - a;
    auto local = [&](int g) { return stamp[g] == p ? loc[g] : -1; };
    auto add = [&](int g, int id) {
      stamp[g] = p;
      loc[g] = id;
    };
    for (int r = a; r < e; ++r) add(r, r - a);
    int next = pr;
    hptr[p] = (int)halo.size();
    for (int r = a; r < e; ++r)
      for (int k = 0; k < W; ++k) {
        const int c = col[(size_t)r * W + k];
        if (local(c) < 0) {
          add(c, next++);
          halo.push_back(c);
        }
      }
    const int n1 = next - pr;
    h1n[p] = n1;
    for (int h = hptr[p]; h < hptr[p] + n1; ++h)
      for (int k = 0; k < W; ++k) {
        const int c = col[(size_t)halo[h] * W + k];
        if (local(c) < 0) {
          add(c, next++);
          halo.push_back(c);
        }
      }
    hptr[p + 1] = (int)halo.size();
    require(next <= 65535, "multigrid: a two-step patch's halo exceeds 16-bit local indices");
    lptr[p] = (int)(lcol.size() / W);
    for (int lr = 0; lr < pr + n1; ++lr) {
      const int g = lr < pr ? a + lr : halo[hptr[p] + lr - pr];
      for (int k = 0; k < W; ++k) lcol.push_back((uint16_t)local(col[(size_t)g * W + k]));
    }
    lptr[p + 1] = (int)(lcol.size() / W);
    max_local = std::max(max_local, next);
    max_l1 = std::max(max_l1, pr + n1);
    sum_local += next;
    sum_l1 += pr + n1;
  }
  // every local column of a patch row or H1 row lies inside its patch's local rows (patch, H1, H2)
  for (int p = 0; p < npatch; ++p) {
    const int pr = std::min(n, (p + 1) * P) - p * P, nloc = pr + hptr[p + 1] - hptr[p];
    for (size_t q = (size_t)lptr[p] * W; q < (size_t)lptr[p + 1] * W; ++q)
      require(lcol[q] < nloc, "multigrid: a two-step patch's local column falls outside its rows");
    require(lptr[p + 1] - lptr[p] == pr + h1n[p], "multigrid: two-step local rows do not match the patch");
  }
  L.ts.P = P;
  L.ts.npatch = npatch;
  L.ts.max_local = max_local;
  L.ts.max_l1 = max_l1;
  L.ts.sum_local = sum_local;
  L.ts.sum_l1 = sum_l1;
  L.ts.hptr.upload(hptr);
  L.ts.h1n.upload(h1n);
  L.ts.lptr.upload(lptr);
  L.ts.halo.upload(halo.empty() ? std::vector<int32_t>(1, 0) : halo);
  L.ts.lcol.upload(lcol);
}

// The dynamic shared memory above 48 KB that k_cheb2 needs, for both of its instances at panel widths
// 16 and 32, once per device (a host call that must not run inside a stream capture).
static void cheb2_opt_in() {
  static std::mutex mu;
  static uint64_t done = 0;  // bit per device ordinal
  int dev = 0;
  DEC_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < 64, "multigrid: device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (done & (1ull << dev)) return;
  constexpr int kMax = 200 * 1024;
  DEC_CUDA(cudaFuncSetAttribute(k_cheb2<16, 16, 6, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax));
  DEC_CUDA(cudaFuncSetAttribute(k_cheb2<16, 16, 6, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax));
  DEC_CUDA(cudaFuncSetAttribute(k_cheb2<32, 16, 6, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax));
  DEC_CUDA(cudaFuncSetAttribute(k_cheb2<32, 16, 6, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax));
  done |= 1ull << dev;
}

template <int K>
static size_t cheb2_smem(const Level& L) {
  constexpr int KS = K >= 16 ? 16 : K;
  return (size_t)(L.ts.max_local + L.ts.max_l1) * KS * sizeof(float);
}

// Can level L's post-smoothing pair of panel width K run as k_cheb2 (FP32, rows of 6 off-diagonal
// slots, no per-RHS shifts, built patches that fit the shared memory), and does the table ask for it?
template <class T, int K>
static bool cheb2_on(const Level& L, const CT<T>* cs) {
  if constexpr (!std::is_same<T, float>::value || K < 16) {
    return false;
  } else {
    if (cs || L.W != 6 || L.n < kCheb2MinRows || !L.ts.npatch) return false;
    if (cheb2_smem<K>(L) > 200 * 1024) return false;
    return tune_get(cheb2_key(K, L.W, L.n), 0) == L.ts.P;
  }
}

template <class T, int K>
static void launch_cheb2(const Level& L, const T* b, const T* x, T* out, double inv_theta, double c1, double c2,
                         int np, cudaStream_t s, double* upd) {
  if constexpr (std::is_same<T, float>::value && K >= 16) {
    constexpr int KS = 16;
    const size_t smem = cheb2_smem<K>(L);
    const size_t ps = (size_t)L.n * K;
    {
      const double v = KS * 4.0, opr = L.W * (2.0 + 4.0) + 8.0;  // local columns, values, diag, 1/diag
      const double per_slice = L.ts.sum_local * v + L.ts.sum_l1 * (v + opr) + (double)L.n * (v + opr) +
                               (double)L.n * (upd ? 2.0 * KS * 8.0 : v);
      add_bytes((double)(K / KS) * np * per_slice + (double)L.ts.sum_local * 4.0);
    }
    auto go = [&](auto kern) {  // both instances were opted in before the capture (cheb2_opt_in)
      launch_pdl_smem(kern, dim3(L.ts.npatch, K / KS, np), dim3(TB), smem, s, L.n, L.ts.P, L.ts.max_local,
                      (const int32_t*)L.ts.hptr.p, (const int32_t*)L.ts.h1n.p, (const int32_t*)L.ts.halo.p,
                      (const int32_t*)L.ts.lptr.p, (const uint16_t*)L.ts.lcol.p, (const float*)L.off32.p,
                      (const float*)L.diag32.p, (const float*)L.dinv32.p, b, x, out, (float)inv_theta, (float)c1,
                      (float)c2, ps, upd);
    };
    if (upd) go(k_cheb2<K, KS, 6, true>);
    else go(k_cheb2<K, KS, 6, false>);
  }
}

// Smooth `sweeps` times starting from x (zero if zero_x); returns the buffer holding the result.
template <class T, int K>
static T* smooth(const dec_mg& mg, const Level& L, LevelBufs<T>& B, T* x, bool zero_x, int sweeps, int np,
                 cudaStream_t s, double* upd = nullptr) {
  const dec_mg_options& o = mg.opt;
  T* other = (x == B.x.p) ? B.y.p : B.x.p;
  if constexpr (!std::is_same<T, __half>::value) {
  if (o.smoother == DEC_SMOOTH_LEARNED && !mg.force_plain) {
    // learned sweep: r = b - A x (skipped from zero: r = b), then x + (s / a_ii) MLP(features(r))
    const MlpWeights wts = mlp_weights(mg.mlp);
    for (int it = 0; it < sweeps; ++it) {
      const T* r = B.b.p;
      if (!zero_x) {
        SweepPrm<CT<T>> prm{};
        prm.mode = S_RESID;
        launch_sweep<T, K>(L, B.b.p, x, B.d.p, prm, np, s, B.cs);
        r = B.d.p;
      }
      add_bytes((double)L.n * (L.W * 4.0 + 32.0 + sizeof(CT<T>)) +
                (double)L.n * K * np * sizeof(T) * (zero_x ? 2.0 : 3.0));  // indices, couplings, diag; r, x, out
      launch_mlp_smooth<T, K>(wts, L.n, L.W, L.col.p, L.mtab.p, pick<T>(L.diag64, L.diag32), r, x, zero_x ? 1 : 0,
                              other, np, s);
      std::swap(x, other);
      zero_x = false;
    }
    return x;
  }
  }
  using C = CT<T>;
  const double hi = L.lmax, lo = L.lmax / o.cheb_ratio;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2, sigma = theta / delta;
  double rho = 1 / sigma;
  const bool started_at_zero = zero_x;
  if (o.smoother == DEC_SMOOTH_CHEBYSHEV && sweeps == 2 && !zero_x && cheb2_on<T, K>(L, B.cs)) {
    // the two steps in one pass: the coefficients of the loop below for it = 0 and it = 1
    const double rho_new = 1 / (2 * sigma - rho);
    launch_cheb2<T, K>(L, B.b.p, x, other, 1.0 / theta, rho_new * rho, 2 * rho_new / delta, np, s, upd);
    return other;
  }
  for (int it = 0; it < sweeps; ++it) {
    SweepPrm<C> prm{};
    prm.zero_x = zero_x ? 1 : 0;
    // step k reads x_{k-2} from the buffer it writes (x and other alternate); after a first step
    // from zero that iterate is zero and the buffer holds nothing
    prm.d_is_x = (it == 1 && started_at_zero) ? 1 : 0;
    if (o.smoother == DEC_SMOOTH_JACOBI) {
      prm.mode = S_JACOBI;
      prm.omega = (C)o.omega;
    } else if (it == 0) {
      prm.mode = S_CHEB0;
      prm.inv_theta = (C)(1.0 / theta);
    } else {
      double rho_new = 1 / (2 * sigma - rho);
      prm.mode = S_CHEBN;
      prm.c1 = (C)(rho_new * rho);
      prm.c2 = (C)(2 * rho_new / delta);
      rho = rho_new;
    }
    launch_sweep<T, K>(L, B.b.p, x, other, prm, np, s, B.cs, it + 1 == sweeps ? upd : nullptr);
    std::swap(x, other);
    zero_x = false;
  }
  return x;
}


// The prolongation x (+)= P z fused into the two Chebyshev steps that follow it (tuning key "pfuse":
// 1 where the level's iterate was zero (x0 = P z); 2 also onto an iterate e (x0 = e + P z); 3, the
// default, 1 and onto an iterate in correction form (two post-smoothing steps: the steps smooth δ on
// A δ = r, r = b - A e the residual the cycle restricted, from δ0 = P z, and the second stores e + δ);
// 0 never): the first step forms A x0 from the coarse panels through A P (k_sweep_ap), the second its
// previous iterate from them (k_sweep_p), so x0 is never stored.  FP32 / FP64 panels,
// binary-subdivision transfers, rows of 6 off-diagonal slots, two or more post-smoothing steps; a
// level whose post-smoothing pair runs as k_cheb2 keeps the stored prolongation.
constexpr int kPfuseDefault = 3;
template <class T, int K>
static bool prolong_fused(const dec_mg& mg, const Level& L, const CT<T>* cs, int sweeps, bool assign) {
  if constexpr (std::is_same<T, __half>::value) {
    return false;
  } else {
    if (mg.opt.smoother != DEC_SMOOTH_CHEBYSHEV || sweeps < 2 || !L.ap_ok) return false;
    if (sweeps == 2 && cheb2_on<T, K>(L, cs)) return false;
    const int mode = tune_get("pfuse", kPfuseDefault);
    return assign ? mode != 0 : (mode == 2 || (mode == 3 && sweeps == 2));
  }
}

// smooth() from x0 = P z (assign) or x + P z, the prolongation fused into the first two steps;
// returns the buffer holding the result, as smooth() after launch_prolong would.
template <class T, int K>
static T* smooth_prolonged(const dec_mg& mg, const Level& L, const Level& Cl, LevelBufs<T>& B, T* x, const T* z,
                           bool assign, int sweeps, int np, cudaStream_t s, double* upd) {
  const dec_mg_options& o = mg.opt;
  using C = CT<T>;
  T* other = (x == B.x.p) ? B.y.p : B.x.p;
  const double hi = L.lmax, lo = L.lmax / o.cheb_ratio;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2, sigma = theta / delta;
  double rho = 1 / sigma;
  // step 1: x (the iterate before the correction, unread when assign) -> other
  launch_sweep_ap<T, K>(L, Cl, B.b.p, x, other, 1.0 / theta, !assign, z, np, s, B.cs);
  std::swap(x, other);
  for (int it = 1; it < sweeps; ++it) {
    SweepPrm<C> prm{};
    const double rho_new = 1 / (2 * sigma - rho);
    prm.mode = S_CHEBN;
    prm.c1 = (C)(rho_new * rho);
    prm.c2 = (C)(2 * rho_new / delta);
    rho = rho_new;
    double* u = it + 1 == sweeps ? upd : nullptr;
    if (it == 1)  // previous iterate x0: P z, or (out, still the iterate before the correction) + P z
      launch_sweep_p<T, K>(L, Cl, B.b.p, x, other, prm, assign ? 1 : 2, z, np, s, B.cs, u);
    else
      launch_sweep<T, K>(L, B.b.p, x, other, prm, np, s, B.cs, u);
    std::swap(x, other);
  }
  return x;
}

// Two post-smoothing Chebyshev steps from e + P z in correction form: δ1 from δ0 = P z on A δ = r
// (k_sweep_ap into B.d), then δ2 and the stored e + δ2 (k_sweep_p, PV 3, into e's buffer x or added to
// the FP64 iterate with upd).  r: the residual b - A e the cycle restricted.  Returns x.
template <class T, int K>
static T* smooth_correction(const dec_mg& mg, const Level& L, const Level& Cl, LevelBufs<T>& B, T* x, const T* r,
                            const T* z, int np, cudaStream_t s, double* upd) {
  const dec_mg_options& o = mg.opt;
  using C = CT<T>;
  const double hi = L.lmax, lo = L.lmax / o.cheb_ratio;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2, sigma = theta / delta;
  const double rho = 1 / sigma, rho_new = 1 / (2 * sigma - rho);
  launch_sweep_ap<T, K>(L, Cl, r, nullptr, B.d.p, 1.0 / theta, false, z, np, s, B.cs);
  SweepPrm<C> prm{};
  prm.mode = S_CHEBN;
  prm.c1 = (C)(rho_new * rho);
  prm.c2 = (C)(2 * rho_new / delta);
  launch_sweep_p<T, K>(L, Cl, r, B.d.p, x, prm, 3, z, np, s, B.cs, upd);
  return x;
}

// steps iterations of the Krylov CG smoother on level L from x (zero if zero_x); returns the
// buffer holding x.  FP64 only.
template <int K>
static double* cg_smooth(const dec_mg& mg, Workspace& w, const Level& L, LevelBufs<double>& B, double* x, bool zero_x,
                         int steps, int np, cudaStream_t s) {
  if (steps == 0) return x;  // steps == 0 skips the smoother (Multigrid.jl:860, issue #178)
  const int ntot = K * np;
  const size_t ps = (size_t)L.n * K;
  dim3 g(grid_for(L.n, TB / K, 8), np);
  const int nb = (int)g.x;
  double* r = (x == B.x.p) ? B.y.p : B.x.p;  // r in the free ping-pong buffer
  double* pp = B.d.p;
  if (L.W == 6)
    k_cg_init<K, 6><<<g, TB, 0, s>>>(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, B.b.p, x, zero_x ? 1 : 0, r, pp,
                                     B.e.p, w.partial.p, ps);
  else
    k_cg_init<K, 0><<<g, TB, 0, s>>>(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, B.b.p, x, zero_x ? 1 : 0, r, pp,
                                     B.e.p, w.partial.p, ps);
  k_cg_scalar<<<ntot, 256, 0, s>>>(CG_PH_INIT, nb, K, ntot, steps, w.partial.p, w.scal.p);
  for (int it = 0; it < steps; ++it) {
    if (L.W == 6)
      k_cg_spmv<K, 6><<<g, TB, 0, s>>>(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, pp, B.q.p, w.scal.p, ntot,
                                       w.partial.p, ps);
    else
      k_cg_spmv<K, 0><<<g, TB, 0, s>>>(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, pp, B.q.p, w.scal.p, ntot,
                                       w.partial.p, ps);
    k_cg_scalar<<<ntot, 256, 0, s>>>(CG_PH_ALPHA, nb, K, ntot, steps, w.partial.p, w.scal.p);
    k_cg_axpy<K><<<g, TB, 0, s>>>(L.n, pp, B.q.p, B.e.p, r, w.scal.p, ntot, w.partial.p, ps);
    k_cg_scalar<<<ntot, 256, 0, s>>>(CG_PH_BETA, nb, K, ntot, steps, w.partial.p, w.scal.p);
    if (it + 1 < steps) k_cg_pupd<K><<<g, TB, 0, s>>>(L.n, r, pp, w.scal.p, ntot, ps);
  }
  // x + Δx goes into the residual buffer (free again), which becomes the result
  k_cg_finish<K><<<g, TB, 0, s>>>(L.n, x, zero_x ? 1 : 0, B.e.p, r, ps);
  DEC_CHECK_LAUNCH();
  return r;
}


template <class T, int K>
static T* mu_cycle(const dec_mg& mg, Workspace& w, std::vector<LevelBufs<T>>& bufs, int l, T* x, bool zero_x, int mu,
                   int np, cudaStream_t s, double* upd = nullptr);

// _multigrid_μ_cycle, Multigrid.jl:857-872, with the Krylov CG smoother: CG (steps) ; if the
// coarsest level, return ; r = b - A u ; restrict ; recurse (twice for μ = 2) ; u += P z ; CG.
template <int K>
static double* cg_mu_cycle(const dec_mg& mg, Workspace& w, std::vector<LevelBufs<double>>& bufs, int l, double* x,
                           bool zero_x, int mu, int np, cudaStream_t s) {
  const Level& L = mg.lv[l];
  LevelBufs<double>& B = bufs[l];
  const int last = (int)mg.lv.size() - 1;
  const int steps_pre = mg.pre_at(l), steps_post = mg.post_at(l);
  x = cg_smooth<K>(mg, w, L, B, x, zero_x, steps_pre, np, s);
  if (steps_pre > 0) zero_x = false;
  if (l >= last) {
    if (zero_x) DEC_CUDA(cudaMemsetAsync(x, 0, (size_t)L.n * K * np * sizeof(double), s));
    return x;
  }
  // with x = 0 the residual is b itself (the residual sweep would copy it bit for bit)
  const double* r = B.b.p;
  if (!zero_x) {
    double* rr = (x == B.x.p) ? B.y.p : B.x.p;
    SweepPrm<double> prm{};
    prm.mode = S_RESID;
    launch_sweep<double, K>(L, B.b.p, x, rr, prm, np, s, B.cs);
    r = rr;
  }
  const Level& Cl = mg.lv[l + 1];
  LevelBufs<double>& Cb = bufs[l + 1];
  launch_restrict<double, K>(L, Cl, r, Cb.b.p, np, s);
  double* z = cg_mu_cycle<K>(mg, w, bufs, l + 1, Cb.x.p, true, mu, np, s);
  if (mu > 1) z = cg_mu_cycle<K>(mg, w, bufs, l + 1, z, false, mu - 1, np, s);
  launch_prolong<double, K>(L, Cl, (const double*)z, x, zero_x, np, s);
  return cg_smooth<K>(mg, w, L, B, x, false, steps_post, np, s);
}

// One μ-cycle at level l on (b = B[l].b, initial guess x); returns the buffer with the result.
// upd (finest level, Jacobi / Chebyshev post-smoothing, not FP16): the last sweep adds its result
// to the FP64 iterate (k_sweep_u) and the returned buffer holds nothing.
template <class T, int K>
static T* mu_cycle(const dec_mg& mg, Workspace& w, std::vector<LevelBufs<T>>& bufs, int l, T* x, bool zero_x, int mu,
                   int np, cudaStream_t s, double* upd) {
  const Level& L = mg.lv[l];
  LevelBufs<T>& B = bufs[l];
  if constexpr (std::is_same<T, double>::value) {
    if (mg.opt.smoother == DEC_SMOOTH_CG) return cg_mu_cycle<K>(mg, w, bufs, l, x, zero_x, mu, np, s);
  }
  if (l == mg.lc) {
    if (mg.opt.coarse_solver == 1)  // the smoother on the coarsest level (pre + post sweeps)
      return smooth<T, K>(mg, L, B, x, zero_x, std::max(1, mg.pre_at(l) + mg.post_at(l)), np, s);
    if (mg.opt.coarse_solver == 2) {  // per-RHS shifted solve through the eigendecomposition
      const dim3 g(grid_for(L.n, TB / K, 64), np);
      add_bytes(2.0 * (double)L.n * L.n * 8.0 + (double)L.n * K * np * (2.0 * sizeof(T) + 16.0));
      launch_pdl(k_coarse_eig1<T, K>, g, dim3(TB), s, L.n, (const double*)mg.eigF.p, (const double*)mg.eigL.p,
                 (const double*)w.cs64.p, (const T*)B.b.p, w.ceig.p, (size_t)L.n * K);
      launch_pdl(k_coarse_eig2<T, K>, g, dim3(TB), s, L.n, (const double*)mg.eigE.p, (const double*)w.ceig.p, B.x.p,
                 (size_t)L.n * K);
      return B.x.p;
    }
    add_bytes((double)L.n * L.n * 8.0 + 2.0 * (double)L.n * K * np * sizeof(T));
    launch_pdl(k_coarse<T, K>, dim3(grid_for(L.n, 1, 8), np), dim3(TB), s, L.n, (const double*)mg.ainv.p,
               (const T*)B.b.p, B.x.p, (size_t)L.n * K);
    return B.x.p;
  }
  x = smooth<T, K>(mg, L, B, x, zero_x, mg.pre_at(l), np, s);
  zero_x = zero_x && mg.pre_at(l) == 0;
  // residual into the free buffer, then restrict into the coarse right-hand side; with x = 0
  // (every coarse level, and the finest one on a refinement step's first cycle) the residual is
  // b itself, which the residual sweep would only copy (bit for bit)
  const T* r = B.b.p;
  if (!zero_x) {
    T* rr = (x == B.x.p) ? B.y.p : B.x.p;
    SweepPrm<CT<T>> prm{};
    prm.mode = S_RESID;
    launch_sweep<T, K>(L, B.b.p, x, rr, prm, np, s, B.cs);
    r = rr;
  }
  const Level& Cl = mg.lv[l + 1];
  LevelBufs<T>& Cb = bufs[l + 1];
  launch_restrict<T, K>(L, Cl, r, Cb.b.p, np, s);
  T* z = mu_cycle<T, K>(mg, w, bufs, l + 1, Cb.x.p, true, mu, np, s);
  if (mu > 1) z = mu_cycle<T, K>(mg, w, bufs, l + 1, z, false, mu - 1, np, s);
  if constexpr (!std::is_same<T, __half>::value) {
    if (prolong_fused<T, K>(mg, L, B.cs, mg.post_at(l), zero_x)) {
      if (!zero_x && tune_get("pfuse", kPfuseDefault) == 3)  // r: the restricted residual b - A x
        return smooth_correction<T, K>(mg, L, Cl, B, x, r, z, np, s, upd);
      return smooth_prolonged<T, K>(mg, L, Cl, B, x, z, zero_x, mg.post_at(l), np, s, upd);
    }
  }
  // x = 0: the prolonged correction is x (written, not added)
  launch_prolong<T, K>(L, Cl, (const T*)z, x, zero_x, np, s);
  return smooth<T, K>(mg, L, B, x, false, mg.post_at(l), np, s, upd);
}

template <class T>
static void alloc_bufs(const dec_mg& mg, std::vector<LevelBufs<T>>& bufs, int K, int np) {
  bufs.resize(mg.lv.size());
  for (size_t l = 0; l < mg.lv.size(); ++l) {
    size_t n = (size_t)mg.lv[l].n * K * np;
    bufs[l].x.alloc(n);
    bufs[l].y.alloc(n);
    bufs[l].b.alloc(n);
    bufs[l].d.alloc(n);
    for (DArr<T>* a : {&bufs[l].x, &bufs[l].y, &bufs[l].b, &bufs[l].d})
      DEC_CUDA(cudaMemset(a->p, 0, a->bytes()));
    if (mg.opt.smoother == DEC_SMOOTH_CG) {
      bufs[l].q.alloc(n);
      bufs[l].e.alloc(n);
      DEC_CUDA(cudaMemset(bufs[l].q.p, 0, bufs[l].q.bytes()));
      DEC_CUDA(cudaMemset(bufs[l].e.p, 0, bufs[l].e.bytes()));
    }
  }
}

static long long ws_key(int K, int np, int prec) { return ((long long)K << 40) | ((long long)np << 8) | prec; }

static int choose_k(const dec_mg& mg, int nrhs, int prec) {
  int K = mg.opt.rhs_block;
  if (K <= 0) {
    auto it = mg.tuned.find(((long long)nrhs << 2) | prec);
    if (it != mg.tuned.end()) return it->second;
    K = 1;
    while (K < nrhs && K < 32) K <<= 1;
  }
  require(K == 1 || K == 2 || K == 4 || K == 8 || K == 16 || K == 32, "multigrid: rhs_block must be 1..32, a power of two");
  return K;
}

// Refinement step, part 1: u += e; r = b - A u in FP64 (r stored in the inner precision as the
// finest right-hand side) with per-RHS squared norms.
template <class T, int K>
static void enqueue_resid_T(dec_mg& mg, Workspace& w, cudaStream_t s, std::vector<LevelBufs<T>>& bufs,
                            bool updated = false) {
  const Level& F = mg.lv[0];
  const int np = w.npanels;
  const size_t total = (size_t)F.n * K * np;
  constexpr bool H = std::is_same<T, __half>::value;
  using R = typename std::conditional<H, float, T>::type;  // the residual kernel's output type
  R* rout;
  if constexpr (H) {
    add_bytes((double)total * (sizeof(__half) + 16.0));
    launch_pdl(k_axpy_scaled<K>, dim3(grid_for((long long)total, 256)), dim3(256), s, total, (size_t)F.n * K,
               (const __half*)bufs[0].x.p, (const double*)w.escale.p, w.U64.p);
    rout = w.r32.p;
  } else {
    if (!updated) {  // else the V-cycles' last sweep added e to u already
      add_bytes((double)total * (sizeof(T) + 16.0));
      launch_pdl(k_axpy_update<T>, dim3(grid_for((long long)total, 256)), dim3(256), s, total,
                 (const T*)bufs[0].x.p, w.U64.p);
    }
    rout = bufs[0].b.p;
  }
  dim3 g(w.nblocks, np);
  const double* cs = w.cs64.p;
  add_bytes((double)F.n * (F.W * 12.0 + 8.0) + (double)total * (16.0 + sizeof(R)));  // A (FP64), b, u; r out
  auto go = [&](auto kern) {
    launch_pdl(kern, g, dim3(TB), s, F.n, F.W, (const int32_t*)F.col.p, (const double*)F.off64.p,
               (const double*)F.diag64.p, (const double*)w.B64.p, (const double*)w.U64.p, rout, w.partial.p,
               (size_t)F.n * K, cs);
  };
  if (cs) {
    if (F.W == 6) go(k_residual64<R, K, 6, true>);
    else go(k_residual64<R, K, 0, true>);
  } else if (F.W == 6) {
    go(k_residual64<R, K, 6, false>);
  } else {
    go(k_residual64<R, K, 0, false>);
  }
  launch_pdl(k_reduce_partials, dim3(K * np), dim3(256), s, w.nblocks, K, np, (const double*)w.partial.p,
             w.norms.p);
  if constexpr (H) add_bytes((double)total * (4.0 + sizeof(__half)));
  if constexpr (H)
    launch_pdl(k_scale_half<K>, dim3(grid_for((long long)total, 256)), dim3(256), s, F.n, np, (const float*)w.r32.p,
               (const double*)w.norms.p, (__half*)bufs[0].b.p, w.escale.p);
  DEC_CHECK_LAUNCH();
}

// Refinement step, part 2: e = V^c(r) (c = inner_cycles) from a zero initial guess, left in
// bufs[0].x.
// upd: the last cycle's last sweep adds e to the FP64 iterate (fused_update) and e is not kept.
template <class T, int K>
static void enqueue_vcycle_T(dec_mg& mg, Workspace& w, cudaStream_t s, std::vector<LevelBufs<T>>& bufs,
                             double* upd = nullptr) {
  const size_t total = (size_t)mg.lv[0].n * K * w.npanels;
  const int c_last = mg.opt.inner_cycles - 1;
  T* e = bufs[0].x.p;
  for (int c = 0; c <= c_last; ++c)
    e = mu_cycle<T, K>(mg, w, bufs, 0, e, c == 0, mg.opt.mu, w.npanels, s, c == c_last ? upd : nullptr);
  if (!upd && e != bufs[0].x.p) {
    add_bytes(2.0 * (double)total * sizeof(T));
    DEC_CUDA(cudaMemcpyAsync(bufs[0].x.p, e, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
  }
  DEC_CHECK_LAUNCH();
}

// One plain FP64 cycle in place on (U64, B64): U <- V(U, B).
template <int K>
static void enqueue_cycle(dec_mg& mg, Workspace& w, cudaStream_t s) {
  auto& bufs = w.f64;
  const size_t total = (size_t)mg.lv[0].n * K * w.npanels;
  DEC_CUDA(cudaMemcpyAsync(bufs[0].b.p, w.B64.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DEC_CUDA(cudaMemcpyAsync(bufs[0].x.p, w.U64.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double* x = mu_cycle<double, K>(mg, w, bufs, 0, bufs[0].x.p, false, mg.opt.mu, w.npanels, s);
  DEC_CUDA(cudaMemcpyAsync(w.U64.p, x, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DEC_CHECK_LAUNCH();
}

// Vectors a smoothing sweep reads or writes once: Jacobi b, x, out; Chebyshev b, x, d (r/w), out.
// vectors a timed sweep moves: b, x, out (+ the previous iterate in out for a Chebyshev step)
static int prm_vectors(int smoother) { return smoother == DEC_SMOOTH_JACOBI ? 3 : 4; }

// plain: learned-smoother fallback; G_STEP: V-cycles with the update fused into the last sweep,
// then the residual (the refinement loops' step when fused_update holds)
enum GraphKind { G_RESID = 0, G_VCYCLE = 1, G_CYCLE = 2, G_VCYCLE_PLAIN = 3, G_STEP = 4 };

// The last finest-level sweep can take the refinement update (k_sweep_u): Jacobi / Chebyshev
// post-smoothing on a finest level that is not the directly solved one, FP32 / FP64 storage.
static bool fused_update(const dec_mg& mg, const Workspace& w) {
  const int s = mg.opt.smoother;
  return (s == DEC_SMOOTH_JACOBI || s == DEC_SMOOTH_CHEBYSHEV) && mg.post_at(0) > 0 && mg.lc > 0 && w.prec != 2;
}

template <int K>
static void enqueue_kind(dec_mg& mg, Workspace& w, cudaStream_t s, int kind) {
  if (kind == G_CYCLE) {
    enqueue_cycle<K>(mg, w, s);
  } else if (w.prec == 2) {
    if (kind == G_RESID) enqueue_resid_T<__half, K>(mg, w, s, w.f16);
    else enqueue_vcycle_T<__half, K>(mg, w, s, w.f16);
  } else if (w.prec == 1) {
    if (kind == G_STEP) {
      enqueue_vcycle_T<float, K>(mg, w, s, w.f32, w.U64.p);
      enqueue_resid_T<float, K>(mg, w, s, w.f32, true);
    } else if (kind == G_RESID) {
      enqueue_resid_T<float, K>(mg, w, s, w.f32);
    } else {
      enqueue_vcycle_T<float, K>(mg, w, s, w.f32);
    }
  } else {
    if (kind == G_STEP) {
      enqueue_vcycle_T<double, K>(mg, w, s, w.f64, w.U64.p);
      enqueue_resid_T<double, K>(mg, w, s, w.f64, true);
    } else if (kind == G_RESID) {
      enqueue_resid_T<double, K>(mg, w, s, w.f64);
    } else {
      enqueue_vcycle_T<double, K>(mg, w, s, w.f64);
    }
  }
}

static void dispatch(dec_mg& mg, Workspace& w, cudaStream_t s, int kind) {
  switch (w.K) {
#define DEC_K(KK) \
  case KK: enqueue_kind<KK>(mg, w, s, kind); break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
    default: throw Error(DEC_ERR_INVALID_ARG, "multigrid: bad panel width");
  }
}

static int64_t count_kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  DEC_CUDA(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) DEC_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
  int64_t k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) {
      // the CUDA 12.9 runtime on a CUDA 13 driver does not name a conditional node's type; the
      // error is not sticky and the node is not a kernel
      (void)cudaGetLastError();
      continue;
    }
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

// Builds the two-step patches of every level whose table entry asks for the pair at panel width K
// (host work and uploads: before a capture starts).
static void ensure_two_step(dec_mg& mg, int K) {
  if (mg.opt.smoother != DEC_SMOOTH_CHEBYSHEV || mg.opt.precision != 1 || K < 16) return;
  for (Level& L : mg.lv)
    if (L.W == 6 && L.n >= kCheb2MinRows) {
      const int P = tune_get(cheb2_key(K, L.W, L.n), 0);
      if (P <= 0) continue;
      cheb2_opt_in();
      if (!L.ts.npatch || L.ts.P != P) build_two_step(L, P);
    }
}

static cudaGraphExec_t capture(dec_mg& mg, Workspace& w, int kind) {
  ensure_two_step(mg, w.K);
  cudaGraph_t g = nullptr;
  require(mg.opt.smoother != DEC_SMOOTH_LEARNED || mg.mlp != nullptr || kind == G_VCYCLE_PLAIN || kind == G_RESID,
          "multigrid: the learned smoother needs a network (dec_mg_set_smoother_mlp)");
  DEC_CUDA(cudaStreamBeginCapture(mg.cap, cudaStreamCaptureModeThreadLocal));
  mg.force_plain = kind == G_VCYCLE_PLAIN;
  try {
    dispatch(mg, w, mg.cap, kind);
  } catch (...) {
    mg.force_plain = false;
    cudaStreamEndCapture(mg.cap, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  mg.force_plain = false;
  DEC_CUDA(cudaStreamEndCapture(mg.cap, &g));
  w.launches[kind] = count_kernel_nodes(g);
  cudaGraphExec_t ex = nullptr;
  cudaError_t err = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  DEC_CUDA(err);
  return ex;
}

// Waits for the pipelined host-buffer solves still running on the hierarchy's workspaces.
static void drain_pipeline(dec_mg& mg) {
  for (cudaStream_t p : mg.pipe)
    if (p) DEC_CUDA(cudaStreamSynchronize(p));
}

static Workspace& workspace_k(dec_mg& mg, int nrhs, int prec, int K, bool drain = true) {
  if (drain) drain_pipeline(mg);
  if (mg.mlp && (mg.mlp->engine != mg.mlp_engine || mg.mlp->version != mg.mlp_version)) {
    // captured cycles hold the other engine's kernels, or the earlier per-unit vectors
    for (auto& kv : mg.ws) kv.second->drop_graphs();
    ++mg.epoch;
    mg.mlp_engine = mg.mlp->engine;
    mg.mlp_version = mg.mlp->version;
  }
  int np = (nrhs + K - 1) / K;
  long long key = ws_key(K, np, prec);
  auto it = mg.ws.find(key);
  if (it != mg.ws.end()) return *it->second;
  auto w = std::make_unique<Workspace>();
  w->K = K;
  w->npanels = np;
  w->prec = prec;
  const size_t total = (size_t)mg.lv[0].n * K * np;
  if (prec == 2) {
    alloc_bufs(mg, w->f16, K, np);
    w->r32.alloc(total);
    std::vector<double> ones((size_t)K * np, 1.0);
    w->escale.upload(ones);
  } else if (prec == 1) {
    alloc_bufs(mg, w->f32, K, np);
  }
  else alloc_bufs(mg, w->f64, K, np);
  w->B64.alloc(total);
  w->U64.alloc(total);
  w->nblocks = (int)std::max<long long>(1, std::min<long long>(8LL * num_sms(), ((long long)mg.lv[0].n * K + TB - 1) / TB));
  w->partial.alloc((size_t)w->nblocks * K * np);
  w->norms.alloc((size_t)K * np);
  if (mg.opt.smoother == DEC_SMOOTH_CG) {
    w->scal.alloc((size_t)CG_NFIELDS * K * np);
    DEC_CUDA(cudaMemset(w->scal.p, 0, w->scal.bytes()));
  }
  if (mg.opt.coarse_solver == 2) {
    w->cs64.alloc((size_t)K * np);
    w->cs32.alloc((size_t)K * np);
    w->ceig.alloc((size_t)mg.lv[mg.lc].n * K * np);
    w->hcs64.assign((size_t)K * np, mg.opt.shift > 0 ? mg.opt.shift : 1.0);
    w->hcs32.assign((size_t)K * np, (float)w->hcs64[0]);
    DEC_CUDA(cudaMemcpy(w->cs64.p, w->hcs64.data(), w->cs64.bytes(), cudaMemcpyHostToDevice));
    DEC_CUDA(cudaMemcpy(w->cs32.p, w->hcs32.data(), w->cs32.bytes(), cudaMemcpyHostToDevice));
    for (auto& b : w->f32) b.cs = w->cs32.p;
    for (auto& b : w->f16) b.cs = w->cs32.p;
    for (auto& b : w->f64) b.cs = w->cs64.p;
  }
  DEC_CUDA(cudaMemset(w->B64.p, 0, w->B64.bytes()));
  DEC_CUDA(cudaMemset(w->U64.p, 0, w->U64.bytes()));
  auto& ref = *w;
  mg.ws[key] = std::move(w);
  return ref;
}

static Workspace& workspace(dec_mg& mg, int nrhs, int prec, bool drain = true) {
  return workspace_k(mg, nrhs, prec, choose_k(mg, nrhs, prec), drain);
}

// ||b_j||² of the FP64 right-hand-side panels into `out` (K * npanels).
static void enqueue_bnorms(const dec_mg& mg, Workspace& w, cudaStream_t s, double* out) {
  const int n = mg.lv[0].n, K = w.K, np = w.npanels;
  dim3 g(w.nblocks, np);
  add_bytes((double)n * K * np * 8.0);
  switch (K) {
#define DEC_K(KK) \
  case KK: k_panel_sumsq<KK><<<g, TB, 0, s>>>(n, w.B64.p, w.partial.p, (size_t)n * KK); break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
  }
  k_reduce_partials<<<K * np, 256, 0, s>>>(w.nblocks, K, np, w.partial.p, out);
  DEC_CHECK_LAUNCH();
}

// e = 0 on the finest level (the correction the first refinement step adds).
static void zero_correction(const dec_mg& mg, Workspace& w, cudaStream_t s) {
  const size_t total = (size_t)mg.lv[0].n * w.K * w.npanels;
  add_bytes((double)total * (w.prec == 2 ? 2.0 : w.prec == 1 ? 4.0 : 8.0));
  if (w.prec == 2) DEC_CUDA(cudaMemsetAsync(w.f16[0].x.p, 0, total * sizeof(__half), s));
  else if (w.prec == 1) DEC_CUDA(cudaMemsetAsync(w.f32[0].x.p, 0, total * sizeof(float), s));
  else DEC_CUDA(cudaMemsetAsync(w.f64[0].x.p, 0, total * sizeof(double), s));
}

// From a zero initial guess (FP32 / FP64 V-cycles): ||b||² and the first right-hand side r = b in
// one pass over b, and ||r||² = ||b||² for the first test.
static void enqueue_first_rhs(const dec_mg& mg, Workspace& w, cudaStream_t s) {
  const int n = mg.lv[0].n, K = w.K, np = w.npanels;
  dim3 g(w.nblocks, np);
  const size_t ps = (size_t)n * K;
  add_bytes((double)ps * np * (8.0 + (w.prec == 1 ? 4.0 : 8.0)));  // b read, r = b written
  switch (K) {
#define DEC_K(KK)                                                                                    \
  case KK:                                                                                           \
    if (w.prec == 1) k_first_rhs<KK, float><<<g, TB, 0, s>>>(n, w.B64.p, w.partial.p, ps, w.f32[0].b.p); \
    else k_first_rhs<KK, double><<<g, TB, 0, s>>>(n, w.B64.p, w.partial.p, ps, w.f64[0].b.p);         \
    break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
  }
  k_reduce_partials<<<K * np, 256, 0, s>>>(w.nblocks, K, np, w.partial.p, w.bn2.p);
  DEC_CHECK_LAUNCH();
  DEC_CUDA(cudaMemcpyAsync(w.norms.p, w.bn2.p, (size_t)K * np * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

// The whole refinement loop of a Jacobi / Chebyshev solve as one graph, from the FP64 panels
// (B64, U64) and the loop state (k_loop_init):
//   ||b||²; e = 0; [u += e; r = b - A u; test]; WHILE (test): { e = V^c(r); u += e; r = b - A u; test }
// The test (k_ir_check) sets the WHILE node's condition, so the solve needs no host round trip.
// zero_guess (u = 0; FP32 / FP64 V-cycles): the bracketed first step is r = b with its norms.
// When the step ends in a Jacobi / Chebyshev post-sweep (fused_update), the body's u += e is that
// sweep's epilogue (G_STEP) instead of a pass of its own.
static void capture_solve(dec_mg& mg, Workspace& w, bool zero_guess) {
  ensure_two_step(mg, w.K);
  if (w.bn2.n < (size_t)w.K * w.npanels) w.bn2.alloc((size_t)w.K * w.npanels);
  if (!w.loop.p) w.loop.alloc(1);
  cudaGraph_t g = nullptr;
  DEC_CUDA(cudaGraphCreate(&g, 0));
  auto fail = [&]() {
    cudaGraph_t junk = nullptr;
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(mg.cap, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
      cudaStreamEndCapture(mg.cap, &junk);
    cudaGraphDestroy(g);
  };
  try {
    cudaGraphConditionalHandle h;
    DEC_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    DEC_CUDA(cudaStreamBeginCaptureToGraph(mg.cap, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    w.solve_pre_bytes[zero_guess] = 0.0;
    t_bytes = &w.solve_pre_bytes[zero_guess];
    if (zero_guess && w.prec != 2) {
      enqueue_first_rhs(mg, w, mg.cap);
    } else {
      enqueue_bnorms(mg, w, mg.cap, w.bn2.p);
      zero_correction(mg, w, mg.cap);
      dispatch(mg, w, mg.cap, G_RESID);
    }
    k_ir_check<<<1, 256, 0, mg.cap>>>(h, w.norms.p, w.bn2.p, w.loop.p);
    DEC_CHECK_LAUNCH();
    t_bytes = nullptr;
    cudaStreamCaptureStatus st;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    DEC_CUDA(cudaStreamGetCaptureInfo(mg.cap, &st, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.handle = h;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    cudaGraphNode_t loop_node;
    DEC_CUDA(cudaGraphAddNode(&loop_node, cg, deps, ndeps, &prm));
    DEC_CUDA(cudaStreamUpdateCaptureDependencies(mg.cap, &loop_node, 1, cudaStreamSetCaptureDependencies));
    DEC_CUDA(cudaStreamEndCapture(mg.cap, &g));
    cudaGraph_t body = prm.conditional.phGraph_out[0];
    DEC_CUDA(cudaStreamBeginCaptureToGraph(mg.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    w.solve_body_bytes = 0.0;
    t_bytes = &w.solve_body_bytes;
    if (fused_update(mg, w)) {
      dispatch(mg, w, mg.cap, G_STEP);
    } else {
      dispatch(mg, w, mg.cap, G_VCYCLE);
      dispatch(mg, w, mg.cap, G_RESID);
    }
    k_ir_check<<<1, 256, 0, mg.cap>>>(h, w.norms.p, w.bn2.p, w.loop.p);
    DEC_CHECK_LAUNCH();
    t_bytes = nullptr;
    DEC_CUDA(cudaStreamEndCapture(mg.cap, &body));
    w.solve_pre[zero_guess] = count_kernel_nodes(g);
    w.solve_body = count_kernel_nodes(body);
    cudaGraphExec_t ex = nullptr;
    DEC_CUDA(cudaGraphInstantiate(&ex, g, 0));
    w.solve_graph[zero_guess] = ex;
  } catch (...) {
    t_bytes = nullptr;
    fail();
    throw;
  }
  cudaGraphDestroy(g);
}

// Panels in (b, and u or zero), the loop graph, panels out: the device part of a Jacobi /
// Chebyshev solve, enqueued on s (bd / ud device column-major).
static void enqueue_solve(dec_mg& mg, Workspace& w, const double* bd, double* ud, int nrhs, double rtol,
                          int max_iters, bool use_initial_guess, cudaStream_t s) {
  const Level& F = mg.lv[0];
  const int n = F.n, K = w.K, np = w.npanels;
  const size_t total = (size_t)n * K * np;
  const int z = use_initial_guess ? 0 : 1;
  if (!w.solve_graph[z]) capture_solve(mg, w, z == 1);
  to_panels(n, nrhs, K, np, F.diperm.p, bd, w.B64.p, s);
  if (use_initial_guess)
    to_panels(n, nrhs, K, np, F.diperm.p, ud, w.U64.p, s);
  else
    DEC_CUDA(cudaMemsetAsync(w.U64.p, 0, total * sizeof(double), s));
  k_loop_init<<<1, 1, 0, s>>>(w.loop.p, nrhs, max_iters, rtol);
  DEC_CHECK_LAUNCH();
  DEC_CUDA(cudaGraphLaunch(w.solve_graph[z], s));
  from_panels(n, nrhs, K, w.npanels, F.diperm.p, w.U64.p, ud, s);
  DEC_CHECK_LAUNCH();
}

static void fill_report(const Workspace& w, const LoopState& st, bool guess, float ms, dec_solve_report* rep) {
  if (!rep) return;
  rep->iterations = st.it;
  rep->converged = st.conv;
  rep->max_rel_residual = st.worst;
  rep->seconds = ms * 1e-3;
  // to_panels (b, and u), loop init, the graph's kernels, from_panels
  rep->launches = (guess ? 2 : 1) + 1 + w.solve_pre[guess ? 0 : 1] + (int64_t)st.it * w.solve_body + 1;
  rep->rhs_block = w.K;
  rep->fallback_iteration = -1;
}

// coarse_solver 2: RHS j gets the operator L + (shift + c_j) I (c_j = 0 without `shifts`).
static void set_shifts(const dec_mg& mg, Workspace& w, const double* shifts, int nrhs, cudaStream_t s) {
  if (mg.opt.coarse_solver != 2) {
    require(shifts == nullptr, "multigrid: per-RHS shifts need coarse_solver = 2");
    return;
  }
  for (size_t j = 0; j < w.hcs64.size(); ++j) {
    double c = mg.opt.shift + (shifts && (int)j < nrhs ? shifts[j] : 0.0);
    if ((int)j >= nrhs) c = 1.0;  // padding columns (zero right-hand sides)
    require(c > 0.0 && std::isfinite(c), "multigrid: every total shift must be positive and finite");
    w.hcs64[j] = c;
    w.hcs32[j] = (float)c;
  }
  DEC_CUDA(cudaMemcpyAsync(w.cs64.p, w.hcs64.data(), w.cs64.bytes(), cudaMemcpyHostToDevice, s));
  DEC_CUDA(cudaMemcpyAsync(w.cs32.p, w.hcs32.data(), w.cs32.bytes(), cudaMemcpyHostToDevice, s));
}

void mg_cycles(dec_mg* mg, double* u, const double* b, int nrhs, int cycles, void* stream) {
  require(mg != nullptr && u != nullptr && b != nullptr, "multigrid: null argument");
  require(nrhs >= 1 && cycles >= 0, "multigrid: bad nrhs / cycles");
  cudaStream_t s = as_stream(stream);
  Workspace& w = workspace(*mg, nrhs, 0);
  set_shifts(*mg, w, nullptr, nrhs, s);
  const Level& F = mg->lv[0];
  const int n = F.n;
  const size_t total = (size_t)n * w.K * w.npanels;
  to_panels(n, nrhs, w.K, w.npanels, F.diperm.p, b, w.B64.p, s);
  to_panels(n, nrhs, w.K, w.npanels, F.diperm.p, u, w.U64.p, s);
  DEC_CHECK_LAUNCH();
  if (!w.graph[G_CYCLE]) w.graph[G_CYCLE] = capture(*mg, w, G_CYCLE);
  for (int c = 0; c < cycles; ++c) DEC_CUDA(cudaGraphLaunch(w.graph[G_CYCLE], s));
  from_panels(n, nrhs, w.K, w.npanels, F.diperm.p, w.U64.p, u, s);
  DEC_CHECK_LAUNCH();
}

// full_multigrid (Multigrid.jl:826-855) at level l, b_l in bufs[l].b: restrict b to the next
// level, solve there recursively, prolong the result as the initial guess (P z onto zero), then
// `cycles` μ-cycles.  The recursion stops at the level the cycles solve directly.  Returns the
// buffer holding z_l.
template <class T, int K>
static T* fmg_T(const dec_mg& mg, Workspace& w, std::vector<LevelBufs<T>>& bufs, int l, int cycles, int np,
                cudaStream_t s) {
  const Level& L = mg.lv[l];
  LevelBufs<T>& B = bufs[l];
  const int last = mg.opt.smoother == DEC_SMOOTH_CG ? (int)mg.lv.size() - 1 : mg.lc;
  T* z = B.x.p;
  bool zero = true;
  if (l < last) {
    const Level& Cl = mg.lv[l + 1];
    LevelBufs<T>& Cb = bufs[l + 1];
    launch_restrict<T, K>(L, Cl, (const T*)B.b.p, Cb.b.p, np, s);
    T* zc = fmg_T<T, K>(mg, w, bufs, l + 1, cycles, np, s);
    launch_prolong<T, K>(L, Cl, (const T*)zc, z, true, np, s);
    zero = false;
  }
  for (int c = 0; c < cycles; ++c) {
    z = mu_cycle<T, K>(mg, w, bufs, l, z, zero, mg.opt.mu, np, s);
    zero = false;
  }
  if (zero) DEC_CUDA(cudaMemsetAsync(z, 0, (size_t)L.n * K * np * sizeof(T), s));
  return z;
}

template <int K>
static void fmg_K(dec_mg& mg, Workspace& w, int cycles, cudaStream_t s) {
  auto& bufs = w.f64;
  const size_t total = (size_t)mg.lv[0].n * K * w.npanels;
  DEC_CUDA(cudaMemcpyAsync(bufs[0].b.p, w.B64.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double* z = fmg_T<double, K>(mg, w, bufs, 0, cycles, w.npanels, s);
  DEC_CUDA(cudaMemcpyAsync(w.U64.p, z, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DEC_CHECK_LAUNCH();
}

void mg_full_multigrid(dec_mg* mg, double* u, const double* b, int nrhs, int cycles, void* stream) {
  require(mg != nullptr && u != nullptr && b != nullptr, "multigrid: null argument");
  require(nrhs >= 1 && cycles >= 0, "multigrid: bad nrhs / cycles");
  require(mg->opt.smoother != DEC_SMOOTH_LEARNED || mg->mlp != nullptr,
          "multigrid: the learned smoother needs a network (dec_mg_set_smoother_mlp)");
  cudaStream_t s = as_stream(stream);
  Workspace& w = workspace(*mg, nrhs, 0);
  set_shifts(*mg, w, nullptr, nrhs, s);
  const Level& F = mg->lv[0];
  const int n = F.n;
  const size_t total = (size_t)n * w.K * w.npanels;
  to_panels(n, nrhs, w.K, w.npanels, F.diperm.p, b, w.B64.p, s);
  DEC_CHECK_LAUNCH();
  switch (w.K) {
#define DEC_K(KK) \
  case KK: fmg_K<KK>(*mg, w, cycles, s); break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
    default: throw Error(DEC_ERR_INVALID_ARG, "multigrid: bad panel width");
  }
  from_panels(n, nrhs, w.K, w.npanels, F.diperm.p, w.U64.p, u, s);
  DEC_CHECK_LAUNCH();
}

dec_status mg_solve(dec_mg* mg, double* u, const double* b, int nrhs, double rtol, int max_iters,
                    dec_solve_report* rep, void* stream, bool host_buffers, bool use_initial_guess,
                    const double* shifts) {
  require(mg != nullptr && u != nullptr && b != nullptr, "multigrid: null argument");
  require(nrhs >= 1 && max_iters >= 1 && rtol > 0, "multigrid: bad nrhs / max_iters / rtol");
  cudaStream_t s = as_stream(stream);
  Workspace& w = workspace(*mg, nrhs, mg->opt.precision);
  set_shifts(*mg, w, shifts, nrhs, s);
  const Level& F = mg->lv[0];
  const int n = F.n;
  const int K = w.K, np = w.npanels;
  const size_t total = (size_t)n * K * np;
  cudaEvent_t e0, e1;
  DEC_CUDA(cudaEventCreate(&e0));
  DEC_CUDA(cudaEventCreate(&e1));
  DEC_CUDA(cudaEventRecord(e0, s));
  const double* bd = b;
  double* ud = u;
  if (host_buffers) {
    if (w.ucm.n < (size_t)n * nrhs) {
      w.ucm.alloc((size_t)n * nrhs);
      w.bcm.alloc((size_t)n * nrhs);
    }
    DEC_CUDA(cudaMemcpyAsync(w.bcm.p, b, (size_t)n * nrhs * 8, cudaMemcpyHostToDevice, s));
    if (use_initial_guess) DEC_CUDA(cudaMemcpyAsync(w.ucm.p, u, (size_t)n * nrhs * 8, cudaMemcpyHostToDevice, s));
    bd = w.bcm.p;
    ud = w.ucm.p;
  }
  if (mg->opt.smoother != DEC_SMOOTH_LEARNED && mg->opt.device_loop) {  // the refinement loop runs on the device
    enqueue_solve(*mg, w, bd, ud, nrhs, rtol, max_iters, use_initial_guess, s);
    if (host_buffers) DEC_CUDA(cudaMemcpyAsync(u, ud, (size_t)n * nrhs * 8, cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaEventRecord(e1, s));
    LoopState st;
    DEC_CUDA(cudaMemcpyAsync(&st, w.loop.p, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaEventSynchronize(e1));
    DEC_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    fill_report(w, st, use_initial_guess, ms, rep);
    return st.conv ? DEC_OK : DEC_ERR_NOT_CONVERGED;
  }
  to_panels(n, nrhs, K, np, F.diperm.p, bd, w.B64.p, s);
  if (use_initial_guess)
    to_panels(n, nrhs, K, np, F.diperm.p, ud, w.U64.p, s);
  else
    DEC_CUDA(cudaMemsetAsync(w.U64.p, 0, total * sizeof(double), s));
  const bool learned = mg->opt.smoother == DEC_SMOOTH_LEARNED;
  // the steps the device loop takes: from u = 0 the first residual is b (k_first_rhs), and the
  // update rides on the last sweep of each step's V-cycles (G_STEP)
  const bool zero_start = !use_initial_guess && !learned && w.prec != 2;
  const bool fuse = !learned && fused_update(*mg, w);
  std::vector<double> bn((size_t)K * np), rn((size_t)K * np);
  if (zero_start) {
    if (w.bn2.n < (size_t)K * np) w.bn2.alloc((size_t)K * np);
    enqueue_first_rhs(*mg, w, s);
    DEC_CUDA(cudaMemcpyAsync(bn.data(), w.bn2.p, bn.size() * 8, cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaStreamSynchronize(s));
    for (auto& x : bn) x = std::sqrt(x);
  } else {
    // the first refinement step adds e = 0
    if (w.prec == 2) DEC_CUDA(cudaMemsetAsync(w.f16[0].x.p, 0, total * sizeof(__half), s));
    else if (w.prec == 1) DEC_CUDA(cudaMemsetAsync(w.f32[0].x.p, 0, total * sizeof(float), s));
    else DEC_CUDA(cudaMemsetAsync(w.f64[0].x.p, 0, total * sizeof(double), s));
    DEC_CHECK_LAUNCH();
    // ||b|| per right-hand side.
    dim3 g(w.nblocks, np);
    switch (K) {
#define DEC_K(KK) \
  case KK: k_panel_sumsq<KK><<<g, TB, 0, s>>>(n, w.B64.p, w.partial.p, (size_t)n * KK); break;
      DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
    }
    k_reduce_partials<<<K * np, 256, 0, s>>>(w.nblocks, K, np, w.partial.p, w.norms.p);
    DEC_CHECK_LAUNCH();
    DEC_CUDA(cudaMemcpyAsync(bn.data(), w.norms.p, bn.size() * 8, cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaStreamSynchronize(s));
    for (auto& x : bn) x = std::sqrt(x);
  }
  if (!w.graph[G_RESID]) w.graph[G_RESID] = capture(*mg, w, G_RESID);
  if (!w.graph[G_VCYCLE]) w.graph[G_VCYCLE] = capture(*mg, w, G_VCYCLE);
  if (fuse && !w.graph[G_STEP]) w.graph[G_STEP] = capture(*mg, w, G_STEP);
  if (learned) {
    if (!w.graph[G_VCYCLE_PLAIN]) w.graph[G_VCYCLE_PLAIN] = capture(*mg, w, G_VCYCLE_PLAIN);
    if (w.Ubak.n < total) w.Ubak.alloc(total);
  }
  int64_t nl = (use_initial_guess ? 2 : 1) + 2;  // to_panels, ||b|| partials + reduce
  auto worst_rel = [&]() {  // the worst relative residual from the norms on the device
    DEC_CUDA(cudaMemcpyAsync(rn.data(), w.norms.p, rn.size() * 8, cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaStreamSynchronize(s));
    double wr = 0.0;
    for (int j = 0; j < nrhs; ++j) {
      const double rel = bn[j] > 0 ? std::sqrt(rn[j]) / bn[j] : std::sqrt(rn[j]);
      if (!std::isfinite(rel)) return HUGE_VAL;
      wr = std::max(wr, rel);
    }
    return wr;
  };
  auto residual = [&]() {  // u += e; r = b - A u; worst relative residual
    DEC_CUDA(cudaGraphLaunch(w.graph[G_RESID], s));
    nl += w.launches[G_RESID];
    return worst_rel();
  };
  int it = 0, fallback_at = -1;
  double worst = 0.0, prev = 0.0;
  bool conv = false, plain = !learned;
  for (;;) {
    const bool check = !plain && it > 0;
    if (check) DEC_CUDA(cudaMemcpyAsync(w.Ubak.p, w.U64.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
    worst = (it == 0 ? zero_start : fuse) ? worst_rel() : residual();
    if (check && !(worst <= mg->opt.fallback_rho * prev)) {
      // the learned step fell behind: undo it (u from before the step, e = 0, same residual)
      // and continue with the plain smoother
      DEC_CUDA(cudaMemcpyAsync(w.U64.p, w.Ubak.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
      if (w.prec == 2) DEC_CUDA(cudaMemsetAsync(w.f16[0].x.p, 0, total * sizeof(__half), s));
  else if (w.prec == 1) DEC_CUDA(cudaMemsetAsync(w.f32[0].x.p, 0, total * sizeof(float), s));
      else DEC_CUDA(cudaMemsetAsync(w.f64[0].x.p, 0, total * sizeof(double), s));
      worst = residual();
      plain = true;
      fallback_at = it;
    }
    if (worst <= rtol) {
      conv = true;
      break;
    }
    if (it >= max_iters) break;
    prev = worst;
    const int kind = fuse ? G_STEP : learned && plain ? G_VCYCLE_PLAIN : G_VCYCLE;
    DEC_CUDA(cudaGraphLaunch(w.graph[kind], s));  // e = V(r) (G_STEP: and u += e, r = b - A u)
    nl += w.launches[kind];
    ++it;
  }
  from_panels(n, nrhs, K, w.npanels, F.diperm.p, w.U64.p, ud, s);
  DEC_CHECK_LAUNCH();
  if (host_buffers) DEC_CUDA(cudaMemcpyAsync(u, ud, (size_t)n * nrhs * 8, cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaEventRecord(e1, s));
  DEC_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (learned) mlp_check_error(mg->mlp, s);  // a tcgen05 smoothing step whose wait timed out
  if (rep) {
    rep->iterations = it;
    rep->converged = conv ? 1 : 0;
    rep->max_rel_residual = worst;
    rep->seconds = ms * 1e-3;
    rep->launches = nl + 1;  // + from_panels
    rep->rhs_block = K;
    rep->fallback_iteration = fallback_at;
  }
  return conv ? DEC_OK : DEC_ERR_NOT_CONVERGED;
}

// Pipelined host-buffer solves.  Submit enqueues, on the hierarchy's own streams, the copy of b
// (and u) into the ticket's staging slot, the device solve (panels, loop graph, panels) and the
// copy of u back, and returns; three tickets may be in flight, so the copies of the solves
// before and after one overlap its compute.  Wait blocks on the ticket's copy-out and returns
// its report.
static void ensure_pipeline(dec_mg& mg) {
  if (mg.pipe[0]) return;
  for (cudaStream_t& p : mg.pipe) DEC_CUDA(cudaStreamCreateWithFlags(&p, cudaStreamNonBlocking));
  for (auto& sl : mg.pev)
    for (cudaEvent_t& e : sl) DEC_CUDA(cudaEventCreate(&e));
  DEC_CUDA(cudaMallocHost(&mg.hstate, dec_mg::kSlots * sizeof(LoopState)));
}

uint64_t mg_solve_submit(dec_mg* mg, double* u, const double* b, int nrhs, double rtol, int max_iters,
                         bool use_initial_guess) {
  require(mg != nullptr && u != nullptr && b != nullptr, "multigrid: null argument");
  require(nrhs >= 1 && max_iters >= 1 && rtol > 0, "multigrid: bad nrhs / max_iters / rtol");
  require(mg->opt.smoother != DEC_SMOOTH_LEARNED,
          "multigrid: pipelined solves run the Jacobi or Chebyshev smoother (the learned smoother's "
          "fallback test runs on the host)");
  const uint64_t ticket = mg->next_ticket;
  const int slot = (int)(ticket % dec_mg::kSlots);
  require(!mg->pend[slot].active, "multigrid: three pipelined solves are in flight; wait for the oldest one first");
  ensure_pipeline(*mg);
  cudaStream_t hin = mg->pipe[0], comp = mg->pipe[1], hout = mg->pipe[2];
  Workspace& w = workspace(*mg, nrhs, mg->opt.precision, false);
  set_shifts(*mg, w, nullptr, nrhs, comp);
  if (!w.solve_graph[use_initial_guess ? 0 : 1]) capture_solve(*mg, w, !use_initial_guess);
  const size_t len = (size_t)mg->lv[0].n * nrhs;
  DArr<double>& bs = w.pb[slot];
  DArr<double>& us = w.pu[slot];
  if (bs.n < len || us.n < len) {
    DEC_CUDA(cudaStreamSynchronize(comp));  // other slots' solves may still read the workspace
    if (bs.n < len) bs.alloc(len);
    if (us.n < len) us.alloc(len);
  }
  cudaEvent_t* ev = mg->pev[slot];
  DEC_CUDA(cudaEventRecord(ev[0], hin));
  DEC_CUDA(cudaMemcpyAsync(bs.p, b, len * 8, cudaMemcpyHostToDevice, hin));
  if (use_initial_guess) DEC_CUDA(cudaMemcpyAsync(us.p, u, len * 8, cudaMemcpyHostToDevice, hin));
  DEC_CUDA(cudaEventRecord(ev[1], hin));
  DEC_CUDA(cudaStreamWaitEvent(comp, ev[1], 0));
  enqueue_solve(*mg, w, bs.p, us.p, nrhs, rtol, max_iters, use_initial_guess, comp);
  DEC_CUDA(cudaMemcpyAsync(mg->hstate + slot, w.loop.p, sizeof(LoopState), cudaMemcpyDeviceToHost, comp));
  DEC_CUDA(cudaEventRecord(ev[2], comp));
  DEC_CUDA(cudaStreamWaitEvent(hout, ev[2], 0));
  DEC_CUDA(cudaMemcpyAsync(u, us.p, len * 8, cudaMemcpyDeviceToHost, hout));
  DEC_CUDA(cudaEventRecord(ev[3], hout));
  auto& pd = mg->pend[slot];
  pd.active = true;
  pd.ticket = ticket;
  pd.w = &w;
  pd.nrhs = nrhs;
  pd.guess = use_initial_guess;
  ++mg->next_ticket;
  return ticket;
}

dec_status mg_solve_wait(dec_mg* mg, uint64_t ticket, dec_solve_report* rep) {
  require(mg != nullptr, "multigrid: null argument");
  const int slot = (int)(ticket % dec_mg::kSlots);
  auto& pd = mg->pend[slot];
  require(pd.active && pd.ticket == ticket, "multigrid: unknown or already collected ticket");
  pd.active = false;
  cudaEvent_t* ev = mg->pev[slot];
  DEC_CUDA(cudaEventSynchronize(ev[3]));
  const LoopState st = mg->hstate[slot];
  float ms = 0;
  DEC_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[3]));
  fill_report(*pd.w, st, pd.guess, ms, rep);
  return st.conv ? DEC_OK : DEC_ERR_NOT_CONVERGED;
}

// ---------------------------------------------------------------------------------------------
// Profiling and autotuning
// ---------------------------------------------------------------------------------------------
template <class T, int K>
static void time_kernel_T(dec_mg& mg, Workspace& w, std::vector<LevelBufs<T>>& bufs, int kernel, int level, int reps,
                          cudaStream_t s, double* ms, double* bytes) {
  const Level& L = mg.lv[level];
  const int np = w.npanels;
  const size_t nk = (size_t)L.n * K * np;
  const double sz = sizeof(T);
  LevelBufs<T>& B = bufs[level];
  cudaEvent_t e0, e1;
  DEC_CUDA(cudaEventCreate(&e0));
  DEC_CUDA(cudaEventCreate(&e1));
  auto launch = [&]() {
    if (kernel == DEC_KERNEL_SWEEP) {
      SweepPrm<CT<T>> prm{};
      prm.mode = mg.opt.smoother == DEC_SMOOTH_JACOBI ? S_JACOBI : S_CHEBN;
      prm.omega = (CT<T>)mg.opt.omega;  // a middle Chebyshev step: reads the previous iterate from out
      prm.c1 = (CT<T>)0.5;
      prm.c2 = (CT<T>)0.25;
      launch_sweep<T, K>(L, B.b.p, B.x.p, B.y.p, prm, np, s, B.cs);
    } else if (kernel == DEC_KERNEL_SWEEP_PAIR) {
      launch_cheb2<T, K>(L, B.b.p, B.x.p, B.y.p, 0.5, 0.5, 0.25, np, s, nullptr);
    } else if (kernel == DEC_KERNEL_SWEEP_PROLONGED0 || kernel == DEC_KERNEL_SWEEP_PROLONGED1) {
      if constexpr (!std::is_same<T, __half>::value) {
        const Level& Cl = mg.lv[level + 1];
        if (kernel == DEC_KERNEL_SWEEP_PROLONGED0) {  // first step from x0 = P z
          launch_sweep_ap<T, K>(L, Cl, B.b.p, B.x.p, B.y.p, 0.5, false, bufs[level + 1].x.p, np, s, B.cs);
        } else {  // second step: x from the buffer, the previous iterate P z
          SweepPrm<CT<T>> prm{};
          prm.mode = S_CHEBN;
          prm.c1 = (CT<T>)0.5;
          prm.c2 = (CT<T>)0.25;
          launch_sweep_p<T, K>(L, Cl, B.b.p, B.x.p, B.y.p, prm, 1, bufs[level + 1].x.p, np, s, B.cs, nullptr);
        }
      }
    } else if (kernel == DEC_KERNEL_MLP) {
      if constexpr (!std::is_same<T, __half>::value)
        launch_mlp_smooth<T, K>(mlp_weights(mg.mlp), L.n, L.W, L.col.p, L.mtab.p, pick<T>(L.diag64, L.diag32),
                                B.b.p, B.x.p, 0, B.y.p, np, s);
    } else if (kernel == DEC_KERNEL_RESIDUAL) {
      dim3 g(w.nblocks, np);
      const Level& F = mg.lv[0];
      using R = typename std::conditional<std::is_same<T, __half>::value, float, T>::type;
      R* rout;
      if constexpr (std::is_same<T, __half>::value) rout = w.r32.p;
      else rout = bufs[0].b.p;
      if (F.W == 6)  // the variant the solve launches
        k_residual64<R, K, 6, false><<<g, TB, 0, s>>>(F.n, F.W, F.col.p, F.off64.p, F.diag64.p, w.B64.p, w.U64.p,
                                                      rout, w.partial.p, (size_t)F.n * K, nullptr);
      else
        k_residual64<R, K, 0, false><<<g, TB, 0, s>>>(F.n, F.W, F.col.p, F.off64.p, F.diag64.p, w.B64.p, w.U64.p,
                                                      rout, w.partial.p, (size_t)F.n * K, nullptr);
    } else if (kernel == DEC_KERNEL_RESTRICT) {
      const Level& Cl = mg.lv[level + 1];
      launch_restrict<T, K>(L, Cl, (const T*)B.x.p, bufs[level + 1].b.p, np, s, false);
    } else {
      const Level& Cl = mg.lv[level + 1];
      launch_prolong<T, K>(L, Cl, (const T*)bufs[level + 1].x.p, B.x.p, false, np, s, false);
    }
  };
  launch();  // warm-up
  DEC_CUDA(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; ++r) launch();
  DEC_CUDA(cudaEventRecord(e1, s));
  DEC_CHECK_LAUNCH();
  DEC_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / reps;
  if (kernel == DEC_KERNEL_SWEEP) {
    double mat = (double)L.n * (L.W * (4.0 + sz) + 2 * sz);
    *bytes = mat + prm_vectors(mg.opt.smoother) * (double)nk * sz;
  } else if (kernel == DEC_KERNEL_SWEEP_PAIR) {
    *bytes = (double)L.n * (L.W * (4.0 + sz) + 2 * sz) + 3.0 * (double)nk * sz;  // operator, x, b, out once
  } else if (kernel == DEC_KERNEL_SWEEP_PROLONGED0 || kernel == DEC_KERNEL_SWEEP_PROLONGED1) {
    // step 1: A P rows, 1/diagonal, the coarse correction, b and out; step 2: the operator row with
    // 1/diagonal, parents, the coarse correction, x, b and out
    const Level& Cl = mg.lv[level + 1];
    const double rows = kernel == DEC_KERNEL_SWEEP_PROLONGED0 ? (double)L.n * (kApW * (4.0 + sz) + sz)
                                                               : (double)L.n * (L.W * (4.0 + sz) + 2 * sz + 8.0);
    *bytes = rows + (double)Cl.n * K * np * sz + (kernel == DEC_KERNEL_SWEEP_PROLONGED0 ? 2.0 : 3.0) * (double)nk * sz;
  } else if (kernel == DEC_KERNEL_MLP) {
    *bytes = (double)L.n * (L.W * (4.0 + sz) + sz) + 3.0 * (double)nk * sz;  // operator, r, x, out
  } else if (kernel == DEC_KERNEL_RESIDUAL) {
    const Level& F = mg.lv[0];
    double mat = (double)F.n * (F.W * 12.0 + 8);
    *bytes = mat + (double)F.n * K * np * (8 + 8 + sz);
  } else if (kernel == DEC_KERNEL_RESTRICT) {
    const Level& Cl = mg.lv[level + 1];
    const double idx = L.gen ? (double)Cl.n * L.Wr * (4.0 + sizeof(CT<T>)) : (double)Cl.n * ((L.Wq + 1) * 4.0 + 2 * sizeof(CT<T>));
    *bytes = idx + (double)nk * sz + (double)Cl.n * K * np * sz;
  } else {
    const Level& Cl = mg.lv[level + 1];
    const double idx = L.gen ? (double)L.n * L.Wp * (4.0 + sizeof(CT<T>)) : (double)L.n * 8.0;
    *bytes = idx + (double)Cl.n * K * np * sz + 2.0 * nk * sz;
  }
}

template <int K>
static void time_kernel_K(dec_mg& mg, Workspace& w, int kernel, int level, int reps, cudaStream_t s, double* ms,
                          double* bytes) {
  if (w.prec == 2) time_kernel_T<__half, K>(mg, w, w.f16, kernel, level, reps, s, ms, bytes);
  else if (w.prec == 1) time_kernel_T<float, K>(mg, w, w.f32, kernel, level, reps, s, ms, bytes);
  else time_kernel_T<double, K>(mg, w, w.f64, kernel, level, reps, s, ms, bytes);
}

void mg_time_kernel(dec_mg* mg, int kernel, int level, int nrhs, int reps, void* stream, double* ms, double* bytes) {
  require(mg != nullptr && ms != nullptr && bytes != nullptr, "multigrid: null argument");
  require(kernel >= 0 && kernel <= 7, "multigrid: unknown kernel");
  if (kernel == DEC_KERNEL_SWEEP_PROLONGED0 || kernel == DEC_KERNEL_SWEEP_PROLONGED1) {
    require(level >= 0 && level + 1 < (int)mg->lv.size(), "multigrid: level out of range");
    const Level& L = mg->lv[level];
    require(mg->opt.precision != 2 && L.ap_ok,
            "multigrid: the prolonged sweeps run on FP32 / FP64 panels over rows of 6 slots with subdivision transfers");
  }
  if (kernel == DEC_KERNEL_SWEEP_PAIR) {
    Level& L = mg->lv[level];
    const int K = choose_k(*mg, nrhs, mg->opt.precision);
    require(mg->opt.precision == 1 && K >= 16 && L.W == 6 && L.n >= kCheb2MinRows,
            "multigrid: the sweep pair runs on FP32 panels of 16 or more over rows of 6 slots");
    cheb2_opt_in();
    const int tuned = tune_get(cheb2_key(K, L.W, L.n), 0);
    const int P = tuned > 0 ? tuned : kTwoStepRows;  // the table's patch size, else the largest
    if (!L.ts.npatch || L.ts.P != P) build_two_step(L, P);
  }
  require(kernel != DEC_KERNEL_MLP || mg->mlp != nullptr, "multigrid: no learned smoother network set");
  require(level >= 0 && level < (int)mg->lv.size() - (kernel == 2 || kernel == 3 || kernel >= 6 ? 1 : 0),
          "multigrid: level out of range");
  require(reps >= 1 && nrhs >= 1, "multigrid: reps and nrhs must be positive");
  Workspace& w = workspace(*mg, nrhs, mg->opt.precision);
  cudaStream_t s = as_stream(stream);
  switch (w.K) {
#define DEC_K(KK) \
  case KK: time_kernel_K<KK>(*mg, w, kernel, level, reps, s, ms, bytes); break;
    DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
  }
}

// Algorithmic bytes of a device-loop solve of nrhs right-hand sides that ran `iterations`
// refinement steps: b (and u) into panels, the graph's part before its loop, `iterations` loop
// bodies, u out of panels.  Captures the solve graph if no solve of this shape ran yet.
double mg_solve_traffic(dec_mg* mg, int nrhs, int from_zero, int iterations) {
  require(mg != nullptr && nrhs >= 1 && iterations >= 0, "multigrid: bad solve-traffic arguments");
  require((mg->opt.smoother == DEC_SMOOTH_JACOBI || mg->opt.smoother == DEC_SMOOTH_CHEBYSHEV) &&
              mg->opt.device_loop == 1,
          "multigrid: solve traffic is counted for the device refinement loop (Jacobi / Chebyshev smoothers)");
  require(!from_zero || mg->opt.precision != 2, "multigrid: FP16 storage has no solve from zero");
  Workspace& w = workspace(*mg, nrhs, mg->opt.precision);
  const int z = from_zero ? 1 : 0;
  if (!w.solve_graph[z]) capture_solve(*mg, w, z == 1);
  const double n = mg->lv[0].n, cm = n * nrhs * 8.0, pan = n * w.K * w.npanels * 8.0;
  double by = cm + pan + n * 4.0;                  // b into panels (with the row permutation)
  by += from_zero ? pan : cm + pan + n * 4.0;      // U cleared, or u into panels
  by += w.solve_pre_bytes[z] + iterations * w.solve_body_bytes;
  by += pan + cm + n * 4.0;                        // u out of panels
  return by;
}

// MultigridData.steps per level (pre = post = steps[l]); null restores the options' pre / post.
void mg_set_level_steps(dec_mg* mg, const int* steps) {
  require(mg != nullptr, "multigrid: null handle");
  drain_pipeline(*mg);
  const int nl = (int)mg->lv.size();
  if (steps) {
    for (int k = 0; k < nl; ++k) require(steps[k] >= 0 && steps[k] <= 16, "multigrid: steps must be in [0, 16]");
    mg->steps.assign(steps, steps + nl);
  } else {
    mg->steps.clear();
  }
  for (auto& kv : mg->ws) kv.second->drop_graphs();  // captured cycles hold the old sweep counts
  ++mg->epoch;
}

void mg_set_smoother_mlp(dec_mg* mg, const dec_mlp* mlp) {
  require(mg != nullptr, "multigrid: null argument");
  require(mlp == nullptr || mg->lv[0].mesh != nullptr,
          "multigrid: the learned smoother needs mesh levels (not a hierarchy built from matrices)");
  if (mg->mlp == mlp) return;
  if (mlp)  // the per-row coupling features the network reads on every level
    for (Level& L : mg->lv)
      if (!L.mtab.p) build_mlp_table(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, L.mtab);
  mg->mlp = mlp;
  for (auto& kv : mg->ws) kv.second->drop_graphs();  // captured cycles hold the old weights' addresses
  ++mg->epoch;
}

int mg_autotune(dec_mg* mg, int nrhs, int reps, void* stream) {
  require(mg != nullptr && nrhs >= 1 && reps >= 1, "multigrid: bad autotune arguments");
  cudaStream_t s = as_stream(stream);
  const int prec = mg->opt.precision;
  int best = 0;
  double best_t = 1e300;
  cudaEvent_t e0, e1;
  DEC_CUDA(cudaEventCreate(&e0));
  DEC_CUDA(cudaEventCreate(&e1));
  for (int K = 1; K <= 32; K <<= 1) {
    if (K > 1 && (K / 2) >= nrhs) break;  // wider panels would only add padding
    Workspace& w = workspace_k(*mg, nrhs, prec, K);
    if (!w.graph[G_VCYCLE]) w.graph[G_VCYCLE] = capture(*mg, w, G_VCYCLE);
    DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
    std::vector<float> ts;
    for (int r = 0; r < std::max(3, reps); ++r) {  // median of single-launch timings
      DEC_CUDA(cudaEventRecord(e0, s));
      DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
      DEC_CUDA(cudaEventRecord(e1, s));
      DEC_CUDA(cudaEventSynchronize(e1));
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      ts.push_back(t);
    }
    std::sort(ts.begin(), ts.end());
    double t = ts[ts.size() / 2];
    if (t < best_t) {
      best_t = t;
      best = K;
    }
  }
  // FP32 panels of 8 or more: the sweep's lanes per row (vector width 4, the default, or 2), timed
  // on the same V-cycle with the variant on every level, kept in the tuning table per level
  if (prec == 1 && best >= 8) {
    Workspace& w = workspace_k(*mg, nrhs, prec, best);
    auto set_all = [&](int v) {
      for (const Level& L : mg->lv) tune_set(sweep_key(best, L.W, L.n), v);
      w.drop_graphs();
    };
    int best_v = 4;
    double best_vt = 1e300;
    for (int v : {4, 2}) {
      set_all(v);
      w.graph[G_VCYCLE] = capture(*mg, w, G_VCYCLE);
      DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
      std::vector<float> ts;
      for (int r = 0; r < std::max(3, reps); ++r) {
        DEC_CUDA(cudaEventRecord(e0, s));
        DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
        DEC_CUDA(cudaEventRecord(e1, s));
        DEC_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        ts.push_back(t);
      }
      std::sort(ts.begin(), ts.end());
      if (ts[ts.size() / 2] < best_vt) {
        best_vt = ts[ts.size() / 2];
        best_v = v;
      }
    }
    set_all(best_v);
  }
  // Chebyshev post-smoothing pairs (post = 2) on FP32 panels of 16 or more: the two steps as one
  // temporal-blocked pass (k_cheb2) or as two sweeps, timed on the same V-cycle with the choice on every
  // level of at least kCheb2MinRows rows
  if (prec == 1 && best >= 16 && mg->opt.smoother == DEC_SMOOTH_CHEBYSHEV && mg->post_at(0) == 2) {
    Workspace& w = workspace_k(*mg, nrhs, prec, best);
    auto set_all = [&](int v) {
      for (const Level& L : mg->lv)
        if (L.W == 6 && L.n >= kCheb2MinRows) tune_set(cheb2_key(best, L.W, L.n), v);
      w.drop_graphs();
    };
    int best_c = 0;
    double best_ct = 1e300;
    for (int v : {0, 512, 256, 128}) {
      set_all(v);
      w.graph[G_VCYCLE] = capture(*mg, w, G_VCYCLE);
      DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
      std::vector<float> ts;
      for (int r = 0; r < std::max(3, reps); ++r) {
        DEC_CUDA(cudaEventRecord(e0, s));
        DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
        DEC_CUDA(cudaEventRecord(e1, s));
        DEC_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        ts.push_back(t);
      }
      std::sort(ts.begin(), ts.end());
      if (ts[ts.size() / 2] < best_ct) {
        best_ct = ts[ts.size() / 2];
        best_c = v;
      }
    }
    set_all(best_c);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int K = 1; K <= 32; K <<= 1) {
    if (K == best) continue;
    int np = (nrhs + K - 1) / K;
    mg->ws.erase(ws_key(K, np, prec));
  }
  ++mg->epoch;
  mg->tuned[((long long)nrhs << 2) | prec] = best;
  return best;
}

}  // namespace decb

// ---------------------------------------------------------------------------------------------
// Batched solves over several hierarchies (meshes of uneven sizes): every refinement step of all
// groups is one CUDA graph whose branches (one per group, on forked streams) run concurrently;
// the host reads all groups' residual norms with one copy per step.
// ---------------------------------------------------------------------------------------------
// The state of a batched solve's refinement loop (one graph with a conditional WHILE node).
struct BatchState {
  int it;         // refinement steps run
  int max_iters;
  int all;        // every group converged
  int pad;
  double rtol;
};

struct dec_batch {
  std::vector<dec_mg*> groups;                 // not owned
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  cudaStream_t cap = nullptr;
  decb::DArr<double> norms, bn2;               // all groups' squared residual / right-hand-side norms
  decb::DArr<int32_t> meta;                    // per group: offset into norms, right-hand sides
  decb::DArr<int32_t> conv_at;                 // per group: step at which it converged, -1 before
  decb::DArr<double> worst;                    // per group: worst relative residual at the last test
  decb::DArr<BatchState> state;
  std::vector<size_t> off;                     // group g's norms at norms[off[g]]
  std::vector<decb::Workspace*> used;          // workspaces the graph was captured on
  std::vector<uint64_t> epochs;
  std::vector<const void*> bufs;               // the caller's u / rhs pointers baked into the graph
  std::vector<int> nrhs;
  cudaGraphExec_t graph = nullptr;             // the whole solve: panels in, loop, panels out
  int64_t launches_pre = 0, launches_body = 0; // kernel nodes outside / inside the WHILE body
  double bytes_pre = 0.0, bytes_body = 0.0;     // algorithmic bytes outside / inside the WHILE body
  void drop_graphs() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  ~dec_batch() {
    drop_graphs();
    for (auto st : streams) cudaStreamDestroy(st);
    for (auto e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (cap) cudaStreamDestroy(cap);
  }
};

namespace decb {

dec_batch* batch_create(dec_mg* const* groups, int ngroups) {
  require(groups != nullptr && ngroups >= 1 && ngroups <= 256, "batch: need 1..256 hierarchies");
  auto b = std::make_unique<dec_batch>();
  for (int g = 0; g < ngroups; ++g) {
    require(groups[g] != nullptr, "batch: null hierarchy");
    for (int h = 0; h < g; ++h) require(groups[h] != groups[g], "batch: a hierarchy appears twice");
    const int sm = groups[g]->opt.smoother;
    require(sm == DEC_SMOOTH_JACOBI || sm == DEC_SMOOTH_CHEBYSHEV, "batch: groups need the Jacobi or Chebyshev smoother");
    b->groups.push_back(groups[g]);
    cudaStream_t st;
    DEC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->streams.push_back(st);
    cudaEvent_t e;
    DEC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->join.push_back(e);
  }
  DEC_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  DEC_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  b->conv_at.alloc(ngroups);
  b->worst.alloc(ngroups);
  b->state.alloc(1);
  return b.release();
}

void batch_destroy(dec_batch* b) { delete b; }

__global__ void k_batch_init(BatchState* st, int* conv_at, int G, int max_iters, double rtol) {
  for (int q = threadIdx.x; q < G; q += blockDim.x) conv_at[q] = -1;
  if (threadIdx.x == 0) {
    st->it = 0;
    st->max_iters = max_iters;
    st->all = 0;
    st->rtol = rtol;
  }
}

// The batch's residual test after step `it` (+1 inside the loop body): per group the worst
// ||b_j - A u_j|| / ||b_j|| over its right-hand sides, the step at which it first reached rtol, and
// the WHILE node's condition: not every group converged and fewer than max_iters steps.
__global__ void __launch_bounds__(256) k_batch_check(cudaGraphConditionalHandle h, int G,
                                                     const int32_t* __restrict__ meta, const double* __restrict__ n2,
                                                     const double* __restrict__ bn2, BatchState* st, int* conv_at,
                                                     double* worst, int step) {
  __shared__ int all;
  if (threadIdx.x == 0) all = 1;
  __syncthreads();
  const int it = st->it + step;
  const double rtol = st->rtol;
  for (int q = threadIdx.x; q < G; q += blockDim.x) {
    const int off = meta[2 * q], nr = meta[2 * q + 1];
    double wr = 0.0;
    for (int j = 0; j < nr; ++j) {
      const double r = sqrt(n2[off + j]), bn = sqrt(bn2[off + j]);
      const double rel = bn > 0 ? r / bn : r;
      wr = isfinite(rel) ? fmax(wr, rel) : HUGE_VAL;
    }
    worst[q] = wr;
    if (conv_at[q] < 0 && wr <= rtol) conv_at[q] = it;
    if (conv_at[q] < 0) atomicAnd(&all, 0);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    st->it = it;
    st->all = all;
    cudaGraphSetConditional(h, (!all && it < st->max_iters) ? 1u : 0u);
  }
}

// Every group's branch of one phase on its own stream, forked from and joined back to bt.cap.
template <class F>
static void per_group(dec_batch& bt, F&& f) {
  DEC_CUDA(cudaEventRecord(bt.fork, bt.cap));
  for (size_t q = 0; q < bt.groups.size(); ++q) {
    cudaStream_t st = bt.streams[q];
    DEC_CUDA(cudaStreamWaitEvent(st, bt.fork, 0));
    f(q, st);
    DEC_CUDA(cudaEventRecord(bt.join[q], st));
    DEC_CUDA(cudaStreamWaitEvent(bt.cap, bt.join[q], 0));
  }
}

// The whole batched solve as one graph (caller buffers u / rhs baked in):
//   per group: b and u into panels, e = 0, ||b||², r = b - A u and its norms;  test (step 0);
//   WHILE (test): { per group: V-cycles, u += e, r = b - A u, norms;  test }
//   per group: u out of panels.
static cudaGraphExec_t batch_capture(dec_batch& bt, double* const* u, const double* const* rhs, const int* nrhs) {
  for (size_t q = 0; q < bt.groups.size(); ++q) ensure_two_step(*bt.groups[q], bt.used[q]->K);
  cudaGraph_t g = nullptr;
  DEC_CUDA(cudaGraphCreate(&g, 0));
  const int G = (int)bt.groups.size();
  auto fail = [&]() {
    cudaGraph_t junk = nullptr;
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(bt.cap, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
      cudaStreamEndCapture(bt.cap, &junk);
    cudaGraphDestroy(g);
  };
  try {
    cudaGraphConditionalHandle h;
    DEC_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    DEC_CUDA(cudaStreamBeginCaptureToGraph(bt.cap, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    bt.bytes_pre = bt.bytes_body = 0.0;
    t_bytes = &bt.bytes_pre;
    per_group(bt, [&](size_t q, cudaStream_t st) {
      dec_mg& mg = *bt.groups[q];
      Workspace& w = *bt.used[q];
      const Level& F = mg.lv[0];
      const int n = F.n, K = w.K, np = w.npanels;
      to_panels(n, nrhs[q], K, np, F.diperm.p, rhs[q], w.B64.p, st);
      to_panels(n, nrhs[q], K, np, F.diperm.p, u[q], w.U64.p, st);
      // b and u into panels, u out of panels at the end: caller vectors, panels, the row permutation
      add_bytes(3.0 * ((double)n * nrhs[q] * 8.0 + (double)n * K * np * 8.0 + n * 4.0));
      zero_correction(mg, w, st);
      enqueue_bnorms(mg, w, st, bt.bn2.p + bt.off[q]);
      dispatch(mg, w, st, G_RESID);
      DEC_CUDA(cudaMemcpyAsync(bt.norms.p + bt.off[q], w.norms.p, w.norms.bytes(), cudaMemcpyDeviceToDevice, st));
    });
    k_batch_check<<<1, 256, 0, bt.cap>>>(h, G, bt.meta.p, bt.norms.p, bt.bn2.p, bt.state.p, bt.conv_at.p,
                                         bt.worst.p, 0);
    DEC_CHECK_LAUNCH();
    t_bytes = nullptr;
    cudaStreamCaptureStatus cst;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    DEC_CUDA(cudaStreamGetCaptureInfo(bt.cap, &cst, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.handle = h;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    cudaGraphNode_t loop_node;
    DEC_CUDA(cudaGraphAddNode(&loop_node, cg, deps, ndeps, &prm));
    DEC_CUDA(cudaStreamUpdateCaptureDependencies(bt.cap, &loop_node, 1, cudaStreamSetCaptureDependencies));
    per_group(bt, [&](size_t q, cudaStream_t st) {
      dec_mg& mg = *bt.groups[q];
      Workspace& w = *bt.used[q];
      const Level& F = mg.lv[0];
      from_panels(F.n, nrhs[q], w.K, w.npanels, F.diperm.p, w.U64.p, u[q], st);
    });
    DEC_CUDA(cudaStreamEndCapture(bt.cap, &g));
    cudaGraph_t body = prm.conditional.phGraph_out[0];
    DEC_CUDA(cudaStreamBeginCaptureToGraph(bt.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    t_bytes = &bt.bytes_body;
    per_group(bt, [&](size_t q, cudaStream_t st) {
      dec_mg& mg = *bt.groups[q];
      Workspace& w = *bt.used[q];
      if (fused_update(mg, w)) {
        dispatch(mg, w, st, G_STEP);  // V-cycles with u += e in the last sweep, then the residual
      } else {
        dispatch(mg, w, st, G_VCYCLE);
        dispatch(mg, w, st, G_RESID);
      }
      DEC_CUDA(cudaMemcpyAsync(bt.norms.p + bt.off[q], w.norms.p, w.norms.bytes(), cudaMemcpyDeviceToDevice, st));
    });
    k_batch_check<<<1, 256, 0, bt.cap>>>(h, G, bt.meta.p, bt.norms.p, bt.bn2.p, bt.state.p, bt.conv_at.p,
                                         bt.worst.p, 1);
    DEC_CHECK_LAUNCH();
    t_bytes = nullptr;
    DEC_CUDA(cudaStreamEndCapture(bt.cap, &body));
    bt.launches_pre = count_kernel_nodes(g);
    bt.launches_body = count_kernel_nodes(body);
    cudaGraphExec_t ex = nullptr;
    DEC_CUDA(cudaGraphInstantiate(&ex, g, 0));
    cudaGraphDestroy(g);
    return ex;
  } catch (...) {
    t_bytes = nullptr;
    fail();
    throw;
  }
}

double batch_traffic(const dec_batch* b, int iterations) {
  require(b != nullptr && iterations >= 0, "batch: bad traffic arguments");
  require(b->graph != nullptr, "batch: no captured solve (call dec_batch_solve first)");
  return b->bytes_pre + iterations * b->bytes_body;
}

void batch_autotune(dec_batch* b, const int* nrhs, int reps, void* stream) {
  require(b != nullptr && nrhs != nullptr, "batch: null argument");
  for (size_t q = 0; q < b->groups.size(); ++q) mg_autotune(b->groups[q], nrhs[q], reps, stream);
  b->drop_graphs();
}

dec_status batch_solve(dec_batch* b, double* const* u, const double* const* rhs, const int* nrhs,
                       const double* const* shifts, double rtol, int max_iters, dec_solve_report* reps,
                       dec_solve_report* total, void* stream) {
  require(b != nullptr && u != nullptr && rhs != nullptr && nrhs != nullptr, "batch: null argument");
  require(max_iters >= 1 && rtol > 0, "batch: bad max_iters / rtol");
  const size_t G = b->groups.size();
  cudaStream_t s = as_stream(stream);
  // workspaces (autotuned panel widths) and the graph's identity: any change recaptures it
  std::vector<Workspace*> ws(G);
  std::vector<uint64_t> ep(G);
  std::vector<const void*> bufs(2 * G);
  std::vector<int> nr(nrhs, nrhs + G);
  size_t nn = 0;
  std::vector<size_t> off(G);
  for (size_t q = 0; q < G; ++q) {
    dec_mg& mg = *b->groups[q];
    require(u[q] != nullptr && rhs[q] != nullptr && nrhs[q] >= 1, "batch: bad group arguments");
    ws[q] = &workspace(mg, nrhs[q], mg.opt.precision);
    ep[q] = mg.epoch;
    off[q] = nn;
    nn += ws[q]->norms.n;
    bufs[2 * q] = u[q];
    bufs[2 * q + 1] = rhs[q];
  }
  if (ws != b->used || ep != b->epochs || b->off != off || bufs != b->bufs || nr != b->nrhs) {
    b->drop_graphs();
    b->used = ws;
    b->epochs = ep;
    b->off = off;
    b->bufs = bufs;
    b->nrhs = nr;
    if (b->norms.n < nn) {
      b->norms.alloc(nn);
      b->bn2.alloc(nn);
    }
    std::vector<int32_t> meta(2 * G);
    for (size_t q = 0; q < G; ++q) {
      meta[2 * q] = (int32_t)off[q];
      meta[2 * q + 1] = nrhs[q];
    }
    b->meta.upload(meta);
  }
  cudaEvent_t e0, e1;
  DEC_CUDA(cudaEventCreate(&e0));
  DEC_CUDA(cudaEventCreate(&e1));
  DEC_CUDA(cudaEventRecord(e0, s));
  for (size_t q = 0; q < G; ++q) set_shifts(*b->groups[q], *ws[q], shifts ? shifts[q] : nullptr, nrhs[q], s);
  if (!b->graph) b->graph = batch_capture(*b, u, rhs, nrhs);
  k_batch_init<<<1, 256, 0, s>>>(b->state.p, b->conv_at.p, (int)G, max_iters, rtol);
  DEC_CHECK_LAUNCH();
  DEC_CUDA(cudaGraphLaunch(b->graph, s));
  DEC_CUDA(cudaEventRecord(e1, s));
  BatchState st;
  std::vector<int32_t> conv(G);
  std::vector<double> worst(G);
  DEC_CUDA(cudaMemcpyAsync(&st, b->state.p, sizeof(BatchState), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaMemcpyAsync(conv.data(), b->conv_at.p, G * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaMemcpyAsync(worst.data(), b->worst.p, G * sizeof(double), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double wmax = 0.0;
  for (size_t q = 0; q < G; ++q) {
    wmax = std::max(wmax, worst[q]);
    if (reps) {
      reps[q].iterations = conv[q] >= 0 ? conv[q] : st.it;
      reps[q].converged = conv[q] >= 0 ? 1 : 0;
      reps[q].max_rel_residual = worst[q];
      reps[q].seconds = ms * 1e-3;
      reps[q].launches = 0;
      reps[q].rhs_block = ws[q]->K;
      reps[q].fallback_iteration = -1;
    }
  }
  if (total) {
    total->iterations = st.it;
    total->converged = st.all ? 1 : 0;
    total->max_rel_residual = wmax;
    total->seconds = ms * 1e-3;
    total->launches = 1 + b->launches_pre + (int64_t)st.it * b->launches_body;  // init kernel, graph
    total->rhs_block = 0;
    total->fallback_iteration = -1;
  }
  return st.all ? DEC_OK : DEC_ERR_NOT_CONVERGED;
}

}  // namespace decb
