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
// Solve layout: right-hand sides are processed in panels of K (1..32) stored row-major
// ([panel][row][K]), so a row's K values are one contiguous 4K- or 8K-byte segment and each
// neighbour gather of the SpMV is a coalesced segment shared by K lanes; the K lanes of a row
// read the same matrix entries (one broadcast transaction).  A panel grid dimension processes
// all panels in one launch, which keeps the coarse levels from being launch-bound.  The
// smoothers are damped Jacobi or Chebyshev-Jacobi (bounds from a GPU power iteration); the
// coarsest level is a dense FP64 solve with the precomputed inverse.  Mixed precision runs the
// V-cycle in FP32 on the FP64 residual inside FP64 iterative refinement.  Each refinement step
// (update, residual, norms, V-cycle) is one CUDA graph.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <numeric>

#include "mg.cuh"

dec_op* op_create_impl(dec_mesh* mh, int kind, double shift, dec_dtype dt);

namespace decb {

// ---------------------------------------------------------------------------------------------
// Host topology refinement (Multigrid.jl:111-219)
// ---------------------------------------------------------------------------------------------
struct HostLevel {
  int nv = 0, ne = 0, nt = 0;
  std::vector<int32_t> ev0, ev1, te0, te1, te2;
  std::vector<int8_t> eo, to;
  std::vector<double> pts;
};

// refine(::BinarySubdivision, topo), Multigrid.jl:130-183 (0-based: coarse edge e -> fine
// edges 2e, 2e+1; triangle t -> interior edges 2ne+3t.., children 4t..4t+3).
static HostLevel refine_level(const HostLevel& c, double radius, const std::vector<int8_t>* flip) {
  HostLevel f;
  f.nv = c.nv + c.ne;
  f.ne = 2 * c.ne + 3 * c.nt;
  f.nt = 4 * c.nt;
  f.ev0.resize(f.ne);
  f.ev1.resize(f.ne);
  for (int e = 0; e < c.ne; ++e) {
    int m = c.nv + e;
    f.ev0[2 * e] = m;
    f.ev1[2 * e] = c.ev0[e];
    f.ev0[2 * e + 1] = m;
    f.ev1[2 * e + 1] = c.ev1[e];
  }
  f.te0.resize(f.nt);
  f.te1.resize(f.nt);
  f.te2.resize(f.nt);
  f.to.resize(f.nt);
  for (int t = 0; t < c.nt; ++t) {
    int e0 = c.te0[t], e1 = c.te1[t], e2 = c.te2[t];
    int m0 = e0 + c.nv, m1 = e1 + c.nv, m2 = e2 + c.nv;
    int m0_m1 = 2 * c.ne + 3 * t, m1_m2 = m0_m1 + 1, m0_m2 = m0_m1 + 2;
    f.ev0[m0_m1] = m1; f.ev1[m0_m1] = m0;
    f.ev0[m1_m2] = m2; f.ev1[m1_m2] = m1;
    f.ev0[m0_m2] = m2; f.ev1[m0_m2] = m0;
    int m0_v1 = 2 * e0 + 1, v2_m0 = 2 * e0, m1_v0 = 2 * e1 + 1, v2_m1 = 2 * e1, m2_v0 = 2 * e2 + 1,
        v1_m2 = 2 * e2;
    int b = 4 * t;
    f.te0[b] = m1_m2;     f.te1[b] = m0_m2;     f.te2[b] = m0_m1;
    f.te0[b + 1] = m1_m2; f.te1[b + 1] = m2_v0; f.te2[b + 1] = m1_v0;
    f.te0[b + 2] = m0_m2; f.te1[b + 2] = v1_m2; f.te2[b + 2] = m0_v1;
    f.te0[b + 3] = m0_m1; f.te1[b + 3] = v2_m1; f.te2[b + 3] = v2_m0;
    int8_t o = c.to[t];
    if (flip && (*flip)[t]) o = (int8_t)!o;
    f.to[b] = o;
    f.to[b + 1] = (int8_t)!o;
    f.to[b + 2] = o;
    f.to[b + 3] = (int8_t)!o;
  }
  f.eo.assign(f.ne, 0);  // unset edge orientations become false (DEC.jl:311-320)
  // propagate_points(::BinarySubdivision), :111-122, optionally projected onto a sphere.
  f.pts.resize(3 * (size_t)f.nv);
  std::copy(c.pts.begin(), c.pts.end(), f.pts.begin());
  for (int e = 0; e < c.ne; ++e) {
    double* o = &f.pts[3 * ((size_t)c.nv + e)];
    for (int k = 0; k < 3; ++k) o[k] = (c.pts[3 * (size_t)c.ev0[e] + k] + c.pts[3 * (size_t)c.ev1[e] + k]) / 2;
    if (radius > 0) {
      double n = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
      for (int k = 0; k < 3; ++k) o[k] = o[k] / n * radius;
    }
  }
  return f;
}

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

static std::unique_ptr<dec_mesh> make_mesh(const HostLevel& h, int center) {
  dec_mesh_desc d{};
  d.nv = h.nv;
  d.ne = h.ne;
  d.nt = h.nt;
  d.index_base = 0;
  d.points = h.pts.data();
  d.e_v0 = h.ev0.data();
  d.e_v1 = h.ev1.data();
  d.t_e0 = h.te0.data();
  d.t_e1 = h.te1.data();
  d.t_e2 = h.te2.data();
  d.edge_orientation = h.eo.data();
  d.tri_orientation = h.to.data();
  d.center = center;
  auto m = std::make_unique<dec_mesh>();
  m->m.build(d);
  return m;
}

// ---------------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------------
enum SweepMode { S_RESID = 0, S_JACOBI = 1, S_CHEB0 = 2, S_CHEBN = 3 };

template <class T>
struct SweepPrm {
  int mode;
  int zero_x;  // x is known to be zero: A x is skipped
  T omega;     // Jacobi
  T inv_theta; // Chebyshev first step
  T c1, c2;    // Chebyshev recurrence
};

constexpr int TB = 256;

// One smoothing sweep / residual on all panels: r = b - A x, then
//   S_RESID : out = r
//   S_JACOBI: out = x + ω D⁻¹ r
//   S_CHEB0 : d = D⁻¹ r / θ; out = x + d
//   S_CHEBN : d = c1 d + c2 D⁻¹ r; out = x + d
template <class T, int K, int W>
__global__ void __launch_bounds__(TB) k_sweep(int n, int Wr, const int32_t* __restrict__ col,
                                              const T* __restrict__ off, const T* __restrict__ diag,
                                              const T* __restrict__ dinv, const T* __restrict__ b,
                                              const T* __restrict__ x, T* __restrict__ out, T* __restrict__ d,
                                              SweepPrm<T> prm, size_t pstride) {
  const int w = W > 0 ? W : Wr;
  const int k = threadIdx.x % K;
  const size_t po = (size_t)blockIdx.y * pstride;
  const int rows_per_grid = gridDim.x * (TB / K);
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += rows_per_grid) {
    const size_t ik = po + (size_t)i * K + k;
    T r = b[ik];
    T xi = T(0);
    if (!prm.zero_x) {
      xi = x[ik];
      T acc = diag[i] * xi;
      const int32_t* c = col + (size_t)i * w;
      const T* v = off + (size_t)i * w;
#pragma unroll
      for (int s = 0; s < (W > 0 ? W : 1); ++s) {
        if (W > 0) acc += v[s] * x[po + (size_t)c[s] * K + k];
      }
      if (W == 0)
        for (int s = 0; s < w; ++s) acc += v[s] * x[po + (size_t)c[s] * K + k];
      r = r - acc;
    }
    if (prm.mode == S_RESID) {
      out[ik] = r;
    } else if (prm.mode == S_JACOBI) {
      out[ik] = xi + prm.omega * (dinv[i] * r);
    } else if (prm.mode == S_CHEB0) {
      T dn = (dinv[i] * r) * prm.inv_theta;
      d[ik] = dn;
      out[ik] = xi + dn;
    } else {
      T dn = prm.c1 * d[ik] + prm.c2 * (dinv[i] * r);
      d[ik] = dn;
      out[ik] = xi + dn;
    }
  }
}

// Restriction R = row-normalised S (make_restriction, Multigrid.jl:595-612):
// rc[i] = (1/rs_i) rf[i] + Σ_e (0.5/rs_i) rf[nc+e], rs_i = 1 + deg_i / 2.
template <class T, int K>
__global__ void __launch_bounds__(TB) k_restrict(int nc, int Wq, const int32_t* __restrict__ ridx,
                                                 const double* __restrict__ rs, const T* __restrict__ rf,
                                                 T* __restrict__ rc, size_t fstride, size_t cstride) {
  const int k = threadIdx.x % K;
  const int rows_per_grid = gridDim.x * (TB / K);
  const T* f = rf + (size_t)blockIdx.y * fstride;
  T* c = rc + (size_t)blockIdx.y * cstride;
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < nc; i += rows_per_grid) {
    const double s = rs[i];
    const T w1 = (T)(1.0 / s), wh = (T)(0.5 / s);
    T acc = w1 * f[(size_t)i * K + k];
    for (int q = 0; q < Wq; ++q) {
      int m = ridx[(size_t)i * Wq + q];
      if (m >= 0) acc += wh * f[(size_t)m * K + k];
    }
    c[(size_t)i * K + k] = acc;
  }
}

// Prolongation and correction x_f += P z (P = Sᵀ, Multigrid.jl:774).
template <class T, int K>
__global__ void __launch_bounds__(TB) k_prolong(int nf, int nc, const int32_t* __restrict__ pa,
                                                const int32_t* __restrict__ pb, const T* __restrict__ z,
                                                T* __restrict__ x, size_t fstride, size_t cstride) {
  const int k = threadIdx.x % K;
  const int rows_per_grid = gridDim.x * (TB / K);
  const T* zc = z + (size_t)blockIdx.y * cstride;
  T* xf = x + (size_t)blockIdx.y * fstride;
  for (int j = blockIdx.x * (TB / K) + threadIdx.x / K; j < nf; j += rows_per_grid) {
    T pz;
    if (j < nc) {
      pz = zc[(size_t)j * K + k];
    } else {
      int e = j - nc;
      pz = T(0.5) * zc[(size_t)pa[e] * K + k] + T(0.5) * zc[(size_t)pb[e] * K + k];
    }
    xf[(size_t)j * K + k] += pz;
  }
}

// Coarsest level: x = A⁻¹ b with the dense FP64 inverse (one CTA per panel).
template <class T, int K>
__global__ void __launch_bounds__(TB) k_coarse(int n, const double* __restrict__ ainv, const T* __restrict__ b,
                                               T* __restrict__ x, size_t pstride) {
  const T* bb = b + (size_t)blockIdx.x * pstride;
  T* xx = x + (size_t)blockIdx.x * pstride;
  for (int q = threadIdx.x; q < n * K; q += blockDim.x) {
    int i = q / K, k = q % K;
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += ainv[(size_t)i * n + j] * (double)bb[(size_t)j * K + k];
    xx[(size_t)i * K + k] = (T)s;
  }
}

// Column-major RHS block (nrhs vectors of length n) <-> panels of K.
template <class T, class S>
__global__ void k_to_panels(int n, int nrhs, int K, int npanels, const S* __restrict__ src, T* __restrict__ dst) {
  size_t total = (size_t)n * K * npanels;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    size_t p = q / ((size_t)n * K), rem = q % ((size_t)n * K);
    int i = (int)(rem / K), k = (int)(rem % K);
    int j = (int)p * K + k;
    dst[q] = j < nrhs ? (T)src[(size_t)j * n + i] : T(0);
  }
}

template <class T, class S>
__global__ void k_from_panels(int n, int nrhs, int K, const S* __restrict__ src, T* __restrict__ dst) {
  size_t total = (size_t)n * nrhs;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    int j = (int)(q / n), i = (int)(q % n);
    int p = j / K, k = j % K;
    dst[q] = (T)src[(size_t)p * n * K + (size_t)i * K + k];
  }
}

// u += (double) z on the panels.
template <class T>
__global__ void k_axpy_update(size_t total, const T* __restrict__ z, double* __restrict__ u) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    u[q] += (double)z[q];
}

// FP64 residual r = b - A u on the panels, written both as FP64 and in the inner precision T,
// with per-block partial sums of r² per right-hand side (deterministic two-stage reduction).
template <class T, int K, int W>
__global__ void __launch_bounds__(TB) k_residual64(int n, int Wr, const int32_t* __restrict__ col,
                                                   const double* __restrict__ off, const double* __restrict__ diag,
                                                   const double* __restrict__ b, const double* __restrict__ u,
                                                   T* __restrict__ rT, double* __restrict__ partial, size_t pstride) {
  const int w = W > 0 ? W : Wr;
  const int k = threadIdx.x % K;
  const size_t po = (size_t)blockIdx.y * pstride;
  double ss = 0.0;
  const int rows_per_grid = gridDim.x * (TB / K);
  for (int i = blockIdx.x * (TB / K) + threadIdx.x / K; i < n; i += rows_per_grid) {
    const size_t ik = po + (size_t)i * K + k;
    double acc = diag[i] * u[ik];
    const int32_t* c = col + (size_t)i * w;
    const double* v = off + (size_t)i * w;
    for (int s = 0; s < w; ++s) acc += v[s] * u[po + (size_t)c[s] * K + k];
    double r = b[ik] - acc;
    rT[ik] = (T)r;
    ss += r * r;
  }
  // reduce over the TB/K rows of this block for lane k
  __shared__ double sh[TB];
  sh[threadIdx.x] = ss;
  __syncthreads();
  for (int stride = TB / 2; stride >= K; stride >>= 1) {
    if (threadIdx.x < stride) sh[threadIdx.x] += sh[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < K) partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * K + threadIdx.x] = sh[threadIdx.x];
}

// Σ over blocks of the partial sums: out[p*K + k] (one thread per (panel, lane)).
__global__ void k_reduce_partials(int nblocks, int K, int npanels, const double* __restrict__ partial,
                                  double* __restrict__ out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= K * npanels) return;
  int p = q / K, k = q % K;
  double s = 0.0;
  for (int bq = 0; bq < nblocks; ++bq) s += partial[((size_t)p * nblocks + bq) * K + k];
  out[q] = s;
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

// Power iteration for λmax(D⁻¹A): y = D⁻¹ A x (single vector, FP64).
__global__ void k_dinv_a(int n, int W, const int32_t* __restrict__ col, const double* __restrict__ off,
                         const double* __restrict__ diag, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double acc = diag[i] * x[i];
    for (int s = 0; s < W; ++s) acc += off[(size_t)i * W + s] * x[col[(size_t)i * W + s]];
    y[i] = acc / diag[i];
  }
}

__global__ void k_hash_init(int n, double* x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint64_t z = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    x[i] = 0.5 + (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
}

__global__ void k_sumsq(int n, const double* __restrict__ x, double* __restrict__ out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i] * x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_scale(int n, double a, double* x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] *= a;
}

// Split layout of the level operator: diagonal + W off-diagonal slots (padding: own column,
// value 0) from the sorted ELL rows.
__global__ void k_split(int n, int Wf, const int32_t* __restrict__ fcol, const double* __restrict__ fval, int W,
                        int32_t* __restrict__ col, double* __restrict__ off, double* __restrict__ diag,
                        double* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int q = 0;
    double dg = 0.0;
    for (int s = 0; s < Wf; ++s) {
      int c = fcol[(size_t)i * Wf + s];
      if (c < 0) continue;
      if (c == i) {
        dg += fval[(size_t)i * Wf + s];
      } else if (q < W) {
        col[(size_t)i * W + q] = c;
        off[(size_t)i * W + q] = fval[(size_t)i * Wf + s];
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
// Hierarchy
// ---------------------------------------------------------------------------------------------
struct Level {
  std::unique_ptr<dec_mesh> mesh;
  std::unique_ptr<dec_op> op;  // A = L + shift I (sorted ELL, FP64): exports and parity
  int n = 0, W = 0;
  DArr<int32_t> col;
  DArr<double> off64, diag64, dinv64;
  DArr<float> off32, diag32, dinv32;
  double lmax = 0.0;
  // transfer to the next coarser level
  int nc = 0, Wq = 0;
  DArr<int32_t> ridx, pa, pb;
  DArr<double> rs;
};

template <class T>
struct LevelBufs {
  DArr<T> x, y, b, d;  // x / y ping-pong, b right-hand side, d Chebyshev direction
};

struct Workspace {
  int K = 0, npanels = 0, prec = 0;
  std::vector<LevelBufs<float>> f32;
  std::vector<LevelBufs<double>> f64;
  DArr<double> B64, U64, R64;  // finest FP64 panels
  DArr<double> partial, norms;
  DArr<double> ucm, bcm;       // column-major device copies for host-buffer solves
  int nblocks = 0;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};  // GraphKind
  int64_t launches[3] = {0, 0, 0};                          // kernel nodes per graph
  ~Workspace() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
  }
};

}  // namespace decb

struct dec_mg {
  dec_mg_options opt{};
  std::vector<decb::Level> lv;  // 0 = finest
  decb::DArr<double> ainv;      // coarsest dense inverse (FP64)
  std::map<long long, std::unique_ptr<decb::Workspace>> ws;
  std::map<long long, int> tuned;  // (nrhs, precision) -> panel width chosen by the autotuner
  cudaStream_t cap = nullptr;   // capture stream
  ~dec_mg() {
    ws.clear();
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
}

static double power_lmax(const Level& L) {
  if (L.n < 2) return 1.0;
  DArr<double> x(L.n), y(L.n), s(1);
  const int T = 256;
  k_hash_init<<<grid_for(L.n, T), T>>>(L.n, x.p);
  double lam = 1.0;
  for (int it = 0; it < 30; ++it) {
    k_sumsq<<<1, 256>>>(L.n, x.p, s.p);
    double nx = std::sqrt(s.download()[0]);
    k_scale<<<grid_for(L.n, T), T>>>(L.n, 1.0 / nx, x.p);
    k_dinv_a<<<grid_for(L.n, T), T>>>(L.n, L.W, L.col.p, L.off64.p, L.diag64.p, x.p, y.p);
    k_sumsq<<<1, 256>>>(L.n, y.p, s.p);
    lam = std::sqrt(s.download()[0]);
    std::swap(x.p, y.p);
  }
  DEC_CHECK_LAUNCH();
  return lam * 1.05;  // power iteration approaches λmax from below
}

// Dense inverse of the coarsest operator (Gauss-Jordan, partial pivoting).
static std::vector<double> dense_inverse(const dec_op& op, int n) {
  {
    auto c = op.col.download();
    auto vv = op.val64.download();
    std::vector<double> A((size_t)n * n, 0.0), Ainv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int q = 0; q < op.W; ++q) {
        int j = c[(size_t)i * op.W + q];
        if (j >= 0) A[(size_t)i * n + j] += vv[(size_t)i * op.W + q];
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
}

static void build_level_operator(Level& L, double shift) {
  L.op.reset(op_create_impl(L.mesh.get(), DEC_OP_HELMHOLTZ0, shift, DEC_F64));
  L.n = L.mesh->m.nv;
  L.W = std::max(1, L.op->W - 1);
  L.col.alloc((size_t)L.n * L.W);
  L.off64.alloc((size_t)L.n * L.W);
  L.diag64.alloc(L.n);
  L.dinv64.alloc(L.n);
  k_split<<<grid_for(L.n, 256), 256>>>(L.n, L.op->W, L.op->col.p, L.op->val64.p, L.W, L.col.p, L.off64.p,
                                       L.diag64.p, L.dinv64.p);
  DEC_CHECK_LAUNCH();
  cast_array(L.off64, L.off32);
  cast_array(L.diag64, L.diag32);
  cast_array(L.dinv64, L.dinv32);
}

// Transfers between fine level L and its coarse level (host topology of the coarse level).
static void build_transfers(Level& L, const HostLevel& c) {
  L.nc = c.nv;
  std::vector<int32_t> pa(c.ne), pb(c.ne);
  std::vector<std::vector<int32_t>> inc(c.nv);
  for (int e = 0; e < c.ne; ++e) {
    pa[e] = std::min(c.ev0[e], c.ev1[e]);
    pb[e] = std::max(c.ev0[e], c.ev1[e]);
    inc[c.ev0[e]].push_back(c.nv + e);
    if (c.ev1[e] != c.ev0[e]) inc[c.ev1[e]].push_back(c.nv + e);
  }
  int Wq = 1;
  for (auto& v : inc) Wq = std::max<int>(Wq, (int)v.size());
  std::vector<int32_t> ridx((size_t)c.nv * Wq, -1);
  std::vector<double> rs(c.nv);
  for (int i = 0; i < c.nv; ++i) {
    double s = 1.0;  // row sum of S in column order: 1.0 then 0.5 per incident edge
    for (size_t q = 0; q < inc[i].size(); ++q) {
      ridx[(size_t)i * Wq + q] = inc[i][q];
      s += 0.5;
    }
    rs[i] = s;
  }
  L.Wq = Wq;
  L.ridx.upload(ridx);
  L.rs.upload(rs);
  L.pa.upload(pa);
  L.pb.upload(pb);
}

dec_mg* mg_create(const dec_mesh_desc& cd, const dec_mg_options& o) {
  require(o.levels >= 0 && o.levels <= 12, "multigrid: levels must be in [0, 12]");
  require(o.smoother >= 0 && o.smoother <= 1, "multigrid: smoother must be DEC_SMOOTH_JACOBI or DEC_SMOOTH_CHEBYSHEV");
  require(o.pre >= 0 && o.post >= 0 && o.pre <= 16 && o.post <= 16, "multigrid: sweeps must be in [0, 16]");
  require(o.mu == 1 || o.mu == 2, "multigrid: mu must be 1 (V) or 2 (W)");
  require(o.precision == 0 || o.precision == 1, "multigrid: precision must be 0 or 1");
  require(o.cheb_ratio > 1.0, "multigrid: cheb_ratio must exceed 1");
  auto mg = std::make_unique<dec_mg>();
  mg->opt = o;
  // Coarse level from the description (orientation resolved by Mesh::build).
  std::vector<HostLevel> hl(o.levels + 1);
  {
    auto m = std::make_unique<dec_mesh>();
    dec_mesh_desc d = cd;
    d.center = o.center;
    m->m.build(d);
    HostLevel& h = hl[0];
    h.nv = m->m.nv;
    h.ne = m->m.ne;
    h.nt = m->m.nt;
    h.ev0 = m->m.h_ev0;
    h.ev1 = m->m.h_ev1;
    h.te0 = m->m.h_te0;
    h.te1 = m->m.h_te1;
    h.te2 = m->m.h_te2;
    h.eo = m->m.h_eo;
    h.to = m->m.h_to;
    h.pts = m->m.h_pts;
    mg->lv.resize(o.levels + 1);
    mg->lv[o.levels].mesh = std::move(m);
  }
  for (int l = 1; l <= o.levels; ++l) {
    std::vector<int8_t> flip;
    if (l == 1) flip = component_flips(hl[0]);
    require(4LL * hl[l - 1].nt < (1LL << 30), "multigrid: hierarchy too large");
    hl[l] = refine_level(hl[l - 1], o.project_radius, l == 1 ? &flip : nullptr);
    mg->lv[o.levels - l].mesh = make_mesh(hl[l], o.center);
  }
  for (int l = 0; l <= o.levels; ++l) {
    Level& L = mg->lv[l];
    build_level_operator(L, o.shift);
    if (l < o.levels) build_transfers(L, hl[o.levels - l - 1]);
    L.lmax = power_lmax(L);
  }
  const Level& C = mg->lv[o.levels];
  if (o.coarse_solver == 0) mg->ainv.upload(dense_inverse(*C.op, C.n));
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
  if (nv) *nv = L.mesh->m.nv;
  if (ne) *ne = L.mesh->m.ne;
  if (nt) *nt = L.mesh->m.nt;
  if (lmax) *lmax = L.lmax;
}

const dec_mesh* mg_level_mesh(const dec_mg* mg, int level) { return level_at(mg, level).mesh.get(); }
const dec_op* mg_level_op(const dec_mg* mg, int level) { return level_at(mg, level).op.get(); }

// ---------------------------------------------------------------------------------------------
// Cycle enqueue
// ---------------------------------------------------------------------------------------------
template <class T>
static const T* pick(const DArr<double>& a64, const DArr<float>& a32) {
  if constexpr (std::is_same<T, double>::value) return a64.p;
  else return a32.p;
}

template <class T, int K>
static void launch_sweep(const Level& L, const T* b, const T* x, T* out, T* d, SweepPrm<T> prm, int np,
                         cudaStream_t s) {
  size_t ps = (size_t)L.n * K;
  dim3 grid(grid_for((long long)L.n * K, TB, 8), np);
  const T* off = pick<T>(L.off64, L.off32);
  const T* dg = pick<T>(L.diag64, L.diag32);
  const T* di = pick<T>(L.dinv64, L.dinv32);
  if (L.W == 6)
    k_sweep<T, K, 6><<<grid, TB, 0, s>>>(L.n, L.W, L.col.p, off, dg, di, b, x, out, d, prm, ps);
  else
    k_sweep<T, K, 0><<<grid, TB, 0, s>>>(L.n, L.W, L.col.p, off, dg, di, b, x, out, d, prm, ps);
}

// Smooth `sweeps` times starting from x (zero if zero_x); returns the buffer holding the result.
template <class T, int K>
static T* smooth(const dec_mg& mg, const Level& L, LevelBufs<T>& B, T* x, bool zero_x, int sweeps, int np,
                 cudaStream_t s) {
  const dec_mg_options& o = mg.opt;
  T* other = (x == B.x.p) ? B.y.p : B.x.p;
  const double hi = L.lmax, lo = L.lmax / o.cheb_ratio;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2, sigma = theta / delta;
  double rho = 1 / sigma;
  for (int it = 0; it < sweeps; ++it) {
    SweepPrm<T> prm{};
    prm.zero_x = zero_x ? 1 : 0;
    if (o.smoother == DEC_SMOOTH_JACOBI) {
      prm.mode = S_JACOBI;
      prm.omega = (T)o.omega;
    } else if (it == 0) {
      prm.mode = S_CHEB0;
      prm.inv_theta = (T)(1.0 / theta);
    } else {
      double rho_new = 1 / (2 * sigma - rho);
      prm.mode = S_CHEBN;
      prm.c1 = (T)(rho_new * rho);
      prm.c2 = (T)(2 * rho_new / delta);
      rho = rho_new;
    }
    launch_sweep<T, K>(L, B.b.p, x, other, B.d.p, prm, np, s);
    std::swap(x, other);
    zero_x = false;
  }
  return x;
}

// One μ-cycle at level l on (b = B[l].b, initial guess x); returns the buffer with the result.
template <class T, int K>
static T* mu_cycle(const dec_mg& mg, std::vector<LevelBufs<T>>& bufs, int l, T* x, bool zero_x, int mu, int np,
                   cudaStream_t s) {
  const Level& L = mg.lv[l];
  LevelBufs<T>& B = bufs[l];
  const int last = (int)mg.lv.size() - 1;
  if (l == last) {
    k_coarse<T, K><<<np, TB, 0, s>>>(L.n, mg.ainv.p, B.b.p, B.x.p, (size_t)L.n * K);
    return B.x.p;
  }
  x = smooth<T, K>(mg, L, B, x, zero_x, mg.opt.pre, np, s);
  zero_x = zero_x && mg.opt.pre == 0;
  // residual into the free buffer, then restrict into the coarse right-hand side
  T* r = (x == B.x.p) ? B.y.p : B.x.p;
  SweepPrm<T> prm{};
  prm.mode = S_RESID;
  prm.zero_x = zero_x ? 1 : 0;
  launch_sweep<T, K>(L, B.b.p, x, r, nullptr, prm, np, s);
  const Level& Cl = mg.lv[l + 1];
  LevelBufs<T>& Cb = bufs[l + 1];
  dim3 gc(grid_for((long long)Cl.n * K, TB, 8), np);
  k_restrict<T, K><<<gc, TB, 0, s>>>(L.nc, L.Wq, L.ridx.p, L.rs.p, r, Cb.b.p, (size_t)L.n * K, (size_t)Cl.n * K);
  T* z = mu_cycle<T, K>(mg, bufs, l + 1, Cb.x.p, true, mu, np, s);
  if (mu > 1) z = mu_cycle<T, K>(mg, bufs, l + 1, z, false, mu - 1, np, s);
  dim3 gf(grid_for((long long)L.n * K, TB, 8), np);
  if (zero_x) {  // x is all zero: start it from the prolonged correction
    DEC_CUDA(cudaMemsetAsync(x, 0, (size_t)L.n * K * np * sizeof(T), s));
  }
  k_prolong<T, K><<<gf, TB, 0, s>>>(L.n, L.nc, L.pa.p, L.pb.p, z, x, (size_t)L.n * K, (size_t)Cl.n * K);
  return smooth<T, K>(mg, L, B, x, false, mg.opt.post, np, s);
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
static void enqueue_resid_T(dec_mg& mg, Workspace& w, cudaStream_t s, std::vector<LevelBufs<T>>& bufs) {
  const Level& F = mg.lv[0];
  const int np = w.npanels;
  const size_t total = (size_t)F.n * K * np;
  k_axpy_update<T><<<grid_for((long long)total, 256), 256, 0, s>>>(total, bufs[0].x.p, w.U64.p);
  dim3 g(w.nblocks, np);
  if (F.W == 6)
    k_residual64<T, K, 6><<<g, TB, 0, s>>>(F.n, F.W, F.col.p, F.off64.p, F.diag64.p, w.B64.p, w.U64.p, bufs[0].b.p,
                                           w.partial.p, (size_t)F.n * K);
  else
    k_residual64<T, K, 0><<<g, TB, 0, s>>>(F.n, F.W, F.col.p, F.off64.p, F.diag64.p, w.B64.p, w.U64.p, bufs[0].b.p,
                                           w.partial.p, (size_t)F.n * K);
  k_reduce_partials<<<(K * np + 127) / 128, 128, 0, s>>>(w.nblocks, K, np, w.partial.p, w.norms.p);
  DEC_CHECK_LAUNCH();
}

// Refinement step, part 2: e = V(r) from a zero initial guess, left in bufs[0].x.
template <class T, int K>
static void enqueue_vcycle_T(dec_mg& mg, Workspace& w, cudaStream_t s, std::vector<LevelBufs<T>>& bufs) {
  const size_t total = (size_t)mg.lv[0].n * K * w.npanels;
  T* e = mu_cycle<T, K>(mg, bufs, 0, bufs[0].x.p, true, mg.opt.mu, w.npanels, s);
  if (e != bufs[0].x.p)
    DEC_CUDA(cudaMemcpyAsync(bufs[0].x.p, e, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
  DEC_CHECK_LAUNCH();
}

// One plain FP64 cycle in place on (U64, B64): U <- V(U, B).
template <int K>
static void enqueue_cycle(dec_mg& mg, Workspace& w, cudaStream_t s) {
  auto& bufs = w.f64;
  const size_t total = (size_t)mg.lv[0].n * K * w.npanels;
  DEC_CUDA(cudaMemcpyAsync(bufs[0].b.p, w.B64.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DEC_CUDA(cudaMemcpyAsync(bufs[0].x.p, w.U64.p, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double* x = mu_cycle<double, K>(mg, bufs, 0, bufs[0].x.p, false, mg.opt.mu, w.npanels, s);
  DEC_CUDA(cudaMemcpyAsync(w.U64.p, x, total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DEC_CHECK_LAUNCH();
}

// Vectors a smoothing sweep reads or writes once: Jacobi b, x, out; Chebyshev b, x, d (r/w), out.
static int prm_vectors(int smoother) { return smoother == DEC_SMOOTH_JACOBI ? 3 : 5; }

enum GraphKind { G_RESID = 0, G_VCYCLE = 1, G_CYCLE = 2 };

template <int K>
static void enqueue_kind(dec_mg& mg, Workspace& w, cudaStream_t s, int kind) {
  if (kind == G_CYCLE) {
    enqueue_cycle<K>(mg, w, s);
  } else if (w.prec == 1) {
    if (kind == G_RESID) enqueue_resid_T<float, K>(mg, w, s, w.f32);
    else enqueue_vcycle_T<float, K>(mg, w, s, w.f32);
  } else {
    if (kind == G_RESID) enqueue_resid_T<double, K>(mg, w, s, w.f64);
    else enqueue_vcycle_T<double, K>(mg, w, s, w.f64);
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
    DEC_CUDA(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

static cudaGraphExec_t capture(dec_mg& mg, Workspace& w, int kind) {
  cudaGraph_t g = nullptr;
  DEC_CUDA(cudaStreamBeginCapture(mg.cap, cudaStreamCaptureModeThreadLocal));
  try {
    dispatch(mg, w, mg.cap, kind);
  } catch (...) {
    cudaStreamEndCapture(mg.cap, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  DEC_CUDA(cudaStreamEndCapture(mg.cap, &g));
  w.launches[kind] = count_kernel_nodes(g);
  cudaGraphExec_t ex = nullptr;
  cudaError_t err = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  DEC_CUDA(err);
  return ex;
}

static Workspace& workspace_k(dec_mg& mg, int nrhs, int prec, int K) {
  int np = (nrhs + K - 1) / K;
  long long key = ws_key(K, np, prec);
  auto it = mg.ws.find(key);
  if (it != mg.ws.end()) return *it->second;
  auto w = std::make_unique<Workspace>();
  w->K = K;
  w->npanels = np;
  w->prec = prec;
  const size_t total = (size_t)mg.lv[0].n * K * np;
  if (prec == 1) alloc_bufs(mg, w->f32, K, np);
  else alloc_bufs(mg, w->f64, K, np);
  w->B64.alloc(total);
  w->U64.alloc(total);
  w->nblocks = (int)std::min<long long>(2LL * num_sms(), ((long long)mg.lv[0].n * K + TB - 1) / TB);
  w->partial.alloc((size_t)w->nblocks * K * np);
  w->norms.alloc((size_t)K * np);
  DEC_CUDA(cudaMemset(w->B64.p, 0, w->B64.bytes()));
  DEC_CUDA(cudaMemset(w->U64.p, 0, w->U64.bytes()));
  auto& ref = *w;
  mg.ws[key] = std::move(w);
  return ref;
}

static Workspace& workspace(dec_mg& mg, int nrhs, int prec) {
  return workspace_k(mg, nrhs, prec, choose_k(mg, nrhs, prec));
}

void mg_cycles(dec_mg* mg, double* u, const double* b, int nrhs, int cycles, void* stream) {
  require(mg != nullptr && u != nullptr && b != nullptr, "multigrid: null argument");
  require(nrhs >= 1 && cycles >= 0, "multigrid: bad nrhs / cycles");
  cudaStream_t s = as_stream(stream);
  Workspace& w = workspace(*mg, nrhs, 0);
  const int n = mg->lv[0].n;
  const size_t total = (size_t)n * w.K * w.npanels;
  k_to_panels<double, double><<<grid_for((long long)total, 256), 256, 0, s>>>(n, nrhs, w.K, w.npanels, b, w.B64.p);
  k_to_panels<double, double><<<grid_for((long long)total, 256), 256, 0, s>>>(n, nrhs, w.K, w.npanels, u, w.U64.p);
  DEC_CHECK_LAUNCH();
  if (!w.graph[G_CYCLE]) w.graph[G_CYCLE] = capture(*mg, w, G_CYCLE);
  for (int c = 0; c < cycles; ++c) DEC_CUDA(cudaGraphLaunch(w.graph[G_CYCLE], s));
  k_from_panels<double, double><<<grid_for((long long)n * nrhs, 256), 256, 0, s>>>(n, nrhs, w.K, w.U64.p, u);
  DEC_CHECK_LAUNCH();
}

dec_status mg_solve(dec_mg* mg, double* u, const double* b, int nrhs, double rtol, int max_iters,
                    dec_solve_report* rep, void* stream, bool host_buffers) {
  require(mg != nullptr && u != nullptr && b != nullptr, "multigrid: null argument");
  require(nrhs >= 1 && max_iters >= 1 && rtol > 0, "multigrid: bad nrhs / max_iters / rtol");
  cudaStream_t s = as_stream(stream);
  Workspace& w = workspace(*mg, nrhs, mg->opt.precision);
  const int n = mg->lv[0].n;
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
    DEC_CUDA(cudaMemcpyAsync(w.ucm.p, u, (size_t)n * nrhs * 8, cudaMemcpyHostToDevice, s));
    bd = w.bcm.p;
    ud = w.ucm.p;
  }
  k_to_panels<double, double><<<grid_for((long long)total, 256), 256, 0, s>>>(n, nrhs, K, np, bd, w.B64.p);
  k_to_panels<double, double><<<grid_for((long long)total, 256), 256, 0, s>>>(n, nrhs, K, np, ud, w.U64.p);
  // the first step adds e = 0
  if (w.prec == 1) DEC_CUDA(cudaMemsetAsync(w.f32[0].x.p, 0, total * sizeof(float), s));
  else DEC_CUDA(cudaMemsetAsync(w.f64[0].x.p, 0, total * sizeof(double), s));
  DEC_CHECK_LAUNCH();
  // ||b|| per right-hand side.
  std::vector<double> bn((size_t)K * np), rn((size_t)K * np);
  {
    dim3 g(w.nblocks, np);
    switch (K) {
#define DEC_K(KK) \
  case KK: k_panel_sumsq<KK><<<g, TB, 0, s>>>(n, w.B64.p, w.partial.p, (size_t)n * KK); break;
      DEC_K(1) DEC_K(2) DEC_K(4) DEC_K(8) DEC_K(16) DEC_K(32)
#undef DEC_K
    }
    k_reduce_partials<<<(K * np + 127) / 128, 128, 0, s>>>(w.nblocks, K, np, w.partial.p, w.norms.p);
    DEC_CHECK_LAUNCH();
    DEC_CUDA(cudaMemcpyAsync(bn.data(), w.norms.p, bn.size() * 8, cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaStreamSynchronize(s));
    for (auto& x : bn) x = std::sqrt(x);
  }
  if (!w.graph[G_RESID]) w.graph[G_RESID] = capture(*mg, w, G_RESID);
  if (!w.graph[G_VCYCLE]) w.graph[G_VCYCLE] = capture(*mg, w, G_VCYCLE);
  int it = 0;
  double worst = 0.0;
  bool conv = false;
  for (;;) {
    DEC_CUDA(cudaGraphLaunch(w.graph[G_RESID], s));  // u += e; r = b - A u; norms
    DEC_CUDA(cudaMemcpyAsync(rn.data(), w.norms.p, rn.size() * 8, cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaStreamSynchronize(s));
    worst = 0.0;
    for (int j = 0; j < nrhs; ++j) {
      double rel = bn[j] > 0 ? std::sqrt(rn[j]) / bn[j] : std::sqrt(rn[j]);
      worst = std::max(worst, rel);
    }
    if (worst <= rtol) {
      conv = true;
      break;
    }
    if (it >= max_iters) break;
    DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));  // e = V(r)
    ++it;
  }
  k_from_panels<double, double><<<grid_for((long long)n * nrhs, 256), 256, 0, s>>>(n, nrhs, K, w.U64.p, ud);
  DEC_CHECK_LAUNCH();
  if (host_buffers) DEC_CUDA(cudaMemcpyAsync(u, ud, (size_t)n * nrhs * 8, cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaEventRecord(e1, s));
  DEC_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rep) {
    rep->iterations = it;
    rep->converged = conv ? 1 : 0;
    rep->max_rel_residual = worst;
    rep->seconds = ms * 1e-3;
    // to_panels x2, sumsq + reduce, residual graph per test, V-cycle graph per step, from_panels
    rep->launches = 2 + 2 + (int64_t)(it + 1) * w.launches[G_RESID] + (int64_t)it * w.launches[G_VCYCLE] + 1;
    rep->rhs_block = K;
  }
  return conv ? DEC_OK : DEC_ERR_NOT_CONVERGED;
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
      SweepPrm<T> prm{};
      prm.mode = mg.opt.smoother == DEC_SMOOTH_JACOBI ? S_JACOBI : S_CHEBN;
      prm.omega = (T)mg.opt.omega;
      prm.c1 = (T)0.5;
      prm.c2 = (T)0.25;
      launch_sweep<T, K>(L, B.b.p, B.x.p, B.y.p, B.d.p, prm, np, s);
    } else if (kernel == DEC_KERNEL_RESIDUAL) {
      dim3 g(w.nblocks, np);
      const Level& F = mg.lv[0];
      k_residual64<T, K, 0><<<g, TB, 0, s>>>(F.n, F.W, F.col.p, F.off64.p, F.diag64.p, w.B64.p, w.U64.p, bufs[0].b.p,
                                             w.partial.p, (size_t)F.n * K);
    } else if (kernel == DEC_KERNEL_RESTRICT) {
      const Level& Cl = mg.lv[level + 1];
      dim3 gc(grid_for((long long)Cl.n * K, TB, 8), np);
      k_restrict<T, K><<<gc, TB, 0, s>>>(L.nc, L.Wq, L.ridx.p, L.rs.p, B.x.p, bufs[level + 1].b.p, (size_t)L.n * K,
                                         (size_t)Cl.n * K);
    } else {
      const Level& Cl = mg.lv[level + 1];
      dim3 gf(grid_for((long long)L.n * K, TB, 8), np);
      k_prolong<T, K><<<gf, TB, 0, s>>>(L.n, L.nc, L.pa.p, L.pb.p, bufs[level + 1].x.p, B.x.p, (size_t)L.n * K,
                                        (size_t)Cl.n * K);
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
    int vecs = (prm_vectors(mg.opt.smoother));
    *bytes = mat + vecs * (double)nk * sz;
  } else if (kernel == DEC_KERNEL_RESIDUAL) {
    const Level& F = mg.lv[0];
    double mat = (double)F.n * (F.W * 12.0 + 8);
    *bytes = mat + (double)F.n * K * np * (8 + 8 + sz);
  } else if (kernel == DEC_KERNEL_RESTRICT) {
    const Level& Cl = mg.lv[level + 1];
    *bytes = (double)Cl.n * (L.Wq * 4.0 + 8) + (double)nk * sz + (double)Cl.n * K * np * sz;
  } else {
    const Level& Cl = mg.lv[level + 1];
    *bytes = (double)(L.n - L.nc) * 8.0 + (double)Cl.n * K * np * sz + 2.0 * nk * sz;
  }
}

template <int K>
static void time_kernel_K(dec_mg& mg, Workspace& w, int kernel, int level, int reps, cudaStream_t s, double* ms,
                          double* bytes) {
  if (w.prec == 1) time_kernel_T<float, K>(mg, w, w.f32, kernel, level, reps, s, ms, bytes);
  else time_kernel_T<double, K>(mg, w, w.f64, kernel, level, reps, s, ms, bytes);
}

void mg_time_kernel(dec_mg* mg, int kernel, int level, int nrhs, int reps, void* stream, double* ms, double* bytes) {
  require(mg != nullptr && ms != nullptr && bytes != nullptr, "multigrid: null argument");
  require(kernel >= 0 && kernel <= 3, "multigrid: unknown kernel");
  require(level >= 0 && level < (int)mg->lv.size() - (kernel >= 2 ? 1 : 0), "multigrid: level out of range");
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

int mg_autotune(dec_mg* mg, int nrhs, int reps, void* stream) {
  require(mg != nullptr && nrhs >= 1 && reps >= 1, "multigrid: bad autotune arguments");
  cudaStream_t s = as_stream(stream);
  const int prec = mg->opt.precision;
  int best = 0;
  double best_t = 1e300;
  for (int K = 1; K <= 32; K <<= 1) {
    if (K > 1 && (K / 2) >= nrhs) break;  // wider panels would only add padding
    Workspace& w = workspace_k(*mg, nrhs, prec, K);
    if (!w.graph[G_VCYCLE]) w.graph[G_VCYCLE] = capture(*mg, w, G_VCYCLE);
    cudaEvent_t e0, e1;
    DEC_CUDA(cudaEventCreate(&e0));
    DEC_CUDA(cudaEventCreate(&e1));
    DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
    DEC_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) DEC_CUDA(cudaGraphLaunch(w.graph[G_VCYCLE], s));
    DEC_CUDA(cudaEventRecord(e1, s));
    DEC_CUDA(cudaEventSynchronize(e1));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (t < best_t) {
      best_t = t;
      best = K;
    }
  }
  // keep only the chosen workspace for this (nrhs, precision)
  for (int K = 1; K <= 32; K <<= 1) {
    if (K == best) continue;
    int np = (nrhs + K - 1) / K;
    mg->ws.erase(ws_key(K, np, prec));
  }
  mg->tuned[((long long)nrhs << 2) | prec] = best;
  return best;
}
}  // namespace decb
