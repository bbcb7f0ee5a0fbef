// Sparse DEC operators of the FastDEC hot path as matrix-free / ELL kernels.
//
// d0 and d1 are applied straight from the incidence arrays (2 or 3 indices and packed ±1
// signs per row instead of a CSR matrix); their transposes use signed incidence lists; the
// Laplace-Beltrami / Helmholtz operator is assembled once on the GPU into a row-major ELL
// (columns sorted, diagonal included) and applied thread-per-row.  Rows accumulate in
// increasing column order, the order of the reference's CSC SpMV, and this file is compiled
// without FMA contraction, so results reproduce the reference CPU arithmetic.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>

#include "mesh.cuh"
#include "ops.cuh"
#include "tune.cuh"

namespace decb {

template <class T>
__device__ __forceinline__ T epilogue(T s, T yold, T alpha, T beta, bool has_beta) {
  if (!has_beta) return alpha == T(1) ? s : alpha * s;
  return alpha * s + beta * yold;
}

// Elementwise kernels handle kOpItems outputs per thread, spaced one block apart, with all
// loads issued before any use.
constexpr int kOpItems = 4;
constexpr int kOpThreads = 256;

// d0 x: row e = σ_e (x[∂v0] - x[∂v1]), src/FastDEC.jl:471-494, one edge per thread (FP32 rows
// whose output is not 16-byte aligned).
template <class T>
__global__ void __launch_bounds__(kOpThreads) k_d0(int ne, const int32_t* __restrict__ ev0,
                                                   const int32_t* __restrict__ ev1, const int8_t* __restrict__ es,
                                                   const T* __restrict__ x, T* __restrict__ y, T alpha, T beta,
                                                   bool hb) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    T s = (T)__ldcs(es + e) * (__ldg(x + __ldcs(ev0 + e)) - __ldg(x + __ldcs(ev1 + e)));
    y[e] = epilogue(s, hb ? y[e] : T(0), alpha, beta, hb);
  }
}

// The same rows, IT edges per thread spaced one block apart (consecutive edges stay in one warp,
// so the two gathers of edges 2e and 2e+1, which share a midpoint vertex, coalesce), every
// index load issued before any gather: the FP64 path (0.83 of the measured HBM copy bandwidth
// on icosphere L9 against 0.69 with one edge per thread).
template <class T, int IT>
__global__ void __launch_bounds__(kOpThreads) k_d0i(int ne, const int32_t* __restrict__ ev0,
                                                    const int32_t* __restrict__ ev1, const int8_t* __restrict__ es,
                                                    const T* __restrict__ x, T* __restrict__ y, T alpha, T beta,
                                                    bool hb) {
  for (long long base = (long long)blockIdx.x * kOpThreads * IT; base < ne;
       base += (long long)gridDim.x * kOpThreads * IT) {
    int i0[IT], i1[IT];
    int8_t sg[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
      const long long e = base + j * kOpThreads + threadIdx.x;
      if (e < ne) {
        i0[j] = __ldcs(ev0 + e);
        i1[j] = __ldcs(ev1 + e);
        sg[j] = __ldcs(es + e);
      }
    }
    T xa[IT], xb[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
      const long long e = base + j * kOpThreads + threadIdx.x;
      if (e < ne) {
        xa[j] = __ldg(x + i0[j]);
        xb[j] = __ldg(x + i1[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < IT; ++j) {
      const long long e = base + j * kOpThreads + threadIdx.x;
      if (e < ne) {
        const T s = (T)sg[j] * (xa[j] - xb[j]);
        y[e] = epilogue(s, hb ? y[e] : T(0), alpha, beta, hb);
      }
    }
  }
}

// d1 x: row t = τ(σ0 x[∂e0] - σ1 x[∂e1] + σ2 x[∂e2]), src/FastDEC.jl:496-524, summed in
// increasing edge order.
template <class T>
__global__ void __launch_bounds__(kOpThreads) k_d1(int nt, const int32_t* __restrict__ c0,
                                                   const int32_t* __restrict__ c1, const int32_t* __restrict__ c2,
                                                   const uint8_t* __restrict__ neg, const T* __restrict__ x,
                                                   T* __restrict__ y, T alpha, T beta, bool hb) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    uint8_t n = __ldcs(neg + t);
    T a = __ldg(x + __ldcs(c0 + t)), b = __ldg(x + __ldcs(c1 + t)), c = __ldg(x + __ldcs(c2 + t));
    T s = (n & 1) ? -a : a;
    s = s + ((n & 2) ? -b : b);
    s = s + ((n & 4) ? -c : c);
    y[t] = epilogue(s, hb ? y[t] : T(0), alpha, beta, hb);
  }
}

// Four consecutive rows per thread with 16-byte index loads, one 32-bit load of the four sign
// bytes and vector stores (y 16-byte aligned); the arithmetic per row is that of k_d0 / k_d1.
template <class T>
__device__ __forceinline__ void store4(T* y, int g, const T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    __stcs(reinterpret_cast<float4*>(y) + g, make_float4(v[0], v[1], v[2], v[3]));
  } else {
    __stcs(reinterpret_cast<double2*>(y) + 2 * g, make_double2(v[0], v[1]));
    __stcs(reinterpret_cast<double2*>(y) + 2 * g + 1, make_double2(v[2], v[3]));
  }
}

template <class T>
__global__ void __launch_bounds__(kOpThreads) k_d0v(int ne, const int32_t* __restrict__ ev0,
                                                    const int32_t* __restrict__ ev1, const int8_t* __restrict__ es,
                                                    const T* __restrict__ x, T* __restrict__ y, T alpha, T beta,
                                                    bool hb) {
  const int ng = ne / 4;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const int4 a = __ldcs(reinterpret_cast<const int4*>(ev0) + g);
    const int4 b = __ldcs(reinterpret_cast<const int4*>(ev1) + g);
    const int sg = __ldcs(reinterpret_cast<const int*>(es) + g);
    const int ia[4] = {a.x, a.y, a.z, a.w}, ib[4] = {b.x, b.y, b.z, b.w};
    T xa[4], xb[4], o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      xa[k] = __ldg(x + ia[k]);
      xb[k] = __ldg(x + ib[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const T sv = (T)(int8_t)((sg >> (8 * k)) & 0xff);
      const T sk = sv * (xa[k] - xb[k]);
      o[k] = epilogue(sk, hb ? y[4 * (size_t)g + k] : T(0), alpha, beta, hb);
    }
    store4(y, g, o);
  }
  for (int e = 4 * ng + blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const T sk = (T)es[e] * (__ldg(x + ev0[e]) - __ldg(x + ev1[e]));
    y[e] = epilogue(sk, hb ? y[e] : T(0), alpha, beta, hb);
  }
}

template <class T>
__global__ void __launch_bounds__(kOpThreads) k_d1v(int nt, const int32_t* __restrict__ c0,
                                                    const int32_t* __restrict__ c1, const int32_t* __restrict__ c2,
                                                    const uint8_t* __restrict__ neg, const T* __restrict__ x,
                                                    T* __restrict__ y, T alpha, T beta, bool hb) {
  const int ng = nt / 4;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const int4 p = __ldcs(reinterpret_cast<const int4*>(c0) + g);
    const int4 q = __ldcs(reinterpret_cast<const int4*>(c1) + g);
    const int4 r = __ldcs(reinterpret_cast<const int4*>(c2) + g);
    const unsigned ng4 = (unsigned)__ldcs(reinterpret_cast<const int*>(neg) + g);
    const int i0[4] = {p.x, p.y, p.z, p.w}, i1[4] = {q.x, q.y, q.z, q.w}, i2[4] = {r.x, r.y, r.z, r.w};
    T va[4], vb[4], vc[4], o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      va[k] = __ldg(x + i0[k]);
      vb[k] = __ldg(x + i1[k]);
      vc[k] = __ldg(x + i2[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const unsigned n = (ng4 >> (8 * k)) & 0xffu;
      T sk = (n & 1) ? -va[k] : va[k];
      sk = sk + ((n & 2) ? -vb[k] : vb[k]);
      sk = sk + ((n & 4) ? -vc[k] : vc[k]);
      o[k] = epilogue(sk, hb ? y[4 * (size_t)g + k] : T(0), alpha, beta, hb);
    }
    store4(y, g, o);
  }
  for (int t = 4 * ng + blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const uint8_t n = neg[t];
    const T a = __ldg(x + c0[t]), b = __ldg(x + c1[t]), c = __ldg(x + c2[t]);
    T sk = (n & 1) ? -a : a;
    sk = sk + ((n & 2) ? -b : b);
    sk = sk + ((n & 4) ? -c : c);
    y[t] = epilogue(sk, hb ? y[t] : T(0), alpha, beta, hb);
  }
}

// Transposed incidence rows: entry ±(j+1) contributes ±x[j].
template <class T>
__global__ void k_signed_rows(int n, const int32_t* __restrict__ ptr, const int32_t* __restrict__ ent,
                              const T* __restrict__ x, T* __restrict__ y, bool negate, T alpha, T beta, bool hb) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    T s = T(0);
    for (int q = ptr[r]; q < ptr[r + 1]; ++q) {
      int v = ent[q];
      T xv = __ldg(x + (v > 0 ? v - 1 : -v - 1));
      s += (v > 0) ? xv : -xv;
    }
    if (negate) s = -s;
    y[r] = epilogue(s, hb ? y[r] : T(0), alpha, beta, hb);
  }
}

template <class T>
__global__ void __launch_bounds__(kOpThreads) k_diag(int n, const T* __restrict__ d, const T* __restrict__ x,
                                                     T* __restrict__ y, T alpha, T beta, bool hb) {
  for (long long base = (long long)blockIdx.x * kOpThreads * kOpItems; base < n;
       base += (long long)gridDim.x * kOpThreads * kOpItems) {
    T dv[kOpItems], xv[kOpItems];
#pragma unroll
    for (int j = 0; j < kOpItems; ++j) {
      long long i = base + j * kOpThreads + threadIdx.x;
      if (i < n) {
        dv[j] = __ldcs(d + i);
        xv[j] = __ldcs(x + i);
      }
    }
#pragma unroll
    for (int j = 0; j < kOpItems; ++j) {
      long long i = base + j * kOpThreads + threadIdx.x;
      if (i < n) y[i] = epilogue(dv[j] * xv[j], hb ? y[i] : T(0), alpha, beta, hb);
    }
  }
}

// Slot-major ELL SpMV (entry (i, q) at q * n + i; padding: column -1), one thread per row: the
// q-th loads of a warp are 32 consecutive rows, one contiguous segment per slot.  All loads of a
// row are issued before the products; the row sum runs in slot (= column) order.
template <class T, int WC>
__global__ void __launch_bounds__(kOpThreads) k_ell(int n, int W, const int32_t* __restrict__ col,
                                                    const T* __restrict__ val, const T* __restrict__ x,
                                                    T* __restrict__ y, T alpha, T beta, bool hb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T s = T(0);
    if constexpr (WC > 0) {
      int c[WC];
      T v[WC], g[WC];
#pragma unroll
      for (int q = 0; q < WC; ++q) {
        c[q] = __ldcs(col + (size_t)q * n + i);
        v[q] = __ldcs(val + (size_t)q * n + i);
      }
#pragma unroll
      for (int q = 0; q < WC; ++q) g[q] = c[q] >= 0 ? __ldg(x + c[q]) : T(0);
#pragma unroll
      for (int q = 0; q < WC; ++q)
        if (c[q] >= 0) s += v[q] * g[q];
    } else {
      for (int q = 0; q < W; ++q) {
        const int j = __ldcs(col + (size_t)q * n + i);
        if (j >= 0) s += __ldcs(val + (size_t)q * n + i) * __ldg(x + j);
      }
    }
    y[i] = epilogue(s, hb ? y[i] : T(0), alpha, beta, hb);
  }
}

template <class T, int R> struct VecOf;
template <> struct VecOf<float, 2> { using t = float2; using i = int2; };
template <> struct VecOf<float, 4> { using t = float4; using i = int4; };
template <> struct VecOf<double, 2> { using t = double2; using i = int2; };

template <class V, class S, int R>
__device__ __forceinline__ void unpack(const V& v, S (&o)[R]) {
  const S* p = reinterpret_cast<const S*>(&v);
#pragma unroll
  for (int r = 0; r < R; ++r) o[r] = p[r];
}

// The same with R consecutive rows per thread (n a multiple of R): each slot's indices and values
// of the R rows come in one R-wide vector load, so a thread issues a third to a half fewer load
// instructions per row (FP32 rows are 4-byte loads, and the one-row kernel waits on the load
// queue); every row sums in slot order as above.
template <class T, int WC, int R>
__global__ void __launch_bounds__(kOpThreads) k_ell_rows(int n, const int32_t* __restrict__ col,
                                                         const T* __restrict__ val, const T* __restrict__ x,
                                                         T* __restrict__ y, T alpha, T beta, bool hb) {
  using VT = typename VecOf<T, R>::t;
  using VI = typename VecOf<T, R>::i;
  const int ng = n / R;
  for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += gridDim.x * blockDim.x) {
    int c[WC][R];
    T v[WC][R], g[WC][R];
#pragma unroll
    for (int q = 0; q < WC; ++q) {
      unpack<VI, int, R>(__ldcs(reinterpret_cast<const VI*>(col + (size_t)q * n) + gi), c[q]);
      unpack<VT, T, R>(__ldcs(reinterpret_cast<const VT*>(val + (size_t)q * n) + gi), v[q]);
    }
#pragma unroll
    for (int q = 0; q < WC; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) g[q][r] = c[q][r] >= 0 ? __ldg(x + c[q][r]) : T(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const size_t i = (size_t)gi * R + r;
      T s = T(0);
#pragma unroll
      for (int q = 0; q < WC; ++q)
        if (c[q][r] >= 0) s += v[q][r] * g[q][r];
      y[i] = epilogue(s, hb ? y[i] : T(0), alpha, beta, hb);
    }
  }
}

// Rows of L = ⋆0⁻¹ d0ᵀ ⋆1 d0 (+ shift I), the product fast_laplace_beltrami forms
// (test/Multigrid.jl:46-48): off-diagonal (i, j) = -(h_i ⋆1_e) per edge e = {i, j},
// diagonal = Σ_e h_i ⋆1_e in increasing edge order, h_i = 1 / ⋆0_i.  Columns are sorted and
// duplicate columns (parallel edges) merged in edge order.
__global__ void k_laplace_rows(int nv, int W, const int32_t* __restrict__ ptr, const int32_t* __restrict__ v2e,
                               const int32_t* __restrict__ ev0, const int32_t* __restrict__ ev1,
                               const double* __restrict__ star0, const double* __restrict__ star1, double shift,
                               int32_t* __restrict__ col, double* __restrict__ val, int* overflow) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const double h = (1 / star0[i]) * 1.0;
    double diag = 0.0;
    int cnt = 0;
    auto c = [&](int q) -> int32_t& { return col[(size_t)q * nv + i]; };  // slot-major
    auto v = [&](int q) -> double& { return val[(size_t)q * nv + i]; };
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
      int ent = v2e[q];
      int e = ent > 0 ? ent - 1 : -ent - 1;
      int j = ev0[e] == i ? ev1[e] : ev0[e];
      double w = h * star1[e];
      diag += w;
      int k = 0;
      while (k < cnt && c(k) != j) ++k;
      if (k < cnt) {
        v(k) = v(k) + (-w);
      } else if (cnt < W - 1) {
        c(cnt) = j;
        v(cnt) = 0.0 + (-w);
        ++cnt;
      } else {
        atomicExch(overflow, 1);
      }
    }
    if (shift != 0.0) diag = diag + shift;
    c(cnt) = i;
    v(cnt) = diag;
    ++cnt;
    for (int a = 1; a < cnt; ++a)
      for (int b = a; b > 0 && c(b - 1) > c(b); --b) {
        int tc = c(b); c(b) = c(b - 1); c(b - 1) = tc;
        double tv = v(b); v(b) = v(b - 1); v(b - 1) = tv;
      }
    for (int q = cnt; q < W; ++q) {
      c(q) = -1;
      v(q) = 0.0;
    }
  }
}

// ---- geometric ⋆1 (FastDEC.jl:660-716) ------------------------------------------------------
// crossdot(a, b) = |a × b| · sign((a × b)_z), +1 when that component is 0 (DEC.jl:1667-1670).
__device__ __forceinline__ double crossdot3(const double* a, const double* b) {
  const double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
  const double nrm = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
  return nrm * (c2 == 0 ? 1.0 : (c2 > 0 ? 1.0 : -1.0));
}
__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// The nine candidate entries of triangle t in the reference's push order: 0..2 the diagonal of
// its edges (∂e2, ∂e1, ∂e0), 3..8 the six ordered triples; bit k of mask set = entry present.
__constant__ int kGeoPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

__global__ void k_geo_tri(int nt, const int32_t* __restrict__ te0, const int32_t* __restrict__ te1,
                          const int32_t* __restrict__ te2, const int32_t* __restrict__ ev0,
                          const int32_t* __restrict__ ev1, const double* __restrict__ pts,
                          const double* __restrict__ tcen, double* __restrict__ coef, uint16_t* __restrict__ mask) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const int e[3] = {te2[t], te1[t], te0[t]};
    double ev[3][3], dv[3][3];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) {
        const double a = pts[3 * (size_t)ev0[e[i]] + k], b = pts[3 * (size_t)ev1[e[i]] + k];
        ev[i][k] = a - b;
        dv[i][k] = tcen[3 * (size_t)t + k] - (a + b) / 2;
      }
    for (int k = 0; k < 3; ++k) dv[1][k] *= -1;
    const double cz = ev[0][0] * dv[0][1] - ev[0][1] * dv[0][0];
    const double rel = cz == 0 ? 1.0 : (cz > 0 ? 1.0 : -1.0);
    uint16_t mk = 0;
    for (int i = 0; i < 3; ++i) {
      const double dc = crossdot3(ev[i], dv[i]);
      coef[9 * (size_t)t + i] = dc != 0.0 ? rel * dc / dot3(ev[i], ev[i]) : 0.0;
      if (dc != 0.0) mk |= (uint16_t)(1u << i);
    }
    for (int q = 0; q < 6; ++q) {
      const int p1 = kGeoPerm[q][0], p2 = kGeoPerm[q][1], p3 = kGeoPerm[q][2];
      const double diag_dot = dot3(ev[p1], dv[p1]) / dot3(ev[p1], ev[p1]);
      const double val = diag_dot * dot3(ev[p1], ev[p3]);
      coef[9 * (size_t)t + 3 + q] = val != 0.0 ? rel * val / crossdot3(ev[p2], ev[p3]) : 0.0;
      if (val != 0.0) mk |= (uint16_t)(1u << (3 + q));
    }
    mask[t] = mk;
  }
}

// Row e: the present entries (e, c) of its incident triangles in increasing triangle order and
// push order, duplicates added in that order (the first kept as is), then sorted by column;
// slot-major ELL of width W, negated when `negate` (the inverse star solves with -⋆1).
__global__ void k_geo_rows(int ne, int W, const int32_t* __restrict__ e2t_ptr, const int32_t* __restrict__ e2t,
                           const int32_t* __restrict__ te0, const int32_t* __restrict__ te1,
                           const int32_t* __restrict__ te2, const double* __restrict__ coef,
                           const uint16_t* __restrict__ mask, int negate, int32_t* __restrict__ col,
                           double* __restrict__ val, int* overflow) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    int tris[8], nts = 0;
    for (int q = e2t_ptr[e]; q < e2t_ptr[e + 1]; ++q) {
      const int t = e2t[q] / 3;
      bool seen = false;
      for (int j = 0; j < nts; ++j) seen |= tris[j] == t;
      if (!seen) {
        if (nts < 8) tris[nts++] = t;
        else atomicExch(overflow, 1);
      }
    }
    for (int a = 1; a < nts; ++a)
      for (int b = a; b > 0 && tris[b - 1] > tris[b]; --b) {
        const int x = tris[b]; tris[b] = tris[b - 1]; tris[b - 1] = x;
      }
    int cols[8];
    double vals[8];
    int cnt = 0;
    auto add = [&](int c, double v) {
      int q = 0;
      while (q < cnt && cols[q] != c) ++q;
      if (q < cnt) vals[q] = vals[q] + v;
      else if (cnt < W && cnt < 8) { cols[cnt] = c; vals[cnt] = v; ++cnt; }
      else atomicExch(overflow, 1);
    };
    for (int j = 0; j < nts; ++j) {
      const int t = tris[j];
      const int ed[3] = {te2[t], te1[t], te0[t]};
      const uint16_t mk = mask[t];
      for (int i = 0; i < 3; ++i)
        if ((mk >> i) & 1 && ed[i] == e) add(ed[i], coef[9 * (size_t)t + i]);
      for (int q = 0; q < 6; ++q)
        if ((mk >> (3 + q)) & 1 && ed[kGeoPerm[q][0]] == e) add(ed[kGeoPerm[q][1]], coef[9 * (size_t)t + 3 + q]);
    }
    for (int a = 1; a < cnt; ++a)
      for (int b = a; b > 0 && cols[b - 1] > cols[b]; --b) {
        const int tc = cols[b]; cols[b] = cols[b - 1]; cols[b - 1] = tc;
        const double tv = vals[b]; vals[b] = vals[b - 1]; vals[b - 1] = tv;
      }
    for (int q = 0; q < W; ++q) {
      col[(size_t)q * ne + e] = q < cnt ? cols[q] : -1;
      val[(size_t)q * ne + e] = q < cnt ? (negate ? -vals[q] : vals[q]) : 0.0;
    }
  }
}

constexpr int kGeoWidth = 6;  // diagonal + the two other edges of each of two incident triangles

static void assemble_geometric_star1(const Mesh& m, bool negate, int& W, DArr<int32_t>& col, DArr<double>& val) {
  W = kGeoWidth;
  col.alloc((size_t)m.ne * W);
  val.alloc((size_t)m.ne * W);
  DArr<double> coef((size_t)9 * m.nt);
  DArr<uint16_t> mask(m.nt);
  DArr<int> overflow(1);
  DEC_CUDA(cudaMemset(overflow.p, 0, sizeof(int)));
  if (m.nt)
    k_geo_tri<<<grid_for(m.nt, 128), 128>>>(m.nt, m.te0.p, m.te1.p, m.te2.p, m.ev0.p, m.ev1.p, m.pts.p,
                                             m.tri_center.p, coef.p, mask.p);
  if (m.ne)
    k_geo_rows<<<grid_for(m.ne, 128), 128>>>(m.ne, W, m.e2t_ptr.p, m.e2t.p, m.te0.p, m.te1.p, m.te2.p, coef.p,
                                              mask.p, negate ? 1 : 0, col.p, val.p, overflow.p);
  DEC_CHECK_LAUNCH();
  if (overflow.download()[0])
    throw Error(DEC_ERR_UNSUPPORTED, "geometric hodge: an edge has more incident triangles than supported");
}

// ---- inverse geometric ⋆1: Jacobi-preconditioned BiCGSTAB on A = -⋆1 (FP64) ----------------
constexpr int kKryBlocks = 256;
// partial sums of up to three dot products (a_k · b_k) per block, then a fixed-order finish
__global__ void __launch_bounds__(256) k_kry_dots(int n, int nd, const double* __restrict__ a0,
                                                  const double* __restrict__ b0, const double* __restrict__ a1,
                                                  const double* __restrict__ b1, const double* __restrict__ a2,
                                                  const double* __restrict__ b2, double* __restrict__ partial) {
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s0 += a0[i] * b0[i];
    if (nd > 1) s1 += a1[i] * b1[i];
    if (nd > 2) s2 += a2[i] * b2[i];
  }
  __shared__ double sh[3][256];
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  sh[2][threadIdx.x] = s2;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 3) partial[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_kry_finish(int nb, const double* __restrict__ partial, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k < 3) {
    double s = 0;
    for (int b = 0; b < nb; ++b) s += partial[(size_t)k * nb + b];
    out[k] = s;
  }
}

// p = r + β (p - ω v); ph = dinv ∘ p
__global__ void k_kry_p(int n, double beta, double omega, const double* __restrict__ r, const double* __restrict__ v,
                        const double* __restrict__ dinv, double* __restrict__ p, double* __restrict__ ph) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double pi = r[i] + beta * (p[i] - omega * v[i]);
    p[i] = pi;
    ph[i] = dinv[i] * pi;
  }
}
// s = r - α v; x += α ph; sh = dinv ∘ s
__global__ void k_kry_s(int n, double alpha, const double* __restrict__ r, const double* __restrict__ v,
                        const double* __restrict__ ph, const double* __restrict__ dinv, double* __restrict__ s,
                        double* __restrict__ x, double* __restrict__ shat) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double si = r[i] - alpha * v[i];
    s[i] = si;
    x[i] += alpha * ph[i];
    shat[i] = dinv[i] * si;
  }
}
// x += ω sh; r = s - ω t
__global__ void k_kry_x(int n, double omega, const double* __restrict__ s, const double* __restrict__ t,
                        const double* __restrict__ shat, double* __restrict__ x, double* __restrict__ r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += omega * shat[i];
    r[i] = s[i] - omega * t[i];
  }
}
__global__ void k_kry_sub(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] - b[i];
}
__global__ void k_ell_diag_inv(int n, int W, const int32_t* __restrict__ col, const double* __restrict__ val,
                               double* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int q = 0; q < W; ++q)
      if (col[(size_t)q * n + i] == i) d += val[(size_t)q * n + i];
    dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
  }
}
template <class S, class T>
__global__ void k_conv(size_t n, const S* __restrict__ a, T* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (T)a[i];
}
template <class T>
__global__ void k_epi(size_t n, const double* __restrict__ s, T* __restrict__ y, double alpha, double beta, int hb) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = hb ? (T)(alpha * s[i] + beta * (double)y[i]) : (T)(alpha * s[i]);
}

template <class T>
__global__ void k_cast_op(size_t n, const double* __restrict__ a, T* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (T)a[i];
}

// Inverse diagonal Hodge star: (1 / ⋆k) * (-1)^(k(2-k)), src/FastDEC.jl:732-737.
__global__ void k_inv_sign(int n, const double* __restrict__ a, double sign, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (1 / a[i]) * sign;
}

// Per-block partial sums of (b - A x)² and b² for right-hand side j = blockIdx.y (column-major
// x, b), A the FP64 ELL operator.  partial layout: [j][block] for the residual, then the same
// for b.
__global__ void __launch_bounds__(kResidThreads) k_resid_partials(int n, int W, const int32_t* __restrict__ col,
                                                                  const double* __restrict__ val,
                                                                  const double* __restrict__ x,
                                                                  const double* __restrict__ b,
                                                                  double* __restrict__ partial, int nrhs) {
  const int j = blockIdx.y;
  const double* xj = x + (size_t)j * n;
  const double* bj = b + (size_t)j * n;
  double sr = 0.0, sb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < W; ++q) {
      int c = col[(size_t)q * n + i];
      if (c >= 0) s += val[(size_t)q * n + i] * xj[c];
    }
    double r = bj[i] - s;
    sr += r * r;
    sb += bj[i] * bj[i];
  }
  __shared__ double shr[kResidThreads], shb[kResidThreads];
  shr[threadIdx.x] = sr;
  shb[threadIdx.x] = sb;
  __syncthreads();
  for (int st = kResidThreads / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      shr[threadIdx.x] += shr[threadIdx.x + st];
      shb[threadIdx.x] += shb[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[(size_t)j * gridDim.x + blockIdx.x] = shr[0];
    partial[(size_t)(nrhs + j) * gridDim.x + blockIdx.x] = shb[0];
  }
}

// dnorms[j] = sqrt(Σ partial residual), dnorms[nrhs + j] = sqrt(Σ partial b), in block order.
__global__ void k_resid_finish(int nblocks, int nrhs, const double* __restrict__ partial, double* __restrict__ dnorms) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * nrhs) return;
  double s = 0.0;
  for (int k = 0; k < nblocks; ++k) s += partial[(size_t)q * nblocks + k];
  dnorms[q] = sqrt(s);
}

void launch_residual_norms(const dec_op& op, const double* x, const double* b, int nrhs, double* partial,
                           double* dnorms, cudaStream_t s) {
  dim3 g(kResidBlocks, nrhs);
  k_resid_partials<<<g, kResidThreads, 0, s>>>((int)op.rows, op.W, op.col.p, op.val64.p, x, b, partial, nrhs);
  k_resid_finish<<<(2 * nrhs + 127) / 128, 128, 0, s>>>(kResidBlocks, nrhs, partial, dnorms);
  DEC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------------------------

static const DArr<double>& star_of(const Mesh& m, int k) {
  return k == 0 ? m.star0 : k == 1 ? m.star1 : m.star2;
}

void hodge_into(const Mesh& m, int k, bool inverse, DArr<double>& out) {
  require(k >= 0 && k <= 2, "hodge: k must be 0, 1 or 2 for a 2D complex");
  const DArr<double>& s = star_of(m, k);
  out.alloc(s.n);
  if (!s.n) return;
  if (inverse) {
    double sign = ((k * (2 - k)) % 2 == 0) ? 1.0 : -1.0;
    k_inv_sign<<<grid_for((long long)s.n, 256), 256>>>((int)s.n, s.p, sign, out.p);
  } else {
    DEC_CUDA(cudaMemcpy(out.p, s.p, s.bytes(), cudaMemcpyDeviceToDevice));
  }
  DEC_CHECK_LAUNCH();
}

void assemble_laplacian(const Mesh& m, double shift, int& W, DArr<int32_t>& col, DArr<double>& val) {
  W = m.max_v2e + 1;  // diagonal + neighbours
  col.alloc((size_t)m.nv * W);
  val.alloc((size_t)m.nv * W);
  DArr<int> overflow(1);
  DEC_CUDA(cudaMemset(overflow.p, 0, sizeof(int)));
  k_laplace_rows<<<grid_for(m.nv, 128), 128>>>(m.nv, W, m.v2e_ptr.p, m.v2e.p, m.ev0.p, m.ev1.p, m.star0.p,
                                               m.star1.p, shift, col.p, val.p, overflow.p);
  DEC_CHECK_LAUNCH();
  if (overflow.download()[0]) throw Error(DEC_ERR_INVALID_ARG, "laplacian: row width overflow");
}

template <class T>
void cast_array(const DArr<double>& a, DArr<T>& b) {
  b.alloc(a.n);
  if (a.n) k_cast_op<T><<<grid_for((long long)a.n, 256), 256>>>(a.n, a.p, b.p);
  DEC_CHECK_LAUNCH();
}
template void cast_array<float>(const DArr<double>&, DArr<float>&);

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Tuning key of the ELL apply: rows-per-thread variants exist for rows of 7 slots (the Laplacian /
// Helmholtz operators of triangle meshes), per dtype and size bucket.
static std::string ell_key(int n, int W, bool f32) {
  return std::string("ell/") + (f32 ? "f32" : "f64") + "/W" + std::to_string(W) + "/n" + std::to_string(size_bucket(n));
}

template <class T>
static void launch_ell(int n, int W, const int32_t* col, const T* val, const T* x, T* y, T a, T b, bool hb,
                       cudaStream_t s, int rows = 1) {
  if (rows > 1 && n % rows != 0) rows = 1;  // the vector variants take whole groups of rows
  if (W == 7 && rows == 2)
    k_ell_rows<T, 7, 2><<<grid_for(n, kOpThreads * 2), kOpThreads, 0, s>>>(n, col, val, x, y, a, b, hb);
  else if (W == 7 && rows == 4 && sizeof(T) == 4)
    k_ell_rows<float, 7, 4><<<grid_for(n, kOpThreads * 4), kOpThreads, 0, s>>>(
        n, col, (const float*)val, (const float*)x, (float*)y, (float)a, (float)b, hb);
  else if (W == 7) k_ell<T, 7><<<grid_for(n, kOpThreads), kOpThreads, 0, s>>>(n, W, col, val, x, y, a, b, hb);
  else if (W == 6) k_ell<T, 6><<<grid_for(n, kOpThreads), kOpThreads, 0, s>>>(n, W, col, val, x, y, a, b, hb);
  else k_ell<T, 0><<<grid_for(n, kOpThreads), kOpThreads, 0, s>>>(n, W, col, val, x, y, a, b, hb);
}

// y = alpha (-⋆1)⁻¹ x + beta y: BiCGSTAB with the Jacobi preconditioner on A = -⋆1 (stored),
// FP64, from x0 = 0 to ||b - A x|| <= 1e-14 ||b|| (or 1e-12 once it stagnates).
static void inverse_geometric_star(dec_op& op, const void* vx, void* vy, double alpha, double beta, cudaStream_t s) {
  const int n = (int)op.rows;
  if (n == 0) return;
  const size_t N = (size_t)n;
  if (op.kry.n < 10 * N + 4 * kKryBlocks) op.kry.alloc(10 * N + 4 * kKryBlocks);
  double* b = op.kry.p;
  double* x = b + N;
  double* r = x + N;
  double* rh = r + N;
  double* p = rh + N;
  double* v = p + N;
  double* ph = v + N;
  double* sv = ph + N;
  double* t = sv + N;
  double* dinv = t + N;
  double* partial = dinv + N;
  double* dres = partial + 3 * kKryBlocks;
  const unsigned g = grid_for(n, 256);
  if (op.dtype == DEC_F64) DEC_CUDA(cudaMemcpyAsync(b, vx, N * 8, cudaMemcpyDeviceToDevice, s));
  else k_conv<float, double><<<g, 256, 0, s>>>(N, (const float*)vx, b);
  k_ell_diag_inv<<<g, 256, 0, s>>>(n, op.W, op.col.p, op.val64.p, dinv);
  DEC_CUDA(cudaMemsetAsync(x, 0, N * 8, s));
  DEC_CUDA(cudaMemcpyAsync(r, b, N * 8, cudaMemcpyDeviceToDevice, s));
  DEC_CUDA(cudaMemcpyAsync(rh, b, N * 8, cudaMemcpyDeviceToDevice, s));
  DEC_CUDA(cudaMemsetAsync(p, 0, N * 8, s));
  DEC_CUDA(cudaMemsetAsync(v, 0, N * 8, s));
  double h[3];
  auto dots = [&](int nd, const double* a0, const double* b0, const double* a1, const double* b1, const double* a2,
                  const double* b2) {
    k_kry_dots<<<kKryBlocks, 256, 0, s>>>(n, nd, a0, b0, a1, b1, a2, b2, partial);
    k_kry_finish<<<1, 32, 0, s>>>(kKryBlocks, partial, dres);
    DEC_CHECK_LAUNCH();
    DEC_CUDA(cudaMemcpyAsync(h, dres, sizeof(h), cudaMemcpyDeviceToHost, s));
    DEC_CUDA(cudaStreamSynchronize(s));
  };
  dots(1, b, b, nullptr, nullptr, nullptr, nullptr);
  const double bnorm = std::sqrt(h[0]);
  double rho_old = 1, alpha_k = 1, omega = 1, best = HUGE_VAL;
  int stall = 0;
  bool done = bnorm == 0.0;
  for (int it = 0; it < 1000 && !done; ++it) {
    dots(1, rh, r, nullptr, nullptr, nullptr, nullptr);
    const double rho = h[0];
    if (rho == 0.0) break;
    const double beta_k = (rho / rho_old) * (alpha_k / omega);
    k_kry_p<<<g, 256, 0, s>>>(n, beta_k, omega, r, v, dinv, p, ph);
    launch_ell<double>(n, op.W, op.col.p, op.val64.p, ph, v, 1.0, 0.0, false, s);
    dots(1, rh, v, nullptr, nullptr, nullptr, nullptr);
    if (h[0] == 0.0) break;
    alpha_k = rho / h[0];
    k_kry_s<<<g, 256, 0, s>>>(n, alpha_k, r, v, ph, dinv, sv, x, ph);  // ph now holds dinv ∘ s
    dots(1, sv, sv, nullptr, nullptr, nullptr, nullptr);
    if (std::sqrt(h[0]) <= 1e-14 * bnorm) break;
    launch_ell<double>(n, op.W, op.col.p, op.val64.p, ph, t, 1.0, 0.0, false, s);
    dots(2, t, sv, t, t, nullptr, nullptr);
    if (h[1] == 0.0) break;
    omega = h[0] / h[1];
    k_kry_x<<<g, 256, 0, s>>>(n, omega, sv, t, ph, x, r);
    dots(1, r, r, nullptr, nullptr, nullptr, nullptr);
    const double rn = std::sqrt(h[0]);
    if (rn <= 1e-14 * bnorm) break;
    if (rn < 0.5 * best) {
      best = rn;
      stall = 0;
    } else if (++stall > 20 && rn <= 1e-12 * bnorm) {
      break;
    }
    rho_old = rho;
    if (omega == 0.0) break;
  }
  // final check on the true residual
  launch_ell<double>(n, op.W, op.col.p, op.val64.p, x, t, 1.0, 0.0, false, s);
  k_kry_sub<<<g, 256, 0, s>>>(n, b, t, r);
  dots(1, r, r, nullptr, nullptr, nullptr, nullptr);
  if (!(std::sqrt(h[0]) <= 1e-10 * std::max(bnorm, 1e-300)) && bnorm != 0.0)
    throw Error(DEC_ERR_NOT_CONVERGED, "inverse geometric hodge: the Krylov solve did not converge");
  if (op.dtype == DEC_F64) k_epi<double><<<g, 256, 0, s>>>(N, x, (double*)vy, alpha, beta, beta != 0.0);
  else k_epi<float><<<g, 256, 0, s>>>(N, x, (float*)vy, alpha, beta, beta != 0.0);
  DEC_CHECK_LAUNCH();
}

template <class T>
static void launch_op(const dec_op& op, const void* vx, void* vy, double alpha, double beta, cudaStream_t s) {
  const T* x = (const T*)vx;
  T* y = (T*)vy;
  const T a = (T)alpha, b = (T)beta;
  const bool hb = beta != 0.0;
  if (op.W == 7 && op.tuned_at != tune_version()) {  // the table changed since the last lookup
    op.tuned_at = tune_version();
    op.ell_rows = tune_get(ell_key((int)op.rows, op.W, std::is_same<T, float>::value), 1);
  }
  if (op.kind == DEC_OP_GENERAL) {  // a caller's matrix: no mesh
    const T* val = std::is_same<T, double>::value ? (const T*)op.val64.p : (const T*)op.val32.p;
    if (op.rows) launch_ell<T>((int)op.rows, op.W, op.col.p, val, x, y, a, b, hb, s, op.ell_rows);
    DEC_CHECK_LAUNCH();
    return;
  }
  const Mesh& m = *op.m;
  const int TH = 256;
  switch (op.kind) {
    case DEC_OP_D0:
      if (!m.ne) break;
      if (sizeof(T) == 8)  // measured: 4 edges a block apart beat 16-byte vectors for FP64 d0
        k_d0i<T, 4><<<grid_for(m.ne, TH * 4), TH, 0, s>>>(m.ne, m.ev0.p, m.ev1.p, m.esign.p, x, y, a, b, hb);
      else if (aligned16(y))
        k_d0v<T><<<grid_for(m.ne / 4 + 1, TH), TH, 0, s>>>(m.ne, m.ev0.p, m.ev1.p, m.esign.p, x, y, a, b, hb);
      else
        k_d0<T><<<grid_for(m.ne, TH), TH, 0, s>>>(m.ne, m.ev0.p, m.ev1.p, m.esign.p, x, y, a, b, hb);
      break;
    case DEC_OP_D1:
      if (!m.nt) break;
      if (aligned16(y))
        k_d1v<T><<<grid_for(m.nt / 4 + 1, TH), TH, 0, s>>>(m.nt, m.d1c0.p, m.d1c1.p, m.d1c2.p, m.d1neg.p, x, y, a, b,
                                                            hb);
      else
        k_d1<T><<<grid_for(m.nt, TH), TH, 0, s>>>(m.nt, m.d1c0.p, m.d1c1.p, m.d1c2.p, m.d1neg.p, x, y, a, b, hb);
      break;
    case DEC_OP_BOUNDARY1:  // ∂1 = d0ᵀ
    case DEC_OP_DUAL_D1:    // dual d(1) = -d0ᵀ
      k_signed_rows<T><<<grid_for(m.nv, TH), TH, 0, s>>>(m.nv, m.v2e_ptr.p, m.v2e.p, x, y,
                                                         op.kind == DEC_OP_DUAL_D1, a, b, hb);
      break;
    case DEC_OP_BOUNDARY2:  // ∂2 = d1ᵀ
    case DEC_OP_DUAL_D0:    // dual d(0) = d1ᵀ
      if (m.ne) k_signed_rows<T><<<grid_for(m.ne, TH), TH, 0, s>>>(m.ne, m.e2ts_ptr.p, m.e2ts.p, x, y, false, a, b, hb);
      break;
    case DEC_OP_LAPLACE0:
    case DEC_OP_HELMHOLTZ0:
    case DEC_OP_STAR1_GEOMETRIC:
    case DEC_OP_FLAT_SHARP: {
      const T* val = std::is_same<T, double>::value ? (const T*)op.val64.p : (const T*)op.val32.p;
      if (op.rows) launch_ell<T>((int)op.rows, op.W, op.col.p, val, x, y, a, b, hb, s, op.ell_rows);
      break;
    }
    case DEC_OP_INV_STAR1_GEOMETRIC:
      inverse_geometric_star(const_cast<dec_op&>(op), vx, vy, alpha, beta, s);
      break;
    default: {  // diagonal stars
      const T* d = std::is_same<T, double>::value ? (const T*)op.diag64.p : (const T*)op.diag32.p;
      int n = (int)op.rows;
      if (n) k_diag<T><<<grid_for(n, TH * kOpItems), TH, 0, s>>>(n, d, x, y, a, b, hb);
      break;
    }
  }
  DEC_CHECK_LAUNCH();
}

}  // namespace decb

using namespace decb;

dec_op* op_create_impl(dec_mesh* mh, int kind, double shift, dec_dtype dt) {
  require(mh != nullptr, "op: null mesh");
  require(dt == DEC_F64 || dt == DEC_F32, "op: dtype must be DEC_F64 or DEC_F32");
  require(kind >= DEC_OP_D0 && kind <= DEC_OP_FLAT_SHARP, "op: unknown operator kind");
  Mesh& m = mh->m;
  auto* op = new dec_op();
  op->m = &m;
  op->kind = kind;
  op->dtype = dt;
  op->shift = kind == DEC_OP_HELMHOLTZ0 ? shift : 0.0;
  try {
    switch (kind) {
      case DEC_OP_D0: op->rows = m.ne; op->cols = m.nv; break;
      case DEC_OP_D1: op->rows = m.nt; op->cols = m.ne; break;
      case DEC_OP_BOUNDARY1: case DEC_OP_DUAL_D1: op->rows = m.nv; op->cols = m.ne; break;
      case DEC_OP_BOUNDARY2: case DEC_OP_DUAL_D0: op->rows = m.ne; op->cols = m.nt; break;
      case DEC_OP_STAR0: case DEC_OP_INV_STAR0: op->rows = op->cols = m.nv; break;
      case DEC_OP_STAR1: case DEC_OP_INV_STAR1: case DEC_OP_STAR1_GEOMETRIC: case DEC_OP_INV_STAR1_GEOMETRIC:
      case DEC_OP_FLAT_SHARP:
        op->rows = op->cols = m.ne; break;
      case DEC_OP_STAR2: case DEC_OP_INV_STAR2: op->rows = op->cols = m.nt; break;
      default: op->rows = op->cols = m.nv; break;
    }
    if (kind >= DEC_OP_STAR0 && kind <= DEC_OP_INV_STAR2) {
      int k = (kind - DEC_OP_STAR0) % 3;
      hodge_into(m, k, kind >= DEC_OP_INV_STAR0, op->diag64);
      if (dt == DEC_F32) cast_array(op->diag64, op->diag32);
    } else if (kind == DEC_OP_LAPLACE0 || kind == DEC_OP_HELMHOLTZ0) {
      assemble_laplacian(m, op->shift, op->W, op->col, op->val64);
      if (dt == DEC_F32) cast_array(op->val64, op->val32);
    } else if (kind == DEC_OP_STAR1_GEOMETRIC || kind == DEC_OP_INV_STAR1_GEOMETRIC) {
      assemble_geometric_star1(m, kind == DEC_OP_INV_STAR1_GEOMETRIC, op->W, op->col, op->val64);
      if (dt == DEC_F32 && kind == DEC_OP_STAR1_GEOMETRIC) cast_array(op->val64, op->val32);
    } else if (kind == DEC_OP_FLAT_SHARP) {
      op->W = assemble_flat_sharp(m, op->col, op->val64);
      if (dt == DEC_F32) cast_array(op->val64, op->val32);
    }
    DEC_CUDA(cudaDeviceSynchronize());
  } catch (...) {
    delete op;
    throw;
  }
  return op;
}

// An n x n FP64 operator from a host CSR (columns sorted within each row), stored as the
// slot-major ELL of the Laplacian kind (apply, residual norms and export as for L + shift I).
dec_op* op_from_csr_impl(dec_mesh* mh, int n, const std::vector<int32_t>& rowptr, const std::vector<int32_t>& colind,
                         const std::vector<double>& val) {
  require((int)rowptr.size() == n + 1, "op: bad CSR");
  auto* op = new dec_op();
  op->m = mh ? &mh->m : nullptr;
  op->kind = DEC_OP_HELMHOLTZ0;
  op->dtype = DEC_F64;
  op->rows = op->cols = n;
  int W = 1;
  for (int i = 0; i < n; ++i) W = std::max(W, rowptr[i + 1] - rowptr[i]);
  op->W = W;
  std::vector<int32_t> c((size_t)W * n, -1);
  std::vector<double> v((size_t)W * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int q = rowptr[i]; q < rowptr[i + 1]; ++q) {
      c[(size_t)(q - rowptr[i]) * n + i] = colind[q];
      v[(size_t)(q - rowptr[i]) * n + i] = val[q];
    }
  try {
    op->col.upload(c);
    op->val64.upload(v);
  } catch (...) {
    delete op;
    throw;
  }
  return op;
}

// CSC (the reference's SparseMatrixCSC layout, any index base) -> 0-based CSR with each row's
// columns increasing (the order a CSC SpMV adds a row's terms in), validated.
void csc_to_csr(const dec_csc& a, std::vector<int32_t>& rp, std::vector<int32_t>& ci, std::vector<double>& vv) {
  require(a.m >= 0 && a.n >= 0, "csc: negative dimensions");
  require(a.index_base == 0 || a.index_base == 1, "csc: index_base must be 0 or 1");
  require(a.colptr != nullptr, "csc: null colptr");
  const int32_t base = a.index_base;
  require(a.colptr[0] == base, "csc: colptr[0] must equal index_base");
  for (int j = 0; j < a.n; ++j) require(a.colptr[j + 1] >= a.colptr[j], "csc: colptr must be nondecreasing");
  const int64_t nnz = (int64_t)a.colptr[a.n] - base;
  require(nnz == 0 || (a.rowval != nullptr && a.nzval != nullptr), "csc: null rowval / nzval");
  rp.assign((size_t)a.m + 1, 0);
  for (int j = 0; j < a.n; ++j)
    for (int32_t q = a.colptr[j] - base; q < a.colptr[j + 1] - base; ++q) {
      const int32_t r = a.rowval[q] - base;
      require(r >= 0 && r < a.m, "csc: row index out of range");
      require(q == a.colptr[j] - base || a.rowval[q] > a.rowval[q - 1],
              "csc: row indices must be strictly increasing within a column");
      rp[(size_t)r + 1]++;
    }
  for (int i = 0; i < a.m; ++i) rp[(size_t)i + 1] += rp[i];
  ci.resize((size_t)nnz);
  vv.resize((size_t)nnz);
  std::vector<int32_t> pos(rp.begin(), rp.end() - 1);
  for (int j = 0; j < a.n; ++j)
    for (int32_t q = a.colptr[j] - base; q < a.colptr[j + 1] - base; ++q) {
      const int32_t r = a.rowval[q] - base;
      ci[pos[r]] = j;
      vv[pos[r]++] = a.nzval[q];
    }
}

dec_op* op_create_csc_impl(const dec_csc* a, dec_dtype dt) {
  require(a != nullptr, "op: null matrix");
  require(dt == DEC_F64 || dt == DEC_F32, "op: dtype must be DEC_F64 or DEC_F32");
  std::vector<int32_t> rp, ci;
  std::vector<double> vv;
  csc_to_csr(*a, rp, ci, vv);
  const int n = a->m;
  auto* op = new dec_op();
  op->m = nullptr;
  op->kind = DEC_OP_GENERAL;
  op->dtype = dt;
  op->rows = a->m;
  op->cols = a->n;
  int W = 1;
  for (int i = 0; i < n; ++i) W = std::max(W, rp[i + 1] - rp[i]);
  op->W = W;
  std::vector<int32_t> c((size_t)W * n, -1);
  std::vector<double> v((size_t)W * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      c[(size_t)(q - rp[i]) * n + i] = ci[q];
      v[(size_t)(q - rp[i]) * n + i] = vv[q];
    }
  try {
    op->col.upload(c);
    op->val64.upload(v);
    if (dt == DEC_F32) cast_array(op->val64, op->val32);
  } catch (...) {
    delete op;
    throw;
  }
  return op;
}

void op_apply_impl(dec_op* op, const void* x, void* y, double alpha, double beta, void* stream) {
  require(op != nullptr && x != nullptr && y != nullptr, "op: null argument");
  if (op->dtype == DEC_F64) launch_op<double>(*op, x, y, alpha, beta, as_stream(stream));
  else launch_op<float>(*op, x, y, alpha, beta, as_stream(stream));
}

// Times each rows-per-thread variant of the operator's ELL apply (rows of 7 slots) on scratch
// vectors and records the fastest in the tuning table; returns the chosen rows per thread, or 0 when
// the operator's kernel has no variants.
int op_autotune_impl(dec_op* op, int reps, void* stream) {
  require(op != nullptr && reps >= 1, "op autotune: bad arguments");
  const bool ell = op->kind == DEC_OP_LAPLACE0 || op->kind == DEC_OP_HELMHOLTZ0 || op->kind == DEC_OP_GENERAL ||
                   op->kind == DEC_OP_STAR1_GEOMETRIC || op->kind == DEC_OP_FLAT_SHARP;
  if (!ell || op->W != 7 || op->rows == 0) return 0;
  cudaStream_t s = as_stream(stream);
  const bool f32 = op->dtype == DEC_F32;
  const size_t es = f32 ? 4 : 8;
  DArr<unsigned char> xb((size_t)op->cols * es), yb((size_t)op->rows * es);
  DEC_CUDA(cudaMemsetAsync(xb.p, 0, xb.bytes(), s));
  cudaEvent_t e0, e1;
  DEC_CUDA(cudaEventCreate(&e0));
  DEC_CUDA(cudaEventCreate(&e1));
  const int n = (int)op->rows;
  int best = 1;
  float best_ms = 1e30f;
  for (int rows : {1, 2, 4}) {
    if (rows == 4 && !f32) continue;  // FP64: 16-byte loads already at two rows
    auto go = [&]() {
      if (f32)
        launch_ell<float>(n, op->W, op->col.p, op->val32.p, (const float*)xb.p, (float*)yb.p, 1.f, 0.f, false, s, rows);
      else
        launch_ell<double>(n, op->W, op->col.p, op->val64.p, (const double*)xb.p, (double*)yb.p, 1.0, 0.0, false, s,
                           rows);
    };
    go();
    DEC_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) go();
    DEC_CUDA(cudaEventRecord(e1, s));
    DEC_CHECK_LAUNCH();
    DEC_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = rows;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tune_set(ell_key(n, op->W, f32), best);
  return best;
}

// CSR of the operator on the host (exact integers for d / ∂ / dual d).
void op_export_csr_impl(const dec_op* op, int64_t* nnz, int32_t* rowptr, int32_t* colind, double* val) {
  require(op != nullptr && nnz != nullptr, "op: null argument");
  static const Mesh kNoMesh;
  const Mesh& m = op->m ? *op->m : kNoMesh;
  std::vector<int32_t> rp(op->rows + 1, 0), ci;
  std::vector<double> vv;
  auto push = [&](int c, double v) { ci.push_back(c); vv.push_back(v); };
  switch (op->kind) {
    case DEC_OP_D0:
      m.ensure_host();
      for (int e = 0; e < m.ne; ++e) {
        double s = m.h_eo[e] ? 1.0 : -1.0;
        int a = m.h_ev0[e], b = m.h_ev1[e];
        if (a < b) { push(a, s); push(b, -s); } else { push(b, -s); push(a, s); }
        rp[e + 1] = (int32_t)ci.size();
      }
      break;
    case DEC_OP_D1: {
      auto c0 = m.d1c0.download(), c1 = m.d1c1.download(), c2 = m.d1c2.download();
      auto ng = m.d1neg.download();
      for (int t = 0; t < m.nt; ++t) {
        push(c0[t], (ng[t] & 1) ? -1.0 : 1.0);
        push(c1[t], (ng[t] & 2) ? -1.0 : 1.0);
        push(c2[t], (ng[t] & 4) ? -1.0 : 1.0);
        rp[t + 1] = (int32_t)ci.size();
      }
      break;
    }
    case DEC_OP_BOUNDARY1: case DEC_OP_DUAL_D1: case DEC_OP_BOUNDARY2: case DEC_OP_DUAL_D0: {
      bool vrows = op->kind == DEC_OP_BOUNDARY1 || op->kind == DEC_OP_DUAL_D1;
      auto p = vrows ? m.v2e_ptr.download() : m.e2ts_ptr.download();
      auto en = vrows ? m.v2e.download() : m.e2ts.download();
      double sg = op->kind == DEC_OP_DUAL_D1 ? -1.0 : 1.0;
      for (int64_t r = 0; r < op->rows; ++r) {
        for (int q = p[r]; q < p[r + 1]; ++q) push(en[q] > 0 ? en[q] - 1 : -en[q] - 1, en[q] > 0 ? sg : -sg);
        rp[r + 1] = (int32_t)ci.size();
      }
      break;
    }
    case DEC_OP_LAPLACE0: case DEC_OP_HELMHOLTZ0: case DEC_OP_STAR1_GEOMETRIC: case DEC_OP_FLAT_SHARP:
    case DEC_OP_GENERAL: {
      auto c = op->col.download();
      auto v = op->val64.download();
      const size_t n = (size_t)op->rows;
      for (size_t i = 0; i < n; ++i) {
        for (int q = 0; q < op->W; ++q)
          if (c[(size_t)q * n + i] >= 0) push(c[(size_t)q * n + i], v[(size_t)q * n + i]);
        rp[i + 1] = (int32_t)ci.size();
      }
      break;
    }
    case DEC_OP_INV_STAR1_GEOMETRIC:
      throw Error(DEC_ERR_UNSUPPORTED, "op: the inverse geometric hodge star is a solve, not a stored matrix");
    default: {
      auto d = op->diag64.download();
      for (int64_t i = 0; i < op->rows; ++i) {
        push((int)i, d[i]);
        rp[i + 1] = (int32_t)ci.size();
      }
    }
  }
  *nnz = (int64_t)ci.size();
  if (rowptr) std::copy(rp.begin(), rp.end(), rowptr);
  if (colind) std::copy(ci.begin(), ci.end(), colind);
  if (val) std::copy(vv.begin(), vv.end(), val);
}

void hodge_diag_impl(const dec_mesh* mh, int k, int inverse, dec_dtype dt, void* out, void* stream) {
  require(mh != nullptr && out != nullptr, "hodge: null argument");
  require(dt == DEC_F64 || dt == DEC_F32, "hodge: dtype must be DEC_F64 or DEC_F32");
  DArr<double> tmp;
  hodge_into(mh->m, k, inverse != 0, tmp);
  cudaStream_t s = as_stream(stream);
  if (dt == DEC_F64) {
    DEC_CUDA(cudaMemcpyAsync(out, tmp.p, tmp.bytes(), cudaMemcpyDeviceToDevice, s));
  } else if (tmp.n) {
    k_cast_op<float><<<grid_for((long long)tmp.n, 256), 256, 0, s>>>(tmp.n, tmp.p, (float*)out);
    DEC_CHECK_LAUNCH();
  }
  DEC_CUDA(cudaStreamSynchronize(s));  // tmp is released on return
}

void op_residual_norms_impl(dec_op* op, const double* x, const double* b, int nrhs, double* norms, double* bnorms,
                            void* stream) {
  require(op != nullptr && x != nullptr && b != nullptr && norms != nullptr, "residual norms: null argument");
  require(op->kind == DEC_OP_LAPLACE0 || op->kind == DEC_OP_HELMHOLTZ0 ||
              (op->kind == DEC_OP_GENERAL && op->rows == op->cols),
          "residual norms: the operator must be the Laplacian, a Helmholtz operator or a square matrix");
  require(nrhs >= 1 && nrhs <= 65535, "residual norms: nrhs must be in [1, 65535]");
  cudaStream_t s = as_stream(stream);
  DArr<double> partial((size_t)2 * kResidBlocks * nrhs), dn((size_t)2 * nrhs);
  launch_residual_norms(*op, x, b, nrhs, partial.p, dn.p, s);
  std::vector<double> h((size_t)2 * nrhs);
  DEC_CUDA(cudaMemcpyAsync(h.data(), dn.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaStreamSynchronize(s));
  std::copy(h.begin(), h.begin() + nrhs, norms);
  if (bnorms) std::copy(h.begin() + nrhs, h.end(), bnorms);
}

// ---- allocation-free residual norms ------------------------------------------------------------
//
// Scratch for callers that cannot allocate: the partial sums (2 * kResidBlocks per right-hand
// side) followed by the 2 * nrhs norms, in a file-scope device array.  Every device that loads
// the library holds it until the process exits.  In host code `g_resid_scratch` only names the
// symbol; its device address is looked up once per device with that device current.
static __device__ __align__(256) double g_resid_scratch[DEC_RESIDUAL_NOALLOC_SCRATCH_DOUBLES];
static_assert(DEC_RESIDUAL_NOALLOC_SCRATCH_DOUBLES ==
                  2 * kResidBlocks * DEC_RESIDUAL_NOALLOC_MAX_RHS + 2 * DEC_RESIDUAL_NOALLOC_MAX_RHS,
              "the header's scratch size must match the reduction's partial sums and norms");

#define DEC_STR_(x) #x
#define DEC_STR(x) DEC_STR_(x)

// Device address of the scratch on the current device.  A filled slot is read without a lock;
// the mutex only serialises first lookups.  The addresses are kept for the life of the process
// (a cudaDeviceReset is not followed).
static double* resid_scratch_for_current_device() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static std::atomic<double*> ptrs[kMaxDevices] = {};
  int dev = 0;
  DEC_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < kMaxDevices, "residual norms (no-alloc): device ordinal out of range");
  if (double* p = ptrs[dev].load(std::memory_order_acquire)) return p;
  std::lock_guard<std::mutex> lock(mu);
  if (ptrs[dev].load(std::memory_order_relaxed) == nullptr) {
    void* p = nullptr;
    DEC_CUDA(cudaGetSymbolAddress(&p, g_resid_scratch));
    ptrs[dev].store(static_cast<double*>(p), std::memory_order_release);
  }
  return ptrs[dev].load(std::memory_order_relaxed);
}

void op_residual_norms_noalloc_impl(dec_op* op, const double* x, const double* b, int nrhs, double* norms,
                                    double* bnorms, void* stream) {
  require(op != nullptr && x != nullptr && b != nullptr && norms != nullptr, "residual norms (no-alloc): null argument");
  require(op->kind == DEC_OP_LAPLACE0 || op->kind == DEC_OP_HELMHOLTZ0 ||
              (op->kind == DEC_OP_GENERAL && op->rows == op->cols),
          "residual norms (no-alloc): the operator must be the Laplacian, a Helmholtz operator or a square matrix");
  require(nrhs >= 1 && nrhs <= DEC_RESIDUAL_NOALLOC_MAX_RHS,
          "residual norms (no-alloc): nrhs must be in [1, " DEC_STR(DEC_RESIDUAL_NOALLOC_MAX_RHS)
          "], the size of its static scratch");
  cudaStream_t s = as_stream(stream);
  double* partial = resid_scratch_for_current_device();
  double* dn = partial + (size_t)2 * kResidBlocks * DEC_RESIDUAL_NOALLOC_MAX_RHS;
  launch_residual_norms(*op, x, b, nrhs, partial, dn, s);
  DEC_CUDA(cudaMemcpyAsync(norms, dn, (size_t)nrhs * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (bnorms) DEC_CUDA(cudaMemcpyAsync(bnorms, dn + nrhs, (size_t)nrhs * sizeof(double), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaStreamSynchronize(s));
}
