// Sparse DEC operators of the FastDEC hot path as matrix-free / ELL kernels.
//
// d0 and d1 are applied straight from the incidence arrays (2 or 3 indices and packed ±1
// signs per row instead of a CSR matrix); their transposes use signed incidence lists; the
// Laplace-Beltrami / Helmholtz operator is assembled once on the GPU into a row-major ELL
// (columns sorted, diagonal included) and applied thread-per-row.  Rows accumulate in
// increasing column order, the order of the reference's CSC SpMV, and this file is compiled
// without FMA contraction, so results reproduce the reference CPU arithmetic.
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "mesh.cuh"
#include "ops.cuh"

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

// d0 x: row e = σ_e (x[∂v0] - x[∂v1]), src/FastDEC.jl:471-494.  (One edge per thread: with
// several edges per thread these gather-bound kernels measured slower on B200.)
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
  const Mesh& m = *op.m;
  dim3 g(kResidBlocks, nrhs);
  k_resid_partials<<<g, kResidThreads, 0, s>>>(m.nv, op.W, op.col.p, op.val64.p, x, b, partial, nrhs);
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

template <class T>
static void launch_op(const dec_op& op, const void* vx, void* vy, double alpha, double beta, cudaStream_t s) {
  const Mesh& m = *op.m;
  const T* x = (const T*)vx;
  T* y = (T*)vy;
  const T a = (T)alpha, b = (T)beta;
  const bool hb = beta != 0.0;
  const int TH = 256;
  switch (op.kind) {
    case DEC_OP_D0:
      if (!m.ne) break;
      if (sizeof(T) == 4 && aligned16(y))  // FP64 measured faster one row per thread
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
    case DEC_OP_HELMHOLTZ0: {
      const T* val = std::is_same<T, double>::value ? (const T*)op.val64.p : (const T*)op.val32.p;
      if (op.W == 7)
        k_ell<T, 7><<<grid_for(m.nv, TH), TH, 0, s>>>(m.nv, op.W, op.col.p, val, x, y, a, b, hb);
      else
        k_ell<T, 0><<<grid_for(m.nv, TH), TH, 0, s>>>(m.nv, op.W, op.col.p, val, x, y, a, b, hb);
      break;
    }
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
  require(kind >= DEC_OP_D0 && kind <= DEC_OP_HELMHOLTZ0, "op: unknown operator kind");
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
      case DEC_OP_STAR1: case DEC_OP_INV_STAR1: op->rows = op->cols = m.ne; break;
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
    }
    DEC_CUDA(cudaDeviceSynchronize());
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

// CSR of the operator on the host (exact integers for d / ∂ / dual d).
void op_export_csr_impl(const dec_op* op, int64_t* nnz, int32_t* rowptr, int32_t* colind, double* val) {
  require(op != nullptr && nnz != nullptr, "op: null argument");
  const Mesh& m = *op->m;
  std::vector<int32_t> rp(op->rows + 1, 0), ci;
  std::vector<double> vv;
  auto push = [&](int c, double v) { ci.push_back(c); vv.push_back(v); };
  switch (op->kind) {
    case DEC_OP_D0:
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
    case DEC_OP_LAPLACE0: case DEC_OP_HELMHOLTZ0: {
      auto c = op->col.download();
      auto v = op->val64.download();
      for (int i = 0; i < m.nv; ++i) {
        for (int q = 0; q < op->W; ++q)
          if (c[(size_t)q * m.nv + i] >= 0) push(c[(size_t)q * m.nv + i], v[(size_t)q * m.nv + i]);
        rp[i + 1] = (int32_t)ci.size();
      }
      break;
    }
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
  require(op->kind == DEC_OP_LAPLACE0 || op->kind == DEC_OP_HELMHOLTZ0,
          "residual norms: the operator must be the Laplacian or a Helmholtz operator");
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
static __device__ __align__(256) double
    g_resid_scratch[2 * kResidBlocks * DEC_RESIDUAL_NOALLOC_MAX_RHS + 2 * DEC_RESIDUAL_NOALLOC_MAX_RHS];

static double* resid_scratch_for_current_device() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static double* ptrs[kMaxDevices] = {};
  int dev = 0;
  DEC_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < kMaxDevices, "residual norms (no-alloc): device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (ptrs[dev] == nullptr) {
    void* p = nullptr;
    DEC_CUDA(cudaGetSymbolAddress(&p, g_resid_scratch));
    ptrs[dev] = static_cast<double*>(p);
  }
  return ptrs[dev];
}

void op_residual_norms_noalloc_impl(dec_op* op, const double* x, const double* b, int nrhs, double* norms,
                                    double* bnorms, void* stream) {
  require(op != nullptr && x != nullptr && b != nullptr && norms != nullptr, "residual norms (no-alloc): null argument");
  require(op->kind == DEC_OP_LAPLACE0 || op->kind == DEC_OP_HELMHOLTZ0,
          "residual norms (no-alloc): the operator must be the Laplacian or a Helmholtz operator");
  require(nrhs >= 1 && nrhs <= DEC_RESIDUAL_NOALLOC_MAX_RHS,
          "residual norms (no-alloc): nrhs must be in [1, " + std::to_string(DEC_RESIDUAL_NOALLOC_MAX_RHS) +
              "], the size of its static scratch");
  cudaStream_t s = as_stream(stream);
  double* partial = resid_scratch_for_current_device();
  double* dn = partial + (size_t)2 * kResidBlocks * DEC_RESIDUAL_NOALLOC_MAX_RHS;
  launch_residual_norms(*op, x, b, nrhs, partial, dn, s);
  DEC_CUDA(cudaMemcpyAsync(norms, dn, (size_t)nrhs * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (bnorms) DEC_CUDA(cudaMemcpyAsync(bnorms, dn + nrhs, (size_t)nrhs * sizeof(double), cudaMemcpyDeviceToHost, s));
  DEC_CUDA(cudaStreamSynchronize(s));
}
