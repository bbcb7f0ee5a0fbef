// Wedge products of the FastDEC hot path (src/FastDEC.jl:38-401) as sm_100a kernels.
//
// Layout: every per-simplex stream (indices, coefficients, the form indexed by the output
// simplex, the output) is a separate SoA array, so a warp's loads of one stream are one
// contiguous 128-256 B segment; only the forms addressed through an index (f[∂v], α[∂e]) are
// gathered, and those come mostly from L2 because neighbouring simplices share faces.  Each
// thread handles ITEMS outputs spaced one block apart, issuing all loads before any use.
//
// The expressions mirror the reference kernels term by term and this file is compiled without
// FMA contraction, so FP64 / FP32 results reproduce the reference CPU arithmetic bit for bit
// where the reference's order of operations is kept (∧01, ∧11, the pd/dd SpMV forms).
//
// Batched application: blockIdx.y selects the form pair; each kernel offsets its form pointers
// by blockIdx.y times the form lengths, so a batch is one launch whose index and coefficient
// streams stay resident in L2 across the pairs.
#include <algorithm>

#include "mesh.cuh"
#include "tune.cuh"

namespace decb {

enum WedgeOp { W01, W10, W02, W20, W11, WDD01, WDD10, WPD01, WDP10, WPD11, WDP11 };

template <class T>
struct CoefSet {
  DArr<T> c[3];
  DArr<int32_t> idx;  // ELL indices for the sparse (pd / dd) forms; slot-major for ♭♯
  DArr<T> val;
  int width = 0;
  DArr<T> tmp;        // pd / dp (1,1): ♭♯ times the dual form, one per batched pair
};

}  // namespace decb

struct dec_wedge_plan {
  decb::Mesh* m = nullptr;
  int op = 0;
  dec_dtype dtype = DEC_F64;
  int64_t len_a = 0, len_b = 0, len_out = 0;
  decb::CoefSet<double> c64;
  decb::CoefSet<float> c32;
};

namespace decb {

constexpr int kItems = 4;
constexpr int kThreads = 256;
constexpr int kFlatSharpWidth = 6;  // ♭♯ row: the edges of the (at most two) incident triangles

// wedge_kernel_01!, FastDEC.jl:159-163: res[e] = ½ α[e] (f[∂v0 e] + f[∂v1 e]).
template <class T>
__global__ void __launch_bounds__(kThreads) k_w01(int ne, const int32_t* __restrict__ ev0,
                                                  const int32_t* __restrict__ ev1, const T* __restrict__ f,
                                                  const T* __restrict__ a, T* __restrict__ out, size_t sf, size_t sa,
                                                  size_t so) {
  f += blockIdx.y * sf;
  a += blockIdx.y * sa;
  out += blockIdx.y * so;
  const T half = T(0.5);
  for (long long base = (long long)blockIdx.x * kThreads * kItems; base < ne;
       base += (long long)gridDim.x * kThreads * kItems) {
    int i0[kItems], i1[kItems];
    T av[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      long long e = base + j * kThreads + threadIdx.x;
      if (e < ne) {
        i0[j] = __ldcs(ev0 + e);
        i1[j] = __ldcs(ev1 + e);
        av[j] = __ldcs(a + e);
      }
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      long long e = base + j * kThreads + threadIdx.x;
      if (e < ne) __stcs(out + e, half * av[j] * (__ldg(f + i0[j]) + __ldg(f + i1[j])));
    }
  }
}

// wedge_kernel_02!, FastDEC.jl:165-170, with the two dual triangles at each vertex folded into
// one coefficient w_k = (dA_2k + dA_2k+1) / area: res[t] = α[t] Σ_k w_k f[v_k].
template <class T>
__global__ void __launch_bounds__(kThreads) k_w02(int nt, const int32_t* __restrict__ tv0,
                                                  const int32_t* __restrict__ tv1, const int32_t* __restrict__ tv2,
                                                  const T* __restrict__ w0, const T* __restrict__ w1,
                                                  const T* __restrict__ w2, const T* __restrict__ f,
                                                  const T* __restrict__ a, T* __restrict__ out, size_t sf, size_t sa,
                                                  size_t so) {
  f += blockIdx.y * sf;
  a += blockIdx.y * sa;
  out += blockIdx.y * so;
  for (long long base = (long long)blockIdx.x * kThreads * kItems; base < nt;
       base += (long long)gridDim.x * kThreads * kItems) {
    int v[kItems][3];
    T w[kItems][3], av[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      long long t = base + j * kThreads + threadIdx.x;
      if (t < nt) {
        v[j][0] = __ldcs(tv0 + t);
        v[j][1] = __ldcs(tv1 + t);
        v[j][2] = __ldcs(tv2 + t);
        w[j][0] = __ldcs(w0 + t);
        w[j][1] = __ldcs(w1 + t);
        w[j][2] = __ldcs(w2 + t);
        av[j] = __ldcs(a + t);
      }
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      long long t = base + j * kThreads + threadIdx.x;
      if (t < nt)
        __stcs(out + t, av[j] * (w[j][0] * __ldg(f + v[j][0]) + w[j][1] * __ldg(f + v[j][1]) +
                                 w[j][2] * __ldg(f + v[j][2])));
    }
  }
}

// wedge_kernel_11!, FastDEC.jl:184-191.
template <class T>
__global__ void __launch_bounds__(kThreads, 4) k_w11(int nt, const int32_t* __restrict__ te0,
                                                  const int32_t* __restrict__ te1, const int32_t* __restrict__ te2,
                                                  const T* __restrict__ c0, const T* __restrict__ c1,
                                                  const T* __restrict__ c2, const T* __restrict__ a,
                                                  const T* __restrict__ b, T* __restrict__ out, size_t sa, size_t sb,
                                                  size_t so) {
  a += blockIdx.y * sa;
  b += blockIdx.y * sb;
  out += blockIdx.y * so;
  for (long long base = (long long)blockIdx.x * kThreads * kItems; base < nt;
       base += (long long)gridDim.x * kThreads * kItems) {
    int e[kItems][3];
    T c[kItems][3];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      long long t = base + j * kThreads + threadIdx.x;
      if (t < nt) {
        e[j][0] = __ldcs(te0 + t);
        e[j][1] = __ldcs(te1 + t);
        e[j][2] = __ldcs(te2 + t);
        c[j][0] = __ldcs(c0 + t);
        c[j][1] = __ldcs(c1 + t);
        c[j][2] = __ldcs(c2 + t);
      }
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      long long t = base + j * kThreads + threadIdx.x;
      if (t < nt) {
        T ae0 = __ldg(a + e[j][0]), ae1 = __ldg(a + e[j][1]), ae2 = __ldg(a + e[j][2]);
        T be0 = __ldg(b + e[j][0]), be1 = __ldg(b + e[j][1]), be2 = __ldg(b + e[j][2]);
        __stcs(out + t, (c[j][0] * (ae2 * be1 - ae1 * be2) + c[j][1] * (ae2 * be0 - ae0 * be2) +
                         c[j][2] * (ae1 * be0 - ae0 * be1)));
      }
    }
  }
}

// FP32 variants with four consecutive outputs per thread: 16-byte loads of the streamed index,
// coefficient and form arrays and 16-byte stores, the per-output expressions unchanged.  Used
// when every streamed pointer of every pair is 16-byte aligned; n4 = n / 4 vector groups, the
// remaining n % 4 outputs by the scalar expression.
__device__ __forceinline__ void f4(const float4& v, float (&o)[4]) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}
__device__ __forceinline__ void i4(const int4& v, int (&o)[4]) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}

__global__ void __launch_bounds__(kThreads) k_w01v(int ne, const int32_t* __restrict__ ev0,
                                                   const int32_t* __restrict__ ev1, const float* __restrict__ f,
                                                   const float* __restrict__ a, float* __restrict__ out, size_t sf,
                                                   size_t sa, size_t so) {
  f += blockIdx.y * sf;
  a += blockIdx.y * sa;
  out += blockIdx.y * so;
  const float half = 0.5f;
  const int n4 = ne / 4;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < n4; g += gridDim.x * kThreads) {
    int i0[4], i1[4];
    float av[4], o[4];
    i4(__ldcs(reinterpret_cast<const int4*>(ev0) + g), i0);
    i4(__ldcs(reinterpret_cast<const int4*>(ev1) + g), i1);
    f4(__ldcs(reinterpret_cast<const float4*>(a) + g), av);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = half * av[k] * (__ldg(f + i0[k]) + __ldg(f + i1[k]));
    __stcs(reinterpret_cast<float4*>(out) + g, make_float4(o[0], o[1], o[2], o[3]));
  }
  for (int e = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; e < ne; e += gridDim.x * kThreads)
    out[e] = half * a[e] * (__ldg(f + ev0[e]) + __ldg(f + ev1[e]));
}

// The same in FP64: four edges per thread, 16-byte index loads and double2 loads / stores
// (0.91 of the measured HBM bandwidth on icosphere L9 against 0.68 for k_w01).
__global__ void __launch_bounds__(kThreads) k_w01v64(int ne, const int32_t* __restrict__ ev0,
                                                     const int32_t* __restrict__ ev1, const double* __restrict__ f,
                                                     const double* __restrict__ a, double* __restrict__ out,
                                                     size_t sf, size_t sa, size_t so) {
  f += blockIdx.y * sf;
  a += blockIdx.y * sa;
  out += blockIdx.y * so;
  const double half = 0.5;
  const int n4 = ne / 4;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < n4; g += gridDim.x * kThreads) {
    int i0[4], i1[4];
    i4(__ldcs(reinterpret_cast<const int4*>(ev0) + g), i0);
    i4(__ldcs(reinterpret_cast<const int4*>(ev1) + g), i1);
    const double2 a0 = __ldcs(reinterpret_cast<const double2*>(a) + 2 * g);
    const double2 a1 = __ldcs(reinterpret_cast<const double2*>(a) + 2 * g + 1);
    const double av[4] = {a0.x, a0.y, a1.x, a1.y};
    double o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = half * av[k] * (__ldg(f + i0[k]) + __ldg(f + i1[k]));
    __stcs(reinterpret_cast<double2*>(out) + 2 * g, make_double2(o[0], o[1]));
    __stcs(reinterpret_cast<double2*>(out) + 2 * g + 1, make_double2(o[2], o[3]));
  }
  for (int e = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; e < ne; e += gridDim.x * kThreads)
    out[e] = half * a[e] * (__ldg(f + ev0[e]) + __ldg(f + ev1[e]));
}

__global__ void __launch_bounds__(kThreads) k_w02v(int nt, const int32_t* __restrict__ tv0,
                                                   const int32_t* __restrict__ tv1, const int32_t* __restrict__ tv2,
                                                   const float* __restrict__ w0, const float* __restrict__ w1,
                                                   const float* __restrict__ w2, const float* __restrict__ f,
                                                   const float* __restrict__ a, float* __restrict__ out, size_t sf,
                                                   size_t sa, size_t so) {
  f += blockIdx.y * sf;
  a += blockIdx.y * sa;
  out += blockIdx.y * so;
  const int n4 = nt / 4;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < n4; g += gridDim.x * kThreads) {
    int v0[4], v1[4], v2[4];
    float c0[4], c1[4], c2[4], av[4], o[4];
    i4(__ldcs(reinterpret_cast<const int4*>(tv0) + g), v0);
    i4(__ldcs(reinterpret_cast<const int4*>(tv1) + g), v1);
    i4(__ldcs(reinterpret_cast<const int4*>(tv2) + g), v2);
    f4(__ldcs(reinterpret_cast<const float4*>(w0) + g), c0);
    f4(__ldcs(reinterpret_cast<const float4*>(w1) + g), c1);
    f4(__ldcs(reinterpret_cast<const float4*>(w2) + g), c2);
    f4(__ldcs(reinterpret_cast<const float4*>(a) + g), av);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      o[k] = av[k] * (c0[k] * __ldg(f + v0[k]) + c1[k] * __ldg(f + v1[k]) + c2[k] * __ldg(f + v2[k]));
    __stcs(reinterpret_cast<float4*>(out) + g, make_float4(o[0], o[1], o[2], o[3]));
  }
  for (int t = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; t < nt; t += gridDim.x * kThreads)
    out[t] = a[t] * (w0[t] * __ldg(f + tv0[t]) + w1[t] * __ldg(f + tv1[t]) + w2[t] * __ldg(f + tv2[t]));
}

__global__ void __launch_bounds__(kThreads) k_w11v(int nt, const int32_t* __restrict__ te0,
                                                   const int32_t* __restrict__ te1, const int32_t* __restrict__ te2,
                                                   const float* __restrict__ cf0, const float* __restrict__ cf1,
                                                   const float* __restrict__ cf2, const float* __restrict__ a,
                                                   const float* __restrict__ b, float* __restrict__ out, size_t sa,
                                                   size_t sb, size_t so) {
  a += blockIdx.y * sa;
  b += blockIdx.y * sb;
  out += blockIdx.y * so;
  const int n4 = nt / 4;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < n4; g += gridDim.x * kThreads) {
    int e0[4], e1[4], e2[4];
    float c0[4], c1[4], c2[4], o[4];
    i4(__ldcs(reinterpret_cast<const int4*>(te0) + g), e0);
    i4(__ldcs(reinterpret_cast<const int4*>(te1) + g), e1);
    i4(__ldcs(reinterpret_cast<const int4*>(te2) + g), e2);
    f4(__ldcs(reinterpret_cast<const float4*>(cf0) + g), c0);
    f4(__ldcs(reinterpret_cast<const float4*>(cf1) + g), c1);
    f4(__ldcs(reinterpret_cast<const float4*>(cf2) + g), c2);
    // all 24 gathers of the four triangles are issued before the first product (measured: 28 against
    // 36 us per L9 application, at 44 registers and five CTAs per SM instead of 40 and six)
    float ae[3][4], be[3][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ae[0][k] = __ldg(a + e0[k]);
      ae[1][k] = __ldg(a + e1[k]);
      ae[2][k] = __ldg(a + e2[k]);
      be[0][k] = __ldg(b + e0[k]);
      be[1][k] = __ldg(b + e1[k]);
      be[2][k] = __ldg(b + e2[k]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      o[k] = (c0[k] * (ae[2][k] * be[1][k] - ae[1][k] * be[2][k]) + c1[k] * (ae[2][k] * be[0][k] - ae[0][k] * be[2][k]) +
              c2[k] * (ae[1][k] * be[0][k] - ae[0][k] * be[1][k]));
    __stcs(reinterpret_cast<float4*>(out) + g, make_float4(o[0], o[1], o[2], o[3]));
  }
  for (int t = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; t < nt; t += gridDim.x * kThreads) {
    const float ae0 = __ldg(a + te0[t]), ae1 = __ldg(a + te1[t]), ae2 = __ldg(a + te2[t]);
    const float be0 = __ldg(b + te0[t]), be1 = __ldg(b + te1[t]), be2 = __ldg(b + te2[t]);
    out[t] = (cf0[t] * (ae2 * be1 - ae1 * be2) + cf1[t] * (ae2 * be0 - ae0 * be2) + cf2[t] * (ae1 * be0 - ae0 * be1));
  }
}

// Batched FP32 ∧11, P form pairs per thread: the four triangles' edge indices and coefficients are
// loaded once (cached, so the next chunk of pairs finds them in L2) and serve pairs p0 .. p0 + P - 1,
// p0 = P blockIdx.y.  Each output keeps the single-pair expression, so every pair equals its single
// application bit for bit.  Needs the streamed pointers of every pair 16-byte aligned, like k_w11v.
template <int P>
__global__ void __launch_bounds__(kThreads) k_w11v_pairs(int nt, int count, const int32_t* __restrict__ te0,
                                                         const int32_t* __restrict__ te1,
                                                         const int32_t* __restrict__ te2,
                                                         const float* __restrict__ cf0, const float* __restrict__ cf1,
                                                         const float* __restrict__ cf2, const float* __restrict__ a,
                                                         const float* __restrict__ b, float* __restrict__ out,
                                                         size_t sa, size_t sb, size_t so) {
  const int p0 = (int)blockIdx.y * P;
  const int np = min(P, count - p0);
  a += (size_t)p0 * sa;
  b += (size_t)p0 * sb;
  out += (size_t)p0 * so;
  const int n4 = nt / 4;
  for (int g = blockIdx.x * kThreads + threadIdx.x; g < n4; g += gridDim.x * kThreads) {
    int e0[4], e1[4], e2[4];
    float c0[4], c1[4], c2[4];
    i4(__ldg(reinterpret_cast<const int4*>(te0) + g), e0);
    i4(__ldg(reinterpret_cast<const int4*>(te1) + g), e1);
    i4(__ldg(reinterpret_cast<const int4*>(te2) + g), e2);
    f4(__ldg(reinterpret_cast<const float4*>(cf0) + g), c0);
    f4(__ldg(reinterpret_cast<const float4*>(cf1) + g), c1);
    f4(__ldg(reinterpret_cast<const float4*>(cf2) + g), c2);
#pragma unroll 1
    for (int p = 0; p < np; ++p) {
      const float* ap = a + (size_t)p * sa;
      const float* bp = b + (size_t)p * sb;
      float ae[3][4], be[3][4], o[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        ae[0][k] = __ldg(ap + e0[k]);
        ae[1][k] = __ldg(ap + e1[k]);
        ae[2][k] = __ldg(ap + e2[k]);
        be[0][k] = __ldg(bp + e0[k]);
        be[1][k] = __ldg(bp + e1[k]);
        be[2][k] = __ldg(bp + e2[k]);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        o[k] = (c0[k] * (ae[2][k] * be[1][k] - ae[1][k] * be[2][k]) +
                c1[k] * (ae[2][k] * be[0][k] - ae[0][k] * be[2][k]) +
                c2[k] * (ae[1][k] * be[0][k] - ae[0][k] * be[1][k]));
      __stcs(reinterpret_cast<float4*>(out + (size_t)p * so) + g, make_float4(o[0], o[1], o[2], o[3]));
    }
  }
  for (int t = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; t < nt; t += gridDim.x * kThreads)
    for (int p = 0; p < np; ++p) {
      const float* ap = a + (size_t)p * sa;
      const float* bp = b + (size_t)p * sb;
      const float ae0 = __ldg(ap + te0[t]), ae1 = __ldg(ap + te1[t]), ae2 = __ldg(ap + te2[t]);
      const float be0 = __ldg(bp + te0[t]), be1 = __ldg(bp + te1[t]), be2 = __ldg(bp + te2[t]);
      out[(size_t)p * so + t] =
          (cf0[t] * (ae2 * be1 - ae1 * be2) + cf1[t] * (ae2 * be0 - ae0 * be2) + cf2[t] * (ae1 * be0 - ae0 * be1));
    }
}

// (M x) .* y with M a row-major ELL matrix (columns sorted, -1 = padding): the
// "matrix then elementwise product" form of the pd / dd wedges, FastDEC.jl:317-325, :381-389.
template <class T, int W>
__global__ void __launch_bounds__(kThreads) k_ell_hadamard(int n, const int32_t* __restrict__ idx,
                                                           const T* __restrict__ val, const T* __restrict__ x,
                                                           const T* __restrict__ y, T* __restrict__ out,
                                                           int mx_first, size_t sx, size_t sy, size_t so) {
  x += blockIdx.y * sx;
  y += blockIdx.y * sy;
  out += blockIdx.y * so;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    T s = T(0);
#pragma unroll
    for (int q = 0; q < W; ++q) {
      int c = __ldcs(idx + (size_t)i * W + q);
      T v = __ldcs(val + (size_t)i * W + q);
      if (c >= 0) s += v * __ldg(x + c);
    }
    T yi = __ldcs(y + i);
    __stcs(out + i, mx_first ? s * yi : yi * s);
  }
}

// ---- coefficient set-up kernels (FP64) -----------------------------------------------------

// wedge_kernel_coeffs(Val(1), Val(1)), FastDEC.jl:78-93.
__global__ void k_coef11(int nt, const int32_t* __restrict__ te0, const int32_t* __restrict__ te1,
                         const int32_t* __restrict__ te2, const int8_t* __restrict__ es,
                         const int8_t* __restrict__ ts, const double* __restrict__ area,
                         const double* __restrict__ da, double* c0, double* c1, double* c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
    double ar = (double)ts[i] * 2 * area[i];
    int e0 = te0[i], e1 = te1[i], e2 = te2[i];
    double s0 = es[e0], s1 = es[e1], s2 = es[e2];
    c0[i] = s1 * s2 * (da[i] + da[i + (size_t)nt]) / ar;
    c1[i] = s0 * s2 * (da[i + 2 * (size_t)nt] + da[i + 3 * (size_t)nt]) / ar;
    c2[i] = s0 * s1 * (da[i + 4 * (size_t)nt] + da[i + 5 * (size_t)nt]) / ar;
  }
}

// wedge_kernel_coeffs(Val(0), Val(2)), FastDEC.jl:50-62, folded per vertex.
__global__ void k_coef02(int nt, const double* __restrict__ area, const double* __restrict__ da,
                         double* w0, double* w1, double* w2) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    double ar = area[t];
    w0[t] = da[t] / ar + da[t + (size_t)nt] / ar;
    w1[t] = da[t + 2 * (size_t)nt] / ar + da[t + 3 * (size_t)nt] / ar;
    w2[t] = da[t + 4 * (size_t)nt] / ar + da[t + 5 * (size_t)nt] / ar;
  }
}

// Rows of wedge_dd_01_mat (FastDEC.jl:293-305) and wedge_pd_01_mat (:329-347).  For edge e the
// dual edges of e are its triangle-center -> edge-center dual edges in (k, t) order; the weight
// of triangle t is dual_length / Σ dual_length.
__global__ void k_rows_dd_pd(int ne, int nt, int pd, const int32_t* __restrict__ e2t_ptr,
                             const int32_t* __restrict__ e2t, const double* __restrict__ dlen,
                             const int32_t* __restrict__ ev0, const int32_t* __restrict__ ev1,
                             const int32_t* __restrict__ tv0, const int32_t* __restrict__ tv1,
                             const int32_t* __restrict__ tv2, int32_t* idx, double* val, int width,
                             int* overflow) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    int b = e2t_ptr[e], n = e2t_ptr[e + 1] - b;
    double sum = 0.0;
    for (int q = 0; q < n; ++q) {
      int tk = e2t[b + q];
      sum += dlen[(size_t)(tk % 3) * nt + tk / 3];
    }
    int cols[8];
    double vals[8];
    int cnt = 0;
    auto add = [&](int c, double v) {  // m[e, c] += v
      for (int q = 0; q < cnt; ++q)
        if (cols[q] == c) { vals[q] = vals[q] + v; return; }
      if (cnt < 8) { cols[cnt] = c; vals[cnt] = 0.0 + v; ++cnt; }
      else atomicExch(overflow, 1);
    };
    int va = ev0[e], vb = ev1[e];
    for (int q = 0; q < n; ++q) {
      int tk = e2t[b + q], t = tk / 3;
      double w = dlen[(size_t)(tk % 3) * nt + t] / sum;
      if (!pd) {
        add(t, w);
      } else {
        int tvs[3] = {tv0[t], tv1[t], tv2[t]};
        int l = -1;
        for (int k = 0; k < 3; ++k)
          if (tvs[k] != va && tvs[k] != vb) l = tvs[k];
        add(va, w * 5 / 12);
        add(vb, w * 5 / 12);
        if (l >= 0) add(l, w * 2 / 12);
      }
    }
    // sort by column (the CSC SpMV order)
    for (int i = 1; i < cnt; ++i)
      for (int j = i; j > 0 && cols[j - 1] > cols[j]; --j) {
        int tc = cols[j]; cols[j] = cols[j - 1]; cols[j - 1] = tc;
        double tv = vals[j]; vals[j] = vals[j - 1]; vals[j - 1] = tv;
      }
    if (cnt > width) { atomicExch(overflow, 1); cnt = width; }
    for (int q = 0; q < width; ++q) {
      idx[(size_t)e * width + q] = q < cnt ? cols[q] : -1;
      val[(size_t)e * width + q] = q < cnt ? vals[q] : 0.0;
    }
  }
}

template <class T>
__global__ void k_cast(size_t n, const double* __restrict__ a, T* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (T)a[i];
}

template <class T>
static void cast_into(const DArr<double>& src, DArr<T>& dst) {
  dst.alloc(src.n);
  if (src.n) k_cast<T><<<grid_for((long long)src.n, 256), 256>>>(src.n, src.p, dst.p);
  DEC_CHECK_LAUNCH();
}

// ---- ♭♯ for the primal-dual (1,1) wedges --------------------------------------------------
// ♭♯_mat = ♭(DPPFlat) * ♯(LLSDDSharp), src/DiscreteExteriorCalculus.jl:687-714, :876-909,
// :1992.  The dual edges of edge e are its triangle-center -> edge-center dual edges
// (D_edges12, (k, t) order = the e2t order); the one from triangle t is the last k with
// ∂e_k(t) = e.  Σ dual lengths per edge:
__global__ void k_fs_sumlen(int ne, int nt, const int32_t* __restrict__ e2t_ptr, const int32_t* __restrict__ e2t,
                            const double* __restrict__ dlen, double* __restrict__ sumlen) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    double sum = 0.0;
    for (int q = e2t_ptr[e]; q < e2t_ptr[e + 1]; ++q) {
      const int tk = e2t[q];
      sum += dlen[(size_t)(tk % 3) * nt + tk / 3];
    }
    sumlen[e] = sum;
  }
}

__device__ __forceinline__ int fs_slot(int t, int e, const int32_t* te0, const int32_t* te1, const int32_t* te2) {
  int k = -1;
  if (te0[t] == e) k = 0;
  if (te1[t] == e) k = 1;
  if (te2[t] == e) k = 2;
  return k;
}

// ♯ per triangle t: its edges sorted by index, and for edge i the 3-vector w_i pinv(X)[:, i]
// with X[i] = σ_i (tri center - edge center) over the three dual edges, w_i = dual length /
// Σ dual lengths of the edge; pinv(X) = B (YᵀY)⁻¹ Yᵀ, B an orthonormal basis of the triangle's
// plane and Y = X B.
__global__ void k_fs_sharp(int nt, const int32_t* __restrict__ te0, const int32_t* __restrict__ te1,
                           const int32_t* __restrict__ te2, const int32_t* __restrict__ tv0,
                           const int32_t* __restrict__ tv1, const int32_t* __restrict__ tv2,
                           const int32_t* __restrict__ ev0, const int32_t* __restrict__ ev1,
                           const int8_t* __restrict__ esign, const int8_t* __restrict__ tsign,
                           const double* __restrict__ pts, const double* __restrict__ tc,
                           const double* __restrict__ dlen, const double* __restrict__ sumlen,
                           int32_t* __restrict__ tedges, double* __restrict__ sharp) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    int es[3] = {te0[t], te1[t], te2[t]};
    for (int a = 1; a < 3; ++a)
      for (int b = a; b > 0 && es[b - 1] > es[b]; --b) {
        const int x = es[b]; es[b] = es[b - 1]; es[b - 1] = x;
      }
    double X[3][3], w[3];
    const bool to = tsign[t] > 0;
    for (int i = 0; i < 3; ++i) {
      const int e = es[i];
      const int k = fs_slot(t, e, te0, te1, te2);
      const bool ok = (k % 2 == 1) ? !to : to;
      const double sg = ((esign[e] > 0) == ok) ? 1.0 : -1.0;
      for (int c = 0; c < 3; ++c) {
        const double mid = (pts[3 * (size_t)ev0[e] + c] + pts[3 * (size_t)ev1[e] + c]) / 2;
        X[i][c] = sg * (tc[3 * (size_t)t + c] - mid);
      }
      w[i] = dlen[(size_t)k * nt + t] / sumlen[e];
      tedges[3 * (size_t)t + i] = e;
    }
    const double* q0 = pts + 3 * (size_t)tv0[t];
    const double* q1 = pts + 3 * (size_t)tv1[t];
    const double* q2 = pts + 3 * (size_t)tv2[t];
    double u[3] = {q1[0] - q0[0], q1[1] - q0[1], q1[2] - q0[2]};
    double v[3] = {q2[0] - q0[0], q2[1] - q0[1], q2[2] - q0[2]};
    const double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (int c = 0; c < 3; ++c) u[c] /= nu;
    const double uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
    for (int c = 0; c < 3; ++c) v[c] -= uv * u[c];
    const double nvv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int c = 0; c < 3; ++c) v[c] /= nvv;
    double Y[3][2];
    for (int i = 0; i < 3; ++i) {
      Y[i][0] = X[i][0] * u[0] + X[i][1] * u[1] + X[i][2] * u[2];
      Y[i][1] = X[i][0] * v[0] + X[i][1] * v[1] + X[i][2] * v[2];
    }
    double g00 = 0, g01 = 0, g11 = 0;
    for (int i = 0; i < 3; ++i) {
      g00 += Y[i][0] * Y[i][0];
      g01 += Y[i][0] * Y[i][1];
      g11 += Y[i][1] * Y[i][1];
    }
    const double det = g00 * g11 - g01 * g01;
    const double i00 = g11 / det, i01 = -g01 / det, i11 = g00 / det;
    for (int i = 0; i < 3; ++i) {
      const double c0 = i00 * Y[i][0] + i01 * Y[i][1];
      const double c1 = i01 * Y[i][0] + i11 * Y[i][1];
      for (int c = 0; c < 3; ++c) sharp[9 * (size_t)t + 3 * i + c] = w[i] * (c0 * u[c] + c1 * v[c]);
    }
  }
}

// ♭ rows and the product: row e sums, over its incident triangles t (increasing), the entries
// (e, edge i of t) = (δ_t e⃗ / Σδ) · ♯_t[i], e⃗ = σ_e (p∂v0 - p∂v1), δ_t the dual length of e in t;
// duplicate columns are added in that order, then the row is sorted by column (slot-major ELL).
__global__ void k_fs_rows(int ne, int nt, const int32_t* __restrict__ e2t_ptr, const int32_t* __restrict__ e2t,
                          const int32_t* __restrict__ te0, const int32_t* __restrict__ te1,
                          const int32_t* __restrict__ te2, const int32_t* __restrict__ ev0,
                          const int32_t* __restrict__ ev1, const int8_t* __restrict__ esign,
                          const double* __restrict__ pts, const double* __restrict__ dlen,
                          const int32_t* __restrict__ tedges, const double* __restrict__ sharp,
                          int32_t* __restrict__ idx, double* __restrict__ val, int* overflow) {
  constexpr int W = kFlatSharpWidth;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    int tris[8];
    int nts = 0;
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
    const double sg = esign[e] > 0 ? 1.0 : -1.0;
    double ev[3];
    for (int c = 0; c < 3; ++c) ev[c] = (pts[3 * (size_t)ev0[e] + c] - pts[3 * (size_t)ev1[e] + c]) * sg;
    double dels[8], dsum = 0;
    for (int j = 0; j < nts; ++j) {
      const int k = fs_slot(tris[j], e, te0, te1, te2);
      dels[j] = dlen[(size_t)k * nt + tris[j]];
      dsum += dels[j];
    }
    int cols[W];
    double vals[W];
    int cnt = 0;
    for (int j = 0; j < nts; ++j) {
      const int t = tris[j];
      double fl[3];
      for (int c = 0; c < 3; ++c) fl[c] = dels[j] * ev[c] / dsum;
      for (int i = 0; i < 3; ++i) {
        const double* sv = sharp + 9 * (size_t)t + 3 * i;
        const double x = fl[0] * sv[0] + fl[1] * sv[1] + fl[2] * sv[2];
        const int cc = tedges[3 * (size_t)t + i];
        int q = 0;
        while (q < cnt && cols[q] != cc) ++q;
        if (q < cnt) {
          vals[q] = vals[q] + x;
        } else if (cnt < W) {
          cols[cnt] = cc;
          vals[cnt] = x;
          ++cnt;
        } else {
          atomicExch(overflow, 1);
        }
      }
    }
    for (int a = 1; a < cnt; ++a)
      for (int b = a; b > 0 && cols[b - 1] > cols[b]; --b) {
        const int tcol = cols[b]; cols[b] = cols[b - 1]; cols[b - 1] = tcol;
        const double tv = vals[b]; vals[b] = vals[b - 1]; vals[b - 1] = tv;
      }
    for (int q = 0; q < W; ++q) {
      idx[(size_t)q * ne + e] = q < cnt ? cols[q] : -1;
      val[(size_t)q * ne + e] = q < cnt ? vals[q] : 0.0;
    }
  }
}

// y = ♭♯ x (slot-major ELL of width kFlatSharpWidth), row sums in column order; batched pairs
// along grid.y.
template <class T>
__global__ void __launch_bounds__(kThreads) k_fs_apply(int ne, const int32_t* __restrict__ idx,
                                                       const T* __restrict__ val, const T* __restrict__ x,
                                                       T* __restrict__ y, size_t sx, size_t sy) {
  x += blockIdx.y * sx;
  y += blockIdx.y * sy;
  constexpr int W = kFlatSharpWidth;
  for (int e = blockIdx.x * kThreads + threadIdx.x; e < ne; e += gridDim.x * kThreads) {
    int c[W];
    T v[W];
#pragma unroll
    for (int q = 0; q < W; ++q) {
      c[q] = __ldcs(idx + (size_t)q * ne + e);
      v[q] = __ldcs(val + (size_t)q * ne + e);
    }
    T s = T(0);
#pragma unroll
    for (int q = 0; q < W; ++q)
      if (c[q] >= 0) s += v[q] * __ldg(x + c[q]);
    y[e] = s;
  }
}

// ♭♯_mat(sd) (DiscreteExteriorCalculus.jl:1992; ♭ :687-714, ♯ :876-909) as a slot-major ELL of
// width kFlatSharpWidth (padding column -1); returns the width.
int assemble_flat_sharp(const Mesh& m, DArr<int32_t>& idx, DArr<double>& val) {
  const int T = 256;
  idx.alloc((size_t)m.ne * kFlatSharpWidth);
  val.alloc((size_t)m.ne * kFlatSharpWidth);
  DArr<double> sumlen(m.ne), sharp((size_t)9 * m.nt);
  DArr<int32_t> tedges((size_t)3 * m.nt);
  DArr<int> overflow(1);
  DEC_CUDA(cudaMemset(overflow.p, 0, sizeof(int)));
  if (m.ne && m.nt) {
    k_fs_sumlen<<<grid_for(m.ne, T), T>>>(m.ne, m.nt, m.e2t_ptr.p, m.e2t.p, m.dual_len_te.p, sumlen.p);
    k_fs_sharp<<<grid_for(m.nt, T), T>>>(m.nt, m.te0.p, m.te1.p, m.te2.p, m.tv0.p, m.tv1.p, m.tv2.p, m.ev0.p,
                                         m.ev1.p, m.esign.p, m.tsign.p, m.pts.p, m.tri_center.p, m.dual_len_te.p,
                                         sumlen.p, tedges.p, sharp.p);
    k_fs_rows<<<grid_for(m.ne, T), T>>>(m.ne, m.nt, m.e2t_ptr.p, m.e2t.p, m.te0.p, m.te1.p, m.te2.p, m.ev0.p,
                                        m.ev1.p, m.esign.p, m.pts.p, m.dual_len_te.p, tedges.p, sharp.p, idx.p,
                                        val.p, overflow.p);
  } else if (m.ne) {
    DEC_CUDA(cudaMemset(idx.p, 0xff, idx.bytes()));
    DEC_CUDA(cudaMemset(val.p, 0, val.bytes()));
  }
  DEC_CHECK_LAUNCH();
  if (overflow.download()[0])
    throw Error(DEC_ERR_UNSUPPORTED, "flat-sharp: an edge has more incident triangles than supported (non-manifold mesh)");
  return kFlatSharpWidth;
}

// ---- plan ---------------------------------------------------------------------------------

static void build_plan(dec_wedge_plan& P) {
  Mesh& m = *P.m;
  const int T = 256;
  CoefSet<double>& c = P.c64;
  if (P.op == W11 || P.op == WPD11 || P.op == WDP11) {
    for (auto& x : c.c) x.alloc(m.nt);
    if (m.nt)
      k_coef11<<<grid_for(m.nt, T), T>>>(m.nt, m.te0.p, m.te1.p, m.te2.p, m.esign.p, m.tsign.p, m.area.p,
                                         m.dual_area.p, c.c[0].p, c.c[1].p, c.c[2].p);
  }
  if (P.op == WPD11 || P.op == WDP11) {
    c.width = assemble_flat_sharp(m, c.idx, c.val);
  } else if (P.op == W02 || P.op == W20) {
    for (auto& x : c.c) x.alloc(m.nt);
    if (m.nt) k_coef02<<<grid_for(m.nt, T), T>>>(m.nt, m.area.p, m.dual_area.p, c.c[0].p, c.c[1].p, c.c[2].p);
  } else if (P.op >= WDD01 && P.op <= WDP10) {
    bool pd = (P.op == WPD01 || P.op == WDP10);
    c.width = pd ? 4 : 2;
    c.idx.alloc((size_t)m.ne * c.width);
    c.val.alloc((size_t)m.ne * c.width);
    DArr<int> overflow(1);
    DEC_CUDA(cudaMemset(overflow.p, 0, sizeof(int)));
    if (m.ne)
      k_rows_dd_pd<<<grid_for(m.ne, T), T>>>(m.ne, m.nt, pd, m.e2t_ptr.p, m.e2t.p, m.dual_len_te.p, m.ev0.p,
                                             m.ev1.p, m.tv0.p, m.tv1.p, m.tv2.p, c.idx.p, c.val.p, c.width,
                                             overflow.p);
    DEC_CHECK_LAUNCH();
    int of = overflow.download()[0];
    if (of) throw Error(DEC_ERR_UNSUPPORTED, "wedge: an edge has more incident triangles than supported (non-manifold mesh)");
  }
  DEC_CHECK_LAUNCH();
  if (P.dtype == DEC_F32) {
    for (int k = 0; k < 3; ++k) cast_into(c.c[k], P.c32.c[k]);
    if (c.width) {
      cast_into(c.val, P.c32.val);
      P.c32.width = c.width;
    }
  }
  DEC_CUDA(cudaDeviceSynchronize());
}

// The batched FP32 ∧11's pairs per thread (k_w11v_pairs), per triangle-count bucket.
static std::string w11_pairs_key(int nt) { return "w11pairs/f32/n" + std::to_string(size_bucket(nt)); }
constexpr int kW11PairsDefault = 4;

static void launch_w11v_pairs(int pairs, const Mesh& m, const CoefSet<float>& c, const float* a, const float* b,
                              float* o, size_t sa, size_t sb, size_t so, int cnt, cudaStream_t s) {
  auto go = [&](auto kernel, int per) {
    const dim3 grid(grid_for(m.nt / 4 + 1, kThreads), (unsigned)((cnt + per - 1) / per));
    kernel<<<grid, kThreads, 0, s>>>(m.nt, cnt, m.te0.p, m.te1.p, m.te2.p, c.c[0].p, c.c[1].p, c.c[2].p, a, b, o, sa,
                                     sb, so);
  };
  switch (pairs) {
    case 2: go(k_w11v_pairs<2>, 2); break;
    case 4: go(k_w11v_pairs<4>, 4); break;
    case 8: go(k_w11v_pairs<8>, 8); break;
    case 16: go(k_w11v_pairs<16>, 16); break;
    default: go(k_w11v_pairs<1>, 1); break;
  }
}

// `count` form pairs (a, b, out consecutive with the plan's lengths), one launch per kind.  pairs:
// the batched FP32 ∧11's pairs per thread (0 = the tuning table's choice).
template <class T>
static void launch_plan(dec_wedge_plan& P, const CoefSet<T>& c, const void* va, const void* vb, void* vo, int count,
                        cudaStream_t s, int pairs = 0) {
  Mesh& m = *P.m;
  const T* a = (const T*)va;
  const T* b = (const T*)vb;
  T* o = (T*)vo;
  const size_t sa = P.len_a, sb = P.len_b, so = P.len_out;
  const int* idx = P.c64.idx.p;
  // the batch is grid.y (at most 65,535 pairs per launch) and every pair keeps the single-pair
  // grid: CTAs are dispatched x-fastest, so a few pairs at a time stream through L2 and each form
  // value shared by neighbouring simplices is read from DRAM once
  auto grid2 = [&](long long n, int per, int cnt) { return dim3(grid_for(n, per), (unsigned)cnt); };
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  // the FP32 vector kernels need every pair's streamed pointers 16-byte aligned
  const bool vec = sizeof(T) == 4 && al16(va) && al16(vb) && al16(vo) && (count == 1 || (sa % 4 == 0 && sb % 4 == 0 && so % 4 == 0));
  // FP64 double2 access: every pair's forms 16-byte aligned
  const bool vec64 = sizeof(T) == 8 && al16(va) && al16(vb) && al16(vo) &&
                     (count == 1 || (sa % 2 == 0 && sb % 2 == 0 && so % 2 == 0));
  for (int done = 0; done < count;) {
    const int cnt = std::min(count - done, 65535);
    const T* ab = a + (size_t)done * sa;
    const T* bb = b + (size_t)done * sb;
    T* ob = o + (size_t)done * so;
    switch (P.op) {
      case W01:
      case W10: {
        const T* f = P.op == W01 ? ab : bb;
        const T* al = P.op == W01 ? bb : ab;
        const size_t sf = P.op == W01 ? sa : sb, sl = P.op == W01 ? sb : sa;
        if (!m.ne) break;
        if constexpr (sizeof(T) == 4) {
          if (vec) {
            k_w01v<<<grid2(m.ne / 4 + 1, kThreads, cnt), kThreads, 0, s>>>(m.ne, m.ev0.p, m.ev1.p, f, al, ob, sf, sl,
                                                                             so);
            break;
          }
        }
        if constexpr (sizeof(T) == 8) {
          if (vec64) {
            k_w01v64<<<grid2(m.ne / 4 + 1, kThreads, cnt), kThreads, 0, s>>>(m.ne, m.ev0.p, m.ev1.p, f, al, ob, sf,
                                                                              sl, so);
            break;
          }
        }
        k_w01<T><<<grid2(m.ne, kThreads * kItems, cnt), kThreads, 0, s>>>(m.ne, m.ev0.p, m.ev1.p, f, al, ob, sf, sl,
                                                                            so);
        break;
      }
      case W02:
      case W20: {
        const T* f = P.op == W02 ? ab : bb;
        const T* al = P.op == W02 ? bb : ab;
        const size_t sf = P.op == W02 ? sa : sb, sl = P.op == W02 ? sb : sa;
        if (!m.nt) break;
        if constexpr (sizeof(T) == 4) {
          if (vec) {
            k_w02v<<<grid2(m.nt / 4 + 1, kThreads, cnt), kThreads, 0, s>>>(m.nt, m.tv0.p, m.tv1.p, m.tv2.p, c.c[0].p,
                                                                             c.c[1].p, c.c[2].p, f, al, ob, sf, sl, so);
            break;
          }
        }
        k_w02<T><<<grid2(m.nt, kThreads * kItems, cnt), kThreads, 0, s>>>(m.nt, m.tv0.p, m.tv1.p, m.tv2.p, c.c[0].p,
                                                                            c.c[1].p, c.c[2].p, f, al, ob, sf, sl, so);
        break;
      }
      case W11:
        if (!m.nt) break;
        if constexpr (sizeof(T) == 4) {
          if (vec && cnt > 1) {
            const int per = pairs > 0 ? pairs : tune_get(w11_pairs_key(m.nt), kW11PairsDefault);
            launch_w11v_pairs(per, m, c, ab, bb, ob, sa, sb, so, cnt, s);
            break;
          }
          if (vec) {
            k_w11v<<<grid2(m.nt / 4 + 1, kThreads, cnt), kThreads, 0, s>>>(m.nt, m.te0.p, m.te1.p, m.te2.p, c.c[0].p,
                                                                             c.c[1].p, c.c[2].p, ab, bb, ob, sa, sb, so);
            break;
          }
        }
        k_w11<T><<<grid2(m.nt, kThreads * kItems, cnt), kThreads, 0, s>>>(m.nt, m.te0.p, m.te1.p, m.te2.p, c.c[0].p,
                                                                            c.c[1].p, c.c[2].p, ab, bb, ob, sa, sb, so);
        break;
      default:
        break;
    }
    if (P.op == WPD11 || P.op == WDP11) {
      // pd(1,1)(f, g) = ∧11(f, ♭♯ g); dp(1,1)(f, g) = ∧11(♭♯ f, g), FastDEC.jl:391-401
      const bool dual_second = P.op == WPD11;
      const T* dform = dual_second ? bb : ab;
      const size_t sd = dual_second ? sb : sa;
      DArr<T>& tmp = const_cast<CoefSet<T>&>(c).tmp;
      if (tmp.n < (size_t)cnt * m.ne) tmp.alloc((size_t)cnt * m.ne);
      if (m.ne)
        k_fs_apply<T><<<grid2(m.ne, kThreads, cnt), kThreads, 0, s>>>(m.ne, idx, c.val.p, dform, tmp.p, sd,
                                                                      (size_t)m.ne);
      const T* fa = dual_second ? ab : tmp.p;
      const T* fb = dual_second ? tmp.p : bb;
      const size_t sfa = dual_second ? sa : (size_t)m.ne, sfb = dual_second ? (size_t)m.ne : sb;
      if (m.nt)
        k_w11<T><<<grid2(m.nt, kThreads * kItems, cnt), kThreads, 0, s>>>(m.nt, m.te0.p, m.te1.p, m.te2.p, c.c[0].p,
                                                                            c.c[1].p, c.c[2].p, fa, fb, ob, sfa, sfb,
                                                                            so);
    } else if (P.op >= WDD01) {
      // x is the form that M acts on; y is multiplied elementwise:
      //  dd(0,1)(f, g) = (M f) .* g,  pd(0,1)(g, f) = (M g) .* f   -> M acts on the first form
      //  dd(1,0)(f, g) = f .* (M g),  dp(1,0)(f, g) = f .* (M g)   -> M acts on the second form
      const bool mfirst = (P.op == WDD01 || P.op == WPD01);
      const T* x = mfirst ? ab : bb;
      const T* y = mfirst ? bb : ab;
      const size_t sx = mfirst ? sa : sb, sy = mfirst ? sb : sa;
      if (m.ne) {
        if (c.width == 2)
          k_ell_hadamard<T, 2><<<grid2(m.ne, kThreads, cnt), kThreads, 0, s>>>(m.ne, idx, c.val.p, x, y, ob, mfirst,
                                                                               sx, sy, so);
        else
          k_ell_hadamard<T, 4><<<grid2(m.ne, kThreads, cnt), kThreads, 0, s>>>(m.ne, idx, c.val.p, x, y, ob, mfirst,
                                                                               sx, sy, so);
      }
    }
    DEC_CHECK_LAUNCH();
    done += cnt;
  }
}

// ---- wedges on caller caches: dec_c_wedge_product!(Val(j), Val(k), res, α, β, p, c) ----------
// (FastDEC.jl:217-232).  The caches are the reference's Julia matrices (column-major): every
// output's indices / coefficients are contiguous (R x n_out), except (0,1) whose p is n_out x 2.
// `base` is subtracted from every index (1 for Julia's 1-based caches).  Each kernel restates
// its reference kernel's arithmetic in the same order (this file compiles without FMA
// contraction).

// wedge_kernel_01! (FastDEC.jl:159-163): res = ½ β[i] (α[p[i,1]] + α[p[i,2]]).
template <class T>
__global__ void k_cw01(int64_t n, const int32_t* __restrict__ p, int base, const T* __restrict__ a,
                       const T* __restrict__ b, T* __restrict__ res) {
  const T half = T(0.5);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    res[i] = half * b[i] * (a[p[i] - base] + a[p[n + i] - base]);
}

// wedge_kernel_02! (FastDEC.jl:165-170): res = β[i] Σ_{j=1..6} c[j,i] α[p[j,i]].
template <class T>
__global__ void k_cw02(int64_t n, const int32_t* __restrict__ p, const T* __restrict__ c, int base,
                       const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ res) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t* q = p + 6 * i;
    const T* w = c + 6 * i;
    res[i] = b[i] * (w[0] * a[q[0] - base] + w[1] * a[q[1] - base] + w[2] * a[q[2] - base] +
                     w[3] * a[q[3] - base] + w[4] * a[q[4] - base] + w[5] * a[q[5] - base]);
  }
}

// wedge_kernel_03! (FastDEC.jl:172-182): res = Σ_{j=1..24} (β[i] c[j,i]) α[p[j,i]], in j order.
template <class T>
__global__ void k_cw03(int64_t n, const int32_t* __restrict__ p, const T* __restrict__ c, int base,
                       const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ res) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t* q = p + 24 * i;
    const T* w = c + 24 * i;
    const T bv = b[i];
    T tmp = T(0);
#pragma unroll 8
    for (int j = 0; j < 24; ++j) tmp += bv * w[j] * a[q[j] - base];
    res[i] = tmp;
  }
}

// wedge_kernel_11! (FastDEC.jl:184-191).
template <class T>
__global__ void k_cw11(int64_t n, const int32_t* __restrict__ p, const T* __restrict__ c, int base,
                       const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ res) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int e0 = p[3 * i] - base, e1 = p[3 * i + 1] - base, e2 = p[3 * i + 2] - base;
    const T c1 = c[3 * i], c2 = c[3 * i + 1], c3 = c[3 * i + 2];
    const T ae0 = a[e0], ae1 = a[e1], ae2 = a[e2];
    const T be0 = b[e0], be1 = b[e1], be2 = b[e2];
    res[i] = (c1 * (ae2 * be1 - ae1 * be2) + c2 * (ae2 * be0 - ae0 * be2) + c3 * (ae1 * be0 - ae0 * be1));
  }
}

// wedge_kernel_21! (FastDEC.jl:193-205): α a 2-form (triangles t0..t3 = p[7..10, i]), β a 1-form
// (edges e0..e5 = p[1..6, i]), twelve coefficients.
template <class T>
__global__ void k_cw21(int64_t n, const int32_t* __restrict__ p, const T* __restrict__ c, int base,
                       const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ res) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t* q = p + 10 * i;
    const T* w = c + 12 * i;
    const T be0 = b[q[0] - base], be1 = b[q[1] - base], be2 = b[q[2] - base], be3 = b[q[3] - base],
            be4 = b[q[4] - base], be5 = b[q[5] - base];
    const T at0 = a[q[6] - base], at1 = a[q[7] - base], at2 = a[q[8] - base], at3 = a[q[9] - base];
    res[i] = w[0] * be3 * at3 - w[1] * be4 * at2 + w[2] * be5 * at1 + w[3] * be1 * at3 - w[4] * be2 * at2 +
             w[5] * be5 * at0 + w[6] * be0 * at3 - w[7] * be2 * at1 + w[8] * be4 * at0 + w[9] * be0 * at2 -
             w[10] * be1 * at1 + w[11] * be3 * at0;
  }
}

template <class T>
static void launch_cw(int j, int k, int64_t n, const int32_t* p, const T* c, int base, const T* a, const T* b, T* res,
                      cudaStream_t s) {
  const unsigned g = grid_for(n, kThreads);
  if (j == 0 && k == 1) k_cw01<T><<<g, kThreads, 0, s>>>(n, p, base, a, b, res);
  else if (j == 0 && k == 2) k_cw02<T><<<g, kThreads, 0, s>>>(n, p, c, base, a, b, res);
  else if (j == 0 && k == 3) k_cw03<T><<<g, kThreads, 0, s>>>(n, p, c, base, a, b, res);
  else if (j == 1 && k == 1) k_cw11<T><<<g, kThreads, 0, s>>>(n, p, c, base, a, b, res);
  else k_cw21<T><<<g, kThreads, 0, s>>>(n, p, c, base, a, b, res);
  DEC_CHECK_LAUNCH();
}

}  // namespace decb

using namespace decb;

dec_wedge_plan* wedge_plan_create_impl(dec_mesh* mh, int kind, int da, int db, dec_dtype dt) {
  require(mh != nullptr, "wedge: null mesh");
  require(dt == DEC_F64 || dt == DEC_F32, "wedge: dtype must be DEC_F64 or DEC_F32");
  Mesh& m = mh->m;
  int op = -1;
  int64_t la = 0, lb = 0, lo = 0;
  const int64_t nv = m.nv, ne = m.ne, nt = m.nt;
  if (kind == DEC_WEDGE_PP) {
    if (da == 0 && db == 1) { op = W01; la = nv; lb = ne; lo = ne; }
    else if (da == 1 && db == 0) { op = W10; la = ne; lb = nv; lo = ne; }
    else if (da == 0 && db == 2) { op = W02; la = nv; lb = nt; lo = nt; }
    else if (da == 2 && db == 0) { op = W20; la = nt; lb = nv; lo = nt; }
    else if (da == 1 && db == 1) { op = W11; la = ne; lb = ne; lo = nt; }
  } else if (kind == DEC_WEDGE_DD) {
    if (da == 0 && db == 1) { op = WDD01; la = nt; lb = ne; lo = ne; }
    else if (da == 1 && db == 0) { op = WDD10; la = ne; lb = nt; lo = ne; }
  } else if (kind == DEC_WEDGE_PD) {
    if (da == 0 && db == 1) { op = WPD01; la = nv; lb = ne; lo = ne; }
    else if (da == 1 && db == 1) { op = WPD11; la = ne; lb = ne; lo = nt; }
  } else if (kind == DEC_WEDGE_DP) {
    if (da == 1 && db == 0) { op = WDP10; la = ne; lb = nv; lo = ne; }
    else if (da == 1 && db == 1) { op = WDP11; la = ne; lb = ne; lo = nt; }
  }
  if (op < 0)
    throw Error(DEC_ERR_UNSUPPORTED,
                "Unsupported combination of degrees " + std::to_string(da) + " and " + std::to_string(db) +
                    ". Ensure that their sum is not greater than the degree of the complex.");
  auto* P = new dec_wedge_plan();
  P->m = &m;
  P->op = op;
  P->dtype = dt;
  P->len_a = la;
  P->len_b = lb;
  P->len_out = lo;
  try {
    build_plan(*P);
  } catch (...) {
    delete P;
    throw;
  }
  return P;
}

void wedge_apply_impl(dec_wedge_plan* P, const void* a, const void* b, void* out, int count, void* stream) {
  require(P != nullptr, "wedge: null plan");
  require(a && b && out, "wedge: null form pointer");
  require(count >= 1, "wedge: count must be >= 1");
  cudaStream_t s = as_stream(stream);
  if (P->dtype == DEC_F64) launch_plan<double>(*P, P->c64, a, b, out, count, s);
  else launch_plan<float>(*P, P->c32, a, b, out, count, s);
}

// Times the batched FP32 ∧11 with 1, 2, 4, 8 and 16 pairs per thread on min(count, 256) pairs of
// zero forms (reps launches each after one untimed) and stores the fastest under the plan's size
// bucket.
int wedge_autotune_impl(dec_wedge_plan* P, int count, int reps, void* stream) {
  require(P != nullptr && count >= 1 && reps >= 1, "wedge autotune: bad arguments");
  if (P->op != W11 || P->dtype != DEC_F32 || count < 2 || P->m->nt == 0) return 0;
  count = std::min(count, 256);
  cudaStream_t s = as_stream(stream);
  DArr<float> a((size_t)count * P->len_a), b((size_t)count * P->len_b), o((size_t)count * P->len_out);
  DEC_CUDA(cudaMemsetAsync(a.p, 0, a.bytes(), s));
  DEC_CUDA(cudaMemsetAsync(b.p, 0, b.bytes(), s));
  cudaEvent_t e0, e1;
  DEC_CUDA(cudaEventCreate(&e0));
  DEC_CUDA(cudaEventCreate(&e1));
  int best = 1;
  float best_ms = 1e30f;
  for (int pairs : {1, 2, 4, 8, 16}) {
    launch_plan<float>(*P, P->c32, a.p, b.p, o.p, count, s, pairs);
    DEC_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) launch_plan<float>(*P, P->c32, a.p, b.p, o.p, count, s, pairs);
    DEC_CUDA(cudaEventRecord(e1, s));
    DEC_CHECK_LAUNCH();
    DEC_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = pairs;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tune_set(w11_pairs_key(P->m->nt), best);
  return best;
}

void wedge_plan_destroy_impl(dec_wedge_plan* P) { delete P; }

void wedge_lengths_impl(const dec_wedge_plan* P, int64_t* la, int64_t* lb, int64_t* lo) {
  require(P != nullptr, "wedge: null plan");
  if (la) *la = P->len_a;
  if (lb) *lb = P->len_b;
  if (lo) *lo = P->len_out;
}

void c_wedge_apply_impl(int j, int k, int64_t n, const int32_t* p, const void* c, dec_dtype dt, const void* a,
                        const void* b, void* res, int index_base, void* stream) {
  const bool ok = (j == 0 && (k == 1 || k == 2 || k == 3)) || (j == 1 && k == 1) || (j == 2 && k == 1);
  if (!ok)
    throw Error(DEC_ERR_UNSUPPORTED,
                "Unsupported combination of degrees " + std::to_string(j) + " and " + std::to_string(k) +
                    ". Ensure that their sum is not greater than the degree of the complex.");
  require(n >= 0, "c_wedge: negative output length");
  require(dt == DEC_F64 || dt == DEC_F32, "c_wedge: dtype must be DEC_F64 or DEC_F32");
  require(index_base == 0 || index_base == 1, "c_wedge: index_base must be 0 or 1");
  if (n == 0) return;
  require(p && a && b && res && (c || (j == 0 && k == 1)), "c_wedge: null pointer");
  cudaStream_t s = as_stream(stream);
  if (dt == DEC_F64)
    launch_cw<double>(j, k, n, p, (const double*)c, index_base, (const double*)a, (const double*)b, (double*)res, s);
  else
    launch_cw<float>(j, k, n, p, (const float*)c, index_base, (const float*)a, (const float*)b, (float*)res, s);
}
