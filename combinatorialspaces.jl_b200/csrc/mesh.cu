// Mesh flattening and dual-complex geometry on the GPU.
//
// The dual complex of src/DiscreteExteriorCalculus.jl:545-608 is kept implicit: its numbering
// is a fixed function of the primal one (dual vertices = [vertices, edge centers, triangle
// centers]; dual triangle block i of nt uses schema i of ((0,1,1),(0,2,1),(1,2,0),(1,0,1),
// (2,0,0),(2,1,0))), so only per-simplex geometry is materialised.  The geometry kernels follow
// the reference's arithmetic (subdivide_duals!, :935-990; volume, src/SimplicialSets.jl:896-902)
// operation by operation; this file is compiled without FMA contraction so the FP64 results
// are reproducible bit for bit.
#include <algorithm>
#include <cmath>

#include <cub/device/device_radix_sort.cuh>

#include "mesh.cuh"

namespace decb {

// ---------------------------------------------------------------------------------------------
// device geometry helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double sqdist3(const double* a, const double* b) {
  double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return d0 * d0 + d1 * d1 + d2 * d2;
}

// volume of the triangle (a, b, c): sqrt(|(v1·v1)(v2·v2) - (v1·v2)^2|) / 2, v1 = b-a, v2 = c-a.
__device__ __forceinline__ double tri_vol(const double* a, const double* b, const double* c) {
  double v1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double v2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double s11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
  double s22 = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2];
  double s12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
  return sqrt(fabs(s11 * s22 - s12 * s12)) / 2;
}

__device__ __forceinline__ void load3(const double* __restrict__ p, int i, double* o) {
  o[0] = p[3 * (size_t)i];
  o[1] = p[3 * (size_t)i + 1];
  o[2] = p[3 * (size_t)i + 2];
}

// Edge lengths: |p(∂v0) - p(∂v1)|.
__global__ void k_edge_geom(int ne, const int32_t* __restrict__ ev0, const int32_t* __restrict__ ev1,
                            const double* __restrict__ pts, double* __restrict__ length) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    double a[3], b[3];
    load3(pts, ev0[e], a);
    load3(pts, ev1[e], b);
    length[e] = sqrt(sqdist3(a, b));
  }
}

// Per triangle: area, center (barycenter or circumcenter), the three
// triangle-center -> edge-center dual lengths and the six dual-triangle areas.
__global__ void k_tri_geom(int nt, int center, const int32_t* __restrict__ ev0,
                           const int32_t* __restrict__ ev1, const int32_t* __restrict__ te0,
                           const int32_t* __restrict__ te1, const int32_t* __restrict__ te2,
                           const int32_t* __restrict__ tv0, const int32_t* __restrict__ tv1,
                           const int32_t* __restrict__ tv2, const double* __restrict__ pts,
                           double* __restrict__ area, double* __restrict__ tcen,
                           double* __restrict__ dlen, double* __restrict__ darea) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    double p[3][3];
    load3(pts, tv0[t], p[0]);
    load3(pts, tv1[t], p[1]);
    load3(pts, tv2[t], p[2]);
    area[t] = tri_vol(p[0], p[1], p[2]);
    double tc[3];
    if (center == DEC_BARYCENTER) {
      for (int k = 0; k < 3; ++k) tc[k] = (p[0][k] + p[1][k] + p[2][k]) / 3;
    } else {
      // Circumcenter in barycentric form λ_i ∝ a_i² (b_i² + c_i² - a_i²) (the inverse
      // Cayley-Menger matrix of geometric_center(::Circumcenter), DEC.jl:114-133).
      double a2 = sqdist3(p[1], p[2]), b2 = sqdist3(p[0], p[2]), c2 = sqdist3(p[0], p[1]);
      double l0 = a2 * (b2 + c2 - a2), l1 = b2 * (c2 + a2 - b2), l2 = c2 * (a2 + b2 - c2);
      double s = l0 + l1 + l2;
      l0 /= s;
      l1 /= s;
      l2 /= s;
      for (int k = 0; k < 3; ++k) tc[k] = l0 * p[0][k] + l1 * p[1][k] + l2 * p[2][k];
    }
    for (int k = 0; k < 3; ++k) tcen[3 * (size_t)t + k] = tc[k];
    // Edge centers of ∂e0, ∂e1, ∂e2: (p(∂v0) + p(∂v1)) / 2.
    int es[3] = {te0[t], te1[t], te2[t]};
    double ec[3][3];
    for (int k = 0; k < 3; ++k) {
      double a[3], b[3];
      load3(pts, ev0[es[k]], a);
      load3(pts, ev1[es[k]], b);
      for (int q = 0; q < 3; ++q) ec[k][q] = (a[q] + b[q]) / 2;
      dlen[(size_t)k * nt + t] = sqrt(sqdist3(tc, ec[k]));
    }
    // Dual triangle i with schema (v, e): vertices (vertex v, center of ∂e_e, triangle center).
    const int sv[6] = {0, 0, 1, 1, 2, 2};
    const int se[6] = {1, 2, 2, 0, 0, 1};
#pragma unroll
    for (int i = 0; i < 6; ++i) darea[(size_t)i * nt + t] = tri_vol(p[sv[i]], ec[se[i]], tc);
  }
}

// ⋆0[v] = Σ dual_area over the dual triangles at v, in the reference's dual-triangle order
// (block-major, then triangle): dec_p_hodge_diag(Val(0)), src/FastDEC.jl:580-587.
__global__ void k_star0(int nv, int nt, const int32_t* __restrict__ ptr, const int32_t* __restrict__ v2t,
                        const double* __restrict__ darea, double* __restrict__ star0) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    int b = ptr[v], e = ptr[v + 1];
    double s = 0.0;
    int g = b;
    for (int k = 0; k < 3; ++k) {
      int ge = g;
      while (ge < e && (v2t[ge] % 3) == k) ++ge;
      for (int blk = 2 * k; blk < 2 * k + 2; ++blk)
        for (int q = g; q < ge; ++q) s += darea[(size_t)blk * nt + v2t[q] / 3];
      g = ge;
    }
    star0[v] = s;
  }
}

// ⋆1[e] = Σ dual_length / length over the triangle-center -> edge-center dual edges of e, in
// the reference's order: dec_p_hodge_diag(Val(1)), src/FastDEC.jl:589-599.
__global__ void k_star1(int ne, int nt, const int32_t* __restrict__ ptr, const int32_t* __restrict__ e2t,
                        const double* __restrict__ dlen, const double* __restrict__ length,
                        double* __restrict__ star1) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    double s = 0.0, len = length[e];
    for (int q = ptr[e]; q < ptr[e + 1]; ++q) {
      int tk = e2t[q];
      s += dlen[(size_t)(tk % 3) * nt + tk / 3] / len;
    }
    star1[e] = s;
  }
}

// ⋆2[t] = 1 / area[t], src/FastDEC.jl:601-604.
__global__ void k_star2(int nt, const double* __restrict__ area, double* __restrict__ star2) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x)
    star2[t] = 1 / area[t];
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

// orient!(s, Val(2)) (src/SimplicialSets.jl:812-852): depth-first propagation from the first
// unvisited triangle of each component, seeded true.  Returns false on the reference's
// inconsistency check.
static bool orient_triangles(int ne, int nt, const std::vector<int32_t>* te, std::vector<int8_t>& to) {
  if (nt == 0) return true;
  std::vector<int32_t> cnt(3 * (size_t)ne + 1, 0), adj(3 * (size_t)nt);
  for (int j = 0; j < 3; ++j)
    for (int t = 0; t < nt; ++t) cnt[(size_t)j * ne + te[j][t] + 1]++;
  for (size_t k = 0; k < 3 * (size_t)ne; ++k) cnt[k + 1] += cnt[k];
  {
    std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
    for (int j = 0; j < 3; ++j)
      for (int t = 0; t < nt; ++t) adj[pos[(size_t)j * ne + te[j][t]]++] = t;
  }
  std::vector<int8_t> ors(nt, 0);
  std::vector<int32_t> stack;
  for (int seed = 0; seed < nt; ++seed) {
    if (ors[seed]) continue;
    stack.assign(1, seed);
    ors[seed] = 1;
    while (!stack.empty()) {
      int x = stack.back();
      stack.pop_back();
      int8_t ox = ors[x];
      for (int i = 0; i < 3; ++i) {
        int f = te[i][x];
        for (int j = 0; j < 3; ++j) {
          bool same = ((i + j) & 1) == 0;
          for (int q = cnt[(size_t)j * ne + f]; q < cnt[(size_t)j * ne + f + 1]; ++q) {
            int y = adj[q];
            if (y == x) continue;
            if (!ors[y]) {
              ors[y] = same ? (int8_t)-ox : ox;
              stack.push_back(y);
            } else if (same && ors[y] == ox) {
              return false;
            }
          }
        }
      }
    }
  }
  for (int t = 0; t < nt; ++t) to[t] = ors[t] == 1 ? 1 : 0;
  return true;
}

// ---------------------------------------------------------------------------------------------
// derived topology on the device
// ---------------------------------------------------------------------------------------------
// Per triangle: its vertices (∂v1∂e1, ∂v0∂e2, ∂v0∂e1) and its d1 row, the three edges sorted by
// index (equal edges by position) with their coefficients τ(σ0, -σ1, σ2) packed as sign bits.
__global__ void k_tri_topo(int nt, const int32_t* __restrict__ ev0, const int32_t* __restrict__ ev1,
                           const int32_t* __restrict__ te0, const int32_t* __restrict__ te1,
                           const int32_t* __restrict__ te2, const int8_t* __restrict__ esign,
                           const int8_t* __restrict__ tsign, int32_t* __restrict__ tv0, int32_t* __restrict__ tv1,
                           int32_t* __restrict__ tv2, int32_t* __restrict__ c0, int32_t* __restrict__ c1,
                           int32_t* __restrict__ c2, uint8_t* __restrict__ neg) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const int es[3] = {te0[t], te1[t], te2[t]};
    tv0[t] = ev1[es[1]];
    tv1[t] = ev0[es[2]];
    tv2[t] = ev0[es[1]];
    const int ts = tsign[t];
    const int sg[3] = {esign[es[0]] * ts, -esign[es[1]] * ts, esign[es[2]] * ts};
    int ord[3] = {0, 1, 2};
    for (int a = 1; a < 3; ++a)
      for (int b = a; b > 0 && es[ord[b - 1]] > es[ord[b]]; --b) {
        const int x = ord[b];
        ord[b] = ord[b - 1];
        ord[b - 1] = x;
      }
    c0[t] = es[ord[0]];
    c1[t] = es[ord[1]];
    c2[t] = es[ord[2]];
    neg[t] = (uint8_t)((sg[ord[0]] < 0) | ((sg[ord[1]] < 0) << 1) | ((sg[ord[2]] < 0) << 2));
  }
}

// Pairs (x_k[t], 3t+k) pushed k-major: entry k*nt + t.
__global__ void k_pairs_tri(int nt, const int32_t* __restrict__ x0, const int32_t* __restrict__ x1,
                            const int32_t* __restrict__ x2, int32_t* __restrict__ keys, int32_t* __restrict__ vals) {
  const long long n = 3LL * nt;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q / nt), t = (int)(q % nt);
    keys[q] = k == 0 ? x0[t] : k == 1 ? x1[t] : x2[t];
    vals[q] = 3 * t + k;
  }
}

// Pairs (edge of d1 row t, ±(t+1)) pushed triangle-major: entry 3t+q.
__global__ void k_pairs_d1t(int nt, const int32_t* __restrict__ c0, const int32_t* __restrict__ c1,
                            const int32_t* __restrict__ c2, const uint8_t* __restrict__ neg,
                            int32_t* __restrict__ keys, int32_t* __restrict__ vals) {
  const long long n = 3LL * nt;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / 3), q = (int)(i % 3);
    keys[i] = q == 0 ? c0[t] : q == 1 ? c1[t] : c2[t];
    vals[i] = ((neg[t] >> q) & 1) ? -(t + 1) : (t + 1);
  }
}

// Pairs (vertex, ±(e+1)) of d0ᵀ pushed edge-major, lower vertex first (entries 2e, 2e+1); a loop
// edge gets the key nv (past every vertex, so it sorts last and is left out of the lists).
__global__ void k_pairs_d0t(int ne, int nv, const int32_t* __restrict__ ev0, const int32_t* __restrict__ ev1,
                            const int8_t* __restrict__ esign, int32_t* __restrict__ keys,
                            int32_t* __restrict__ vals) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const int a = ev0[e], b = ev1[e], s = esign[e];
    if (a == b) {
      keys[2 * (size_t)e] = keys[2 * (size_t)e + 1] = nv;
      vals[2 * (size_t)e] = vals[2 * (size_t)e + 1] = 0;
      continue;
    }
    const int lo = min(a, b), hi = max(a, b);
    const int slo = lo == a ? s : -s, shi = hi == a ? s : -s;
    keys[2 * (size_t)e] = lo;
    vals[2 * (size_t)e] = slo > 0 ? e + 1 : -(e + 1);
    keys[2 * (size_t)e + 1] = hi;
    vals[2 * (size_t)e + 1] = shi > 0 ? e + 1 : -(e + 1);
  }
}

__global__ void k_iota(long long n, int32_t* __restrict__ a) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    a[q] = (int32_t)q;
}
__global__ void k_gather_vals(long long n, const int32_t* __restrict__ order, const int32_t* __restrict__ vals,
                              int32_t* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    out[q] = vals[order[q]];
}
// Row pointers from keys sorted ascending: ptr[k] = first position whose key is >= k (keys past
// nkeys - 1 count as nkeys), ptr[nkeys] = the pairs with a key below nkeys.
__global__ void k_bounds(long long n, int nkeys, const int32_t* __restrict__ ks, int32_t* __restrict__ ptr) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q <= n; q += (long long)gridDim.x * blockDim.x) {
    const int prev = q == 0 ? -1 : min(ks[q - 1], nkeys);
    const int cur = q == n ? nkeys : min(ks[q], nkeys);
    for (int k = prev + 1; k <= cur; ++k) ptr[k] = (int32_t)q;
  }
}
__global__ void k_max_degree(int n, const int32_t* __restrict__ ptr, int* __restrict__ mx) {
  int m = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    m = max(m, ptr[v + 1] - ptr[v]);
  if (m) atomicMax(mx, m);
}

// CSR of (key, value) pairs with each key's values in push order: a stable radix sort of the
// keys with their push positions, then the values gathered in that order.
static void csr_from_pairs_dev(int nkeys, long long npairs, const int32_t* keys, const int32_t* vals,
                               DArr<int32_t>& ptr, DArr<int32_t>& out) {
  const int T = 256;
  ptr.alloc((size_t)nkeys + 1);
  out.alloc(std::max<size_t>(1, (size_t)npairs));
  if (npairs == 0) {
    DEC_CUDA(cudaMemset(ptr.p, 0, ptr.bytes()));
    return;
  }
  DArr<int32_t> idx(npairs), ks(npairs), is(npairs);
  k_iota<<<grid_for(npairs, T), T>>>(npairs, idx.p);
  DEC_CHECK_LAUNCH();
  int bits = 1;
  while (bits < 31 && (1LL << bits) <= nkeys) ++bits;  // keys lie in [0, nkeys]
  size_t tmp_bytes = 0;
  DEC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, ks.p, idx.p, is.p, (int)npairs, 0, bits));
  DArr<unsigned char> tmp(std::max<size_t>(1, tmp_bytes));
  DEC_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys, ks.p, idx.p, is.p, (int)npairs, 0, bits));
  k_gather_vals<<<grid_for(npairs, T), T>>>(npairs, is.p, vals, out.p);
  k_bounds<<<grid_for(npairs + 1, T), T>>>(npairs, nkeys, ks.p, ptr.p);
  DEC_CHECK_LAUNCH();
}

void Mesh::build(const dec_mesh_desc& d) {
  require(d.nv > 0 && d.ne >= 0 && d.nt >= 0, "mesh: counts must be positive");
  require(d.points && d.e_v0 && d.e_v1, "mesh: points and edge arrays are required");
  require(d.nt == 0 || (d.t_e0 && d.t_e1 && d.t_e2), "mesh: triangle arrays are required");
  require(d.index_base == 0 || d.index_base == 1, "mesh: index_base must be 0 or 1");
  require(d.center == DEC_BARYCENTER || d.center == DEC_CIRCUMCENTER, "mesh: unknown center");
  require(3LL * d.nt < (1LL << 31) && 2LL * d.ne < (1LL << 31), "mesh: too large for int32 indexing");
  nv = d.nv;
  ne = d.ne;
  nt = d.nt;
  center = d.center;
  const int base = d.index_base;
  h_pts.assign(d.points, d.points + 3 * (size_t)nv);
  h_ev0.resize(ne);
  h_ev1.resize(ne);
  for (int e = 0; e < ne; ++e) {
    h_ev0[e] = d.e_v0[e] - base;
    h_ev1[e] = d.e_v1[e] - base;
    require(h_ev0[e] >= 0 && h_ev0[e] < nv && h_ev1[e] >= 0 && h_ev1[e] < nv, "mesh: edge vertex out of range");
  }
  h_te0.resize(nt);
  h_te1.resize(nt);
  h_te2.resize(nt);
  for (int t = 0; t < nt; ++t) {
    h_te0[t] = d.t_e0[t] - base;
    h_te1[t] = d.t_e1[t] - base;
    h_te2[t] = d.t_e2[t] - base;
    require(h_te0[t] >= 0 && h_te0[t] < ne && h_te1[t] >= 0 && h_te1[t] < ne && h_te2[t] >= 0 &&
                h_te2[t] < ne,
            "mesh: triangle edge out of range");
  }
  // Orientation: unset edges become false (make_dual_simplices_1d!, DEC.jl:311-320); any unset
  // triangle runs orient! (make_dual_simplices_2d!, DEC.jl:570-579).
  h_eo.assign(ne, 0);
  if (d.edge_orientation)
    for (int e = 0; e < ne; ++e) h_eo[e] = d.edge_orientation[e] > 0 ? 1 : 0;
  h_to.assign(nt, 0);
  bool unset = d.tri_orientation == nullptr;
  if (!unset)
    for (int t = 0; t < nt; ++t) {
      if (d.tri_orientation[t] < 0) unset = true;
      h_to[t] = d.tri_orientation[t] > 0 ? 1 : 0;
    }
  if (unset) {
    std::vector<int32_t> te[3] = {h_te0, h_te1, h_te2};
    if (!orient_triangles(ne, nt, te, h_to))
      throw Error(DEC_ERR_NON_ORIENTABLE, "The 2-simplices of the given 2D delta set are non-orientable.");
  }

  // Derived topology on the device, from the raw arrays only.
  ev0.upload(h_ev0);
  ev1.upload(h_ev1);
  te0.upload(h_te0);
  te1.upload(h_te1);
  te2.upload(h_te2);
  std::vector<int8_t> es(ne), ts(nt);
  for (int e = 0; e < ne; ++e) es[e] = h_eo[e] ? 1 : -1;
  for (int t = 0; t < nt; ++t) ts[t] = h_to[t] ? 1 : -1;
  esign.upload(es);
  tsign.upload(ts);
  pts.upload(h_pts);
  host_ready = true;
  derive();
}

// refine(::BinarySubdivision) on the device (Multigrid.jl:130-183, 0-based): coarse edge e splits
// into fine edge 2e (midpoint -> ∂v0) and 2e+1 (midpoint -> ∂v1), its midpoint vertex nv + e placed by
// propagate_points (:111-122) and optionally projected onto the sphere of the given radius
// (the arithmetic of the host statement, uncontracted).
__global__ void k_refine_edges(int nvc, int nec, const int32_t* __restrict__ cev0, const int32_t* __restrict__ cev1,
                               const double* __restrict__ cpts, double radius, int32_t* __restrict__ fev0,
                               int32_t* __restrict__ fev1, double* __restrict__ fpts) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nec; e += gridDim.x * blockDim.x) {
    const int a = cev0[e], b = cev1[e], m = nvc + e;
    fev0[2 * e] = m;
    fev1[2 * e] = a;
    fev0[2 * e + 1] = m;
    fev1[2 * e + 1] = b;
    double o[3];
    for (int k = 0; k < 3; ++k) o[k] = (cpts[3 * (size_t)a + k] + cpts[3 * (size_t)b + k]) / 2;
    if (radius > 0) {
      const double nrm = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
      for (int k = 0; k < 3; ++k) o[k] = o[k] / nrm * radius;
    }
    for (int k = 0; k < 3; ++k) fpts[3 * (size_t)m + k] = o[k];
  }
}

// The triangles' part of refine: per coarse triangle t its three interior edges 2ne + 3t + (0, 1, 2)
// and its four children 4t .. 4t+3 with their ∂e wiring (Multigrid.jl:160-179), and the children's
// orientation in closed form (o, ¬o, o, ¬o), o the coarse triangle's (flipped where flip[t] is set:
// the first refinement follows orient!'s DFS seeded true at each component's first triangle).
__global__ void k_refine_tris(int nvc, int nec, int ntc, const int32_t* __restrict__ cte0,
                              const int32_t* __restrict__ cte1, const int32_t* __restrict__ cte2,
                              const int8_t* __restrict__ ctsign, const int8_t* __restrict__ flip,
                              int32_t* __restrict__ fev0, int32_t* __restrict__ fev1, int32_t* __restrict__ fte0,
                              int32_t* __restrict__ fte1, int32_t* __restrict__ fte2, int8_t* __restrict__ ftsign) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntc; t += gridDim.x * blockDim.x) {
    const int e0 = cte0[t], e1 = cte1[t], e2 = cte2[t];
    const int m0 = e0 + nvc, m1 = e1 + nvc, m2 = e2 + nvc;
    const int m0_m1 = 2 * nec + 3 * t, m1_m2 = m0_m1 + 1, m0_m2 = m0_m1 + 2;
    fev0[m0_m1] = m1;
    fev1[m0_m1] = m0;
    fev0[m1_m2] = m2;
    fev1[m1_m2] = m1;
    fev0[m0_m2] = m2;
    fev1[m0_m2] = m0;
    const int m0_v1 = 2 * e0 + 1, v2_m0 = 2 * e0, m1_v0 = 2 * e1 + 1, v2_m1 = 2 * e1, m2_v0 = 2 * e2 + 1,
              v1_m2 = 2 * e2;
    const int b = 4 * t;
    fte0[b] = m1_m2;
    fte1[b] = m0_m2;
    fte2[b] = m0_m1;
    fte0[b + 1] = m1_m2;
    fte1[b + 1] = m2_v0;
    fte2[b + 1] = m1_v0;
    fte0[b + 2] = m0_m2;
    fte1[b + 2] = v1_m2;
    fte2[b + 2] = m0_v1;
    fte0[b + 3] = m0_m1;
    fte1[b + 3] = v2_m1;
    fte2[b + 3] = v2_m0;
    bool o = ctsign[t] > 0;
    if (flip && flip[t]) o = !o;
    const int8_t so = o ? 1 : -1;
    ftsign[b] = so;
    ftsign[b + 1] = (int8_t)-so;
    ftsign[b + 2] = so;
    ftsign[b + 3] = (int8_t)-so;
  }
}

void Mesh::refine_from(const Mesh& c, double radius, const int8_t* dflip, int center_kind) {
  require(4LL * c.nt < (1LL << 30) && 2LL * c.ne + 3LL * c.nt < (1LL << 30) && (long long)c.nv + c.ne < (1LL << 30),
          "multigrid: hierarchy too large");
  nv = c.nv + c.ne;
  ne = 2 * c.ne + 3 * c.nt;
  nt = 4 * c.nt;
  center = center_kind;
  ev0.alloc(ne);
  ev1.alloc(ne);
  te0.alloc(nt);
  te1.alloc(nt);
  te2.alloc(nt);
  esign.alloc(ne);
  tsign.alloc(nt);
  pts.alloc(3 * (size_t)nv);
  const int T = 256;
  // the coarse vertices keep their places; unset edge orientations become false (DEC.jl:311-320)
  DEC_CUDA(cudaMemcpy(pts.p, c.pts.p, 3 * (size_t)c.nv * sizeof(double), cudaMemcpyDeviceToDevice));
  if (ne) DEC_CUDA(cudaMemset(esign.p, 0xFF, (size_t)ne));
  if (c.ne)
    k_refine_edges<<<grid_for(c.ne, T), T>>>(c.nv, c.ne, c.ev0.p, c.ev1.p, c.pts.p, radius, ev0.p, ev1.p, pts.p);
  if (c.nt)
    k_refine_tris<<<grid_for(c.nt, T), T>>>(c.nv, c.ne, c.nt, c.te0.p, c.te1.p, c.te2.p, c.tsign.p, dflip, ev0.p,
                                            ev1.p, te0.p, te1.p, te2.p, tsign.p);
  DEC_CHECK_LAUNCH();
  host_ready = false;
  derive();
}

void Mesh::ensure_host() const {
  if (host_ready) return;
  h_ev0 = ev0.download();
  h_ev1 = ev1.download();
  h_te0 = te0.download();
  h_te1 = te1.download();
  h_te2 = te2.download();
  h_pts = pts.download();
  auto es = esign.download();
  auto ts = tsign.download();
  h_eo.resize(ne);
  h_to.resize(nt);
  for (int e = 0; e < ne; ++e) h_eo[e] = es[e] > 0 ? 1 : 0;
  for (int t = 0; t < nt; ++t) h_to[t] = ts[t] > 0 ? 1 : 0;
  host_ready = true;
}

// Derived topology, incidence and geometry, on the device from the raw arrays only.
void Mesh::derive() {
  tv0.alloc(nt);
  tv1.alloc(nt);
  tv2.alloc(nt);
  d1c0.alloc(nt);
  d1c1.alloc(nt);
  d1c2.alloc(nt);
  d1neg.alloc(nt);
  const int T = 256;
  if (nt)
    k_tri_topo<<<grid_for(nt, T), T>>>(nt, ev0.p, ev1.p, te0.p, te1.p, te2.p, esign.p, tsign.p, tv0.p, tv1.p, tv2.p,
                                       d1c0.p, d1c1.p, d1c2.p, d1neg.p);
  DEC_CHECK_LAUNCH();
  {
    DArr<int32_t> keys(std::max<size_t>(1, std::max(3 * (size_t)nt, 2 * (size_t)ne)));
    DArr<int32_t> vals(keys.n);
    // v2t: vertex -> 3t+k pushed k-major (k, then t); e2t likewise over the triangles' edges
    if (nt) k_pairs_tri<<<grid_for(3LL * nt, T), T>>>(nt, tv0.p, tv1.p, tv2.p, keys.p, vals.p);
    DEC_CHECK_LAUNCH();
    csr_from_pairs_dev(nv, 3LL * nt, keys.p, vals.p, v2t_ptr, v2t);
    if (nt) k_pairs_tri<<<grid_for(3LL * nt, T), T>>>(nt, te0.p, te1.p, te2.p, keys.p, vals.p);
    DEC_CHECK_LAUNCH();
    csr_from_pairs_dev(ne, 3LL * nt, keys.p, vals.p, e2t_ptr, e2t);
    // d1ᵀ rows: for edge e, entries ±(t+1) pushed triangle-major
    if (nt) k_pairs_d1t<<<grid_for(3LL * nt, T), T>>>(nt, d1c0.p, d1c1.p, d1c2.p, d1neg.p, keys.p, vals.p);
    DEC_CHECK_LAUNCH();
    csr_from_pairs_dev(ne, 3LL * nt, keys.p, vals.p, e2ts_ptr, e2ts);
    // d0ᵀ rows: for vertex v, entries ±(e+1) (d0[e,∂v0] = σ, d0[e,∂v1] = -σ) pushed edge-major,
    // the lower vertex first; loops (∂v0 = ∂v1) are skipped
    if (ne) k_pairs_d0t<<<grid_for(2LL * ne, T), T>>>(ne, nv, ev0.p, ev1.p, esign.p, keys.p, vals.p);
    DEC_CHECK_LAUNCH();
    csr_from_pairs_dev(nv, 2LL * ne, keys.p, vals.p, v2e_ptr, v2e);
    DArr<int> mx(1);
    DEC_CUDA(cudaMemset(mx.p, 0, sizeof(int)));
    k_max_degree<<<grid_for(nv, T), T>>>(nv, v2e_ptr.p, mx.p);
    DEC_CHECK_LAUNCH();
    max_v2e = mx.download()[0];
  }

  // Geometry.
  length.alloc(ne);
  area.alloc(nt);
  tri_center.alloc(3 * (size_t)nt);
  dual_area.alloc(6 * (size_t)nt);
  dual_len_te.alloc(3 * (size_t)nt);
  star0.alloc(nv);
  star1.alloc(ne);
  star2.alloc(nt);
  if (ne) k_edge_geom<<<grid_for(ne, T), T>>>(ne, ev0.p, ev1.p, pts.p, length.p);
  if (nt)
    k_tri_geom<<<grid_for(nt, T), T>>>(nt, center, ev0.p, ev1.p, te0.p, te1.p, te2.p, tv0.p, tv1.p,
                                         tv2.p, pts.p, area.p, tri_center.p, dual_len_te.p, dual_area.p);
  DEC_CHECK_LAUNCH();
  k_star0<<<grid_for(nv, T), T>>>(nv, nt, v2t_ptr.p, v2t.p, dual_area.p, star0.p);
  if (ne) k_star1<<<grid_for(ne, T), T>>>(ne, nt, e2t_ptr.p, e2t.p, dual_len_te.p, length.p, star1.p);
  if (nt) k_star2<<<grid_for(nt, T), T>>>(nt, area.p, star2.p);
  DEC_CHECK_LAUNCH();
  DEC_CUDA(cudaDeviceSynchronize());
}

}  // namespace decb
