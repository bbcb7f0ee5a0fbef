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

// Counting sort of (key, value) pairs, stable in insertion order.
static void csr_from_pairs(int nkeys, const std::vector<int32_t>& keys, const std::vector<int32_t>& vals,
                           std::vector<int32_t>& ptr, std::vector<int32_t>& out) {
  ptr.assign(nkeys + 1, 0);
  for (auto k : keys) ptr[k + 1]++;
  for (int i = 0; i < nkeys; ++i) ptr[i + 1] += ptr[i];
  out.resize(keys.size());
  std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1);
  for (size_t q = 0; q < keys.size(); ++q) out[pos[keys[q]]++] = vals[q];
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

  // Triangle vertices and the simplicial identities they rely on.
  std::vector<int32_t> h_tv0(nt), h_tv1(nt), h_tv2(nt);
  for (int t = 0; t < nt; ++t) {
    h_tv0[t] = h_ev1[h_te1[t]];
    h_tv1[t] = h_ev0[h_te2[t]];
    h_tv2[t] = h_ev0[h_te1[t]];
  }
  // d1 rows sorted by edge index, with signs τ(σ0, -σ1, σ2).
  std::vector<int32_t> c0(nt), c1(nt), c2(nt);
  std::vector<uint8_t> neg(nt);
  for (int t = 0; t < nt; ++t) {
    int ts = h_to[t] ? 1 : -1;
    int es[3] = {h_te0[t], h_te1[t], h_te2[t]};
    int sg[3] = {(h_eo[es[0]] ? 1 : -1) * ts, -(h_eo[es[1]] ? 1 : -1) * ts, (h_eo[es[2]] ? 1 : -1) * ts};
    int ord[3] = {0, 1, 2};
    std::sort(ord, ord + 3, [&](int a, int b) { return es[a] < es[b] || (es[a] == es[b] && a < b); });
    c0[t] = es[ord[0]];
    c1[t] = es[ord[1]];
    c2[t] = es[ord[2]];
    neg[t] = (uint8_t)((sg[ord[0]] < 0) | ((sg[ord[1]] < 0) << 1) | ((sg[ord[2]] < 0) << 2));
  }
  // Incidence lists.
  std::vector<int32_t> keys, vals, ptr, out;
  keys.reserve(3 * (size_t)nt);
  vals.reserve(3 * (size_t)nt);
  for (int k = 0; k < 3; ++k)
    for (int t = 0; t < nt; ++t) {
      keys.push_back(k == 0 ? h_tv0[t] : k == 1 ? h_tv1[t] : h_tv2[t]);
      vals.push_back(3 * t + k);
    }
  csr_from_pairs(nv, keys, vals, ptr, out);
  v2t_ptr.upload(ptr);
  v2t.upload(out);
  keys.clear();
  vals.clear();
  for (int k = 0; k < 3; ++k)
    for (int t = 0; t < nt; ++t) {
      keys.push_back(k == 0 ? h_te0[t] : k == 1 ? h_te1[t] : h_te2[t]);
      vals.push_back(3 * t + k);
    }
  csr_from_pairs(ne, keys, vals, ptr, out);
  e2t_ptr.upload(ptr);
  e2t.upload(out);
  // d1ᵀ rows: for edge e, entries (t, coefficient of e in d1 row t), sorted by t.
  keys.clear();
  vals.clear();
  for (int t = 0; t < nt; ++t) {
    int cs[3] = {c0[t], c1[t], c2[t]};
    for (int q = 0; q < 3; ++q) {
      keys.push_back(cs[q]);
      vals.push_back(((neg[t] >> q) & 1) ? -(t + 1) : (t + 1));
    }
  }
  csr_from_pairs(ne, keys, vals, ptr, out);
  e2ts_ptr.upload(ptr);
  e2ts.upload(out);
  // d0ᵀ rows: for vertex v, entries (e, d0[e, v]) sorted by e (d0[e,∂v0] = σ, d0[e,∂v1] = -σ).
  keys.clear();
  vals.clear();
  for (int e = 0; e < ne; ++e) {
    int s = h_eo[e] ? 1 : -1;
    int a = h_ev0[e], b = h_ev1[e];
    if (a == b) continue;
    int lo = std::min(a, b), hi = std::max(a, b);
    int slo = (lo == a) ? s : -s, shi = (hi == a) ? s : -s;
    keys.push_back(lo);
    vals.push_back(slo > 0 ? e + 1 : -(e + 1));
    keys.push_back(hi);
    vals.push_back(shi > 0 ? e + 1 : -(e + 1));
  }
  csr_from_pairs(nv, keys, vals, ptr, out);
  max_v2e = 0;
  for (int v = 0; v < nv; ++v) max_v2e = std::max(max_v2e, ptr[v + 1] - ptr[v]);
  // entries of one vertex were pushed in increasing edge order
  v2e_ptr.upload(ptr);
  v2e.upload(out);

  // Upload topology.
  ev0.upload(h_ev0);
  ev1.upload(h_ev1);
  te0.upload(h_te0);
  te1.upload(h_te1);
  te2.upload(h_te2);
  tv0.upload(h_tv0);
  tv1.upload(h_tv1);
  tv2.upload(h_tv2);
  d1c0.upload(c0);
  d1c1.upload(c1);
  d1c2.upload(c2);
  d1neg.upload(neg);
  std::vector<int8_t> es(ne), ts(nt);
  for (int e = 0; e < ne; ++e) es[e] = h_eo[e] ? 1 : -1;
  for (int t = 0; t < nt; ++t) ts[t] = h_to[t] ? 1 : -1;
  esign.upload(es);
  tsign.upload(ts);
  pts.upload(h_pts);

  // Geometry.
  length.alloc(ne);
  area.alloc(nt);
  tri_center.alloc(3 * (size_t)nt);
  dual_area.alloc(6 * (size_t)nt);
  dual_len_te.alloc(3 * (size_t)nt);
  star0.alloc(nv);
  star1.alloc(ne);
  star2.alloc(nt);
  const int T = 256;
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
