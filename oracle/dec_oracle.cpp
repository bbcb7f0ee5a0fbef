// TEST INFRASTRUCTURE ONLY: CPU restatement of the CombinatorialSpaces.jl DEC hot path.
// See dec_oracle.hpp for the scope.  Reference paths below are relative to the
// CombinatorialSpaces.jl repository root.
#include "dec_oracle.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <cstring>

#include <thread>

namespace orc {

static int g_threads = 1;
void set_num_threads(int n) { g_threads = n < 1 ? 1 : n; }
int num_threads() { return g_threads; }

// Static-partition parallel loop over [0, n) on g_threads host threads.
template <class F>
static void parallel_for(int n, F f) {
  int nt = std::min(g_threads, std::max(1, n / 4096));
  if (nt <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  for (int k = 0; k < nt; ++k)
    th.emplace_back([=, &f]() {
      int lo = (int)((long long)n * k / nt), hi = (int)((long long)n * (k + 1) / nt);
      for (int i = lo; i < hi; ++i) f(i);
    });
  for (auto& t : th) t.join();
}

static inline uint64_t ekey(int src, int tgt) {
  return ((uint64_t)(uint32_t)src << 32) | (uint32_t)tgt;
}

// ----------------------------------------------------------------------------------------
// Primal delta set
// ----------------------------------------------------------------------------------------
int Mesh::add_vertex(double x, double y, double z) {
  pts.push_back(x);
  pts.push_back(y);
  pts.push_back(z);
  return nv() - 1;
}

// add_edge!(s, src, tgt) stores ∂v1 = src and ∂v0 = tgt (SimplicialSets.jl:143-144).
int Mesh::add_edge(int src, int tgt) {
  ev1.push_back(src);
  ev0.push_back(tgt);
  eo.push_back(-1);
  int e = ne() - 1;
  emap.emplace(ekey(src, tgt), e);  // keeps the first edge of a directed pair
  return e;
}

// get_edge!(s, src, tgt), SimplicialSets.jl:348-351: reuse the first edge with ∂v1 = src
// and ∂v0 = tgt, else add one.  The reverse pair (tgt, src) is a distinct edge.
int Mesh::get_edge(int src, int tgt) {
  auto it = emap.find(ekey(src, tgt));
  if (it != emap.end()) return it->second;
  return add_edge(src, tgt);
}

// add_triangle!(s, src2_first, src2_last, tgt2), SimplicialSets.jl:323-324:
// ∂e0 = src2_last, ∂e1 = tgt2, ∂e2 = src2_first.
int Mesh::add_triangle(int src2_first, int src2_last, int tgt2, int8_t o) {
  te0.push_back(src2_last);
  te1.push_back(tgt2);
  te2.push_back(src2_first);
  to.push_back(o);
  return nt() - 1;
}

// glue_triangle!(s, v0, v1, v2), SimplicialSets.jl:343-346.  The three get_edge! calls run
// in argument order: (v0,v1), (v1,v2), (v0,v2).
int Mesh::glue_triangle(int v0, int v1, int v2, int8_t o) {
  int a = get_edge(v0, v1);
  int b = get_edge(v1, v2);
  int c = get_edge(v0, v2);
  return add_triangle(a, b, c, o);
}

// glue_sorted_triangle!, SimplicialSets.jl:361-364.
int Mesh::glue_sorted_triangle(int v0, int v1, int v2, int8_t o) {
  int v[3] = {v0, v1, v2};
  std::sort(v, v + 3);
  return glue_triangle(v[0], v[1], v[2], o);
}

void Mesh::rebuild_edge_map() {
  emap.clear();
  for (int e = 0; e < ne(); ++e) emap.emplace(ekey(ev1[e], ev0[e]), e);
}

// orient!(s, Val(2)), SimplicialSets.jl:812-852.  Depth-first search from the first
// unvisited triangle (seeded +1); two triangles sharing an edge at face slots i and j get
// opposite flags when i + j is even, equal flags otherwise.  The reference only rejects
// the case "same parity and equal flags"; that check is kept as is.
bool orient2(Mesh& m) {
  const int nt = m.nt(), ne = m.ne();
  if (nt == 0) return true;
  // coface(2, j, s, e): triangles whose ∂e_j is e, in increasing triangle order.
  std::vector<i32> cnt(3 * (size_t)ne + 1, 0), adj(3 * (size_t)nt);
  const std::vector<i32>* te[3] = {&m.te0, &m.te1, &m.te2};
  for (int j = 0; j < 3; ++j)
    for (int t = 0; t < nt; ++t) cnt[(size_t)j * ne + (*te[j])[t] + 1]++;
  for (size_t k = 0; k < 3 * (size_t)ne; ++k) cnt[k + 1] += cnt[k];
  {
    std::vector<i32> pos(cnt.begin(), cnt.end() - 1);
    for (int j = 0; j < 3; ++j)
      for (int t = 0; t < nt; ++t) adj[pos[(size_t)j * ne + (*te[j])[t]]++] = t;
  }
  std::vector<int8_t> ors(nt, 0);
  std::vector<i32> stack;
  for (int seed = 0; seed < nt; ++seed) {
    if (ors[seed] != 0) continue;
    stack.clear();
    stack.push_back(seed);
    ors[seed] = 1;
    while (!stack.empty()) {
      int x = stack.back();
      stack.pop_back();
      int8_t ox = ors[x], nox = (int8_t)-ox;
      for (int i = 0; i < 3; ++i) {
        int face = (*te[i])[x];
        for (int j = 0; j < 3; ++j) {
          bool same_parity = ((i + j) % 2) == 0;
          size_t k0 = cnt[(size_t)j * ne + face], k1 = cnt[(size_t)j * ne + face + 1];
          for (size_t k = k0; k < k1; ++k) {
            int y = adj[k];
            if (y == x) continue;
            int8_t oy = ors[y];
            if (oy == 0) {
              ors[y] = same_parity ? nox : ox;
              stack.push_back(y);
            } else if (same_parity && oy == ox) {
              return false;
            }
          }
        }
      }
    }
  }
  for (int t = 0; t < nt; ++t) m.to[t] = ors[t] == 1 ? 1 : 0;
  return true;
}

// Length of the Julia float range 0:step:stop (the grid generator's nx, ny).
static int range_len(double stop, double step) {
  double r = stop / step;
  double rr = std::round(r);
  double n = (std::fabs(r - rr) <= 1e-10 * std::max(1.0, std::fabs(r))) ? rr : std::floor(r);
  return (int)n + 1;
}

// triangulated_grid(lx, ly, dx, dy, Point3d, compress), CombMeshes.jl:79-133.
Mesh triangulated_grid(double lx, double ly, double dx, double dy, bool compress) {
  Mesh s;
  const double scale = lx / (lx + dx / 2);
  const double shift = dx / 2;
  const int nx = range_len(lx, dx), ny = range_len(ly, dy);
  s.pts.resize(3 * (size_t)nx * ny);
  for (int yi = 1; yi <= ny; ++yi) {
    double raw_y = (yi - 1) * dy;
    for (int xi = 1; xi <= nx; ++xi) {
      double raw_x = (xi - 1) * dx;
      double x = raw_x + shift * ((yi % 2) == 0 ? 1.0 : 0.0);
      if (compress) x *= scale;
      size_t i = (size_t)(xi - 1) + (size_t)nx * (yi - 1);
      s.pts[3 * i] = x;
      s.pts[3 * i + 1] = raw_y;
      s.pts[3 * i + 2] = 0.0;
    }
  }
  // for y in 1:ny-1, x in 1:nx-1 (1-based vertex numbers converted at the call)
  for (int y = 1; y <= ny - 1; ++y) {
    for (int x = 1; x <= nx - 1; ++x) {
      int i = x + nx * (y - 1);
      if (y % 2 == 0) {
        s.glue_triangle(i - 1, i + nx - 1, i + nx);
        s.glue_triangle(i - 1, i, i + nx);
      } else {
        s.glue_triangle(i - 1, i, i + nx - 1);
        s.glue_triangle(i, i + nx - 1, i + nx);
      }
    }
  }
  for (auto& o : s.eo) o = 0;
  const int nxtri = 2 * (nx - 1), nytri = ny - 1;
  for (int y = 1; y <= nytri; ++y) {
    int8_t tri_orient = (y % 2 == 0) ? 0 : 1;
    for (int x = 1; x <= nxtri; x += 2) {
      int i = x + nxtri * (y - 1);  // 1-based
      s.to[i - 1] = tri_orient;
      s.to[i] = (int8_t)!tri_orient;
    }
  }
  return s;
}

// Unit icosahedron (12 vertices, 20 faces), glued with glue_sorted_triangle! and oriented by
// orient!.  The reference loads this mesh from a downloaded artifact that is not available
// here; this generator stands in for it.
Mesh icosahedron() {
  const double p = (1.0 + std::sqrt(5.0)) / 2.0;
  const double v[12][3] = {{-1, p, 0}, {1, p, 0}, {-1, -p, 0}, {1, -p, 0},
                           {0, -1, p}, {0, 1, p}, {0, -1, -p}, {0, 1, -p},
                           {p, 0, -1}, {p, 0, 1}, {-p, 0, -1}, {-p, 0, 1}};
  const int f[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                        {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                        {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                        {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
  Mesh s;
  const double nrm = std::sqrt(1.0 + p * p);
  for (auto& q : v) s.add_vertex(q[0] / nrm, q[1] / nrm, q[2] / nrm);
  for (auto& t : f) s.glue_sorted_triangle(t[0], t[1], t[2]);
  for (auto& o : s.eo) o = 0;
  if (!orient2(s)) throw std::runtime_error("icosahedron: orient failed");
  return s;
}

// tri_345 / tri_345_false, CombMeshes.jl:348-370.
Mesh tri_345(bool orientation) {
  Mesh s;
  s.add_vertex(0, 0, 0);
  s.add_vertex(3, 0, 0);
  s.add_vertex(3, 4, 0);
  s.glue_triangle(0, 1, 2, orientation ? 1 : 0);
  for (auto& o : s.eo) o = 1;
  return s;
}

// grid_345, CombMeshes.jl:378-398.
Mesh grid_345() {
  Mesh s;
  const double P[9][2] = {{0, 4}, {3, 4}, {6, 4}, {0, 0}, {3, 0}, {6, 0}, {0, -4}, {3, -4}, {6, -4}};
  for (auto& q : P) s.add_vertex(q[0], q[1], 0);
  const int T[8][3] = {{1, 2, 4}, {5, 2, 4}, {5, 2, 3}, {5, 6, 3},
                       {5, 7, 4}, {5, 7, 8}, {5, 6, 8}, {9, 6, 8}};
  for (auto& t : T) s.glue_sorted_triangle(t[0] - 1, t[1] - 1, t[2] - 1);
  for (auto& o : s.eo) o = 1;
  if (!orient2(s)) throw std::runtime_error("grid_345: orient failed");
  for (auto& o : s.to) o = (int8_t)!o;  // flips orientation to ccw
  return s;
}

// ----------------------------------------------------------------------------------------
// Dual complex and geometry
// ----------------------------------------------------------------------------------------
static inline double sqdist(const double* a, const double* b) {
  double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return d0 * d0 + d1 * d1 + d2 * d2;  // sum((x-y).^2), SimplicialSets.jl:945
}

// volume(points) for 2 and 3 points, SimplicialSets.jl:896-902.
static inline double vol1(const double* a, const double* b) { return std::sqrt(sqdist(a, b)); }
static inline double vol2(const double* a, const double* b, const double* c) {
  double v1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double v2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double s11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
  double s22 = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2];
  double s12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
  return std::sqrt(std::fabs(s11 * s22 - s12 * s12)) / 2;
}

// geometric_center for a triangle, DiscreteExteriorCalculus.jl:100-102 (Barycenter) and
// :114-133 (Circumcenter: barycentric coordinates from the inverse Cayley-Menger matrix,
// written here in their closed form a^2 (b^2 + c^2 - a^2) : ... over the squared side lengths).
static void tri_center_point(const double* p0, const double* p1, const double* p2, int center,
                             double* out) {
  if (center == BARYCENTER) {
    for (int k = 0; k < 3; ++k) out[k] = (p0[k] + p1[k] + p2[k]) / 3;
    return;
  }
  double a2 = sqdist(p1, p2), b2 = sqdist(p0, p2), c2 = sqdist(p0, p1);
  double l0 = a2 * (b2 + c2 - a2), l1 = b2 * (c2 + a2 - b2), l2 = c2 * (a2 + b2 - c2);
  double s = l0 + l1 + l2;
  l0 /= s;
  l1 /= s;
  l2 /= s;
  for (int k = 0; k < 3; ++k) out[k] = l0 * p0[k] + l1 * p1[k] + l2 * p2[k];
}

Dual dualize(const Mesh& m0, int center) {
  Dual d;
  d.mesh = m0;
  Mesh& m = d.mesh;
  const int nv = m.nv(), ne = m.ne(), nt = m.nt();
  d.nv = nv;
  d.ne = ne;
  d.nt = nt;
  // make_dual_simplices_1d!, DiscreteExteriorCalculus.jl:301-328: in a 2D complex unset edge
  // orientations become false.
  for (auto& o : m.eo)
    if (o < 0) o = 0;
  // make_dual_simplices_2d!, :545-608: any unset triangle orientation triggers orient!.
  bool any_unset = false;
  for (auto o : m.to) any_unset |= (o < 0);
  if (any_unset && !orient2(m))
    throw std::runtime_error("The 2-simplices of the given 2D delta set are non-orientable.");

  const size_t nde = 2 * (size_t)ne + 6 * (size_t)nt, ndt = 6 * (size_t)nt;
  d.dv0.resize(nde);
  d.dv1.resize(nde);
  d.de_orient.resize(nde);
  // D_edges01: two blocks of ne, D_∂v0 = edge center, D_∂v1 = vertex center of ∂v0 / ∂v1.
  for (int e = 0; e < ne; ++e) {
    d.dv0[e] = d.edge_center(e);
    d.dv1[e] = m.ev0[e];
    d.dv0[ne + e] = d.edge_center(e);
    d.dv1[ne + e] = m.ev1[e];
    d.de_orient[e] = (int8_t)!m.eo[e];
    d.de_orient[ne + e] = m.eo[e];
  }
  const std::vector<i32>* te[3] = {&m.te0, &m.te1, &m.te2};
  // D_edges12[k]: tri center -> edge center of ∂e_k.
  for (int k = 0; k < 3; ++k)
    for (int t = 0; t < nt; ++t) {
      size_t de = 2 * (size_t)ne + (size_t)k * nt + t;
      d.dv0[de] = d.tri_center(t);
      d.dv1[de] = d.edge_center((*te[k])[t]);
      int8_t to = (k % 2 == 1) ? (int8_t)!m.to[t] : m.to[t];
      d.de_orient[de] = (int8_t)(m.eo[(*te[k])[t]] == to);  // relative_sign, :610-611
    }
  // D_edges02[k]: tri center -> vertex center of tri vertex k.
  for (int t = 0; t < nt; ++t) {
    auto tv = m.tri_vertices(t);
    for (int k = 0; k < 3; ++k) {
      size_t de = 2 * (size_t)ne + 3 * (size_t)nt + (size_t)k * nt + t;
      d.dv0[de] = d.tri_center(t);
      d.dv1[de] = tv[k];
      d.de_orient[de] = 1;
    }
  }
  // Dual triangles: schemas (v, e, ev) in this order, :584-590.
  static const int schema[6][3] = {{0, 1, 1}, {0, 2, 1}, {1, 2, 0}, {1, 0, 1}, {2, 0, 0}, {2, 1, 0}};
  d.dte0.resize(ndt);
  d.dte1.resize(ndt);
  d.dte2.resize(ndt);
  d.dt_orient.resize(ndt);
  for (int i = 0; i < 6; ++i) {
    int v = schema[i][0], e = schema[i][1], ev = schema[i][2];
    for (int t = 0; t < nt; ++t) {
      size_t dt = (size_t)i * nt + t;
      d.dte0[dt] = 2 * ne + e * nt + t;
      d.dte1[dt] = 2 * ne + 3 * nt + v * nt + t;
      d.dte2[dt] = ev * ne + (*te[e])[t];
      d.dt_orient[dt] = (i % 2 == 0) ? (int8_t)!m.to[t] : m.to[t];  // isodd(i+1) -> reversed
    }
  }

  // subdivide_duals!, :935-990.
  const size_t ndv = (size_t)nv + ne + nt;
  d.dual_point.assign(3 * ndv, 0.0);
  for (size_t k = 0; k < 3 * (size_t)nv; ++k) d.dual_point[k] = m.pts[k];
  for (int e = 0; e < ne; ++e) {  // edge_vertices = (∂v0, ∂v1)
    const double* a = &m.pts[3 * (size_t)m.ev0[e]];
    const double* b = &m.pts[3 * (size_t)m.ev1[e]];
    double* o = &d.dual_point[3 * (size_t)d.edge_center(e)];
    for (int k = 0; k < 3; ++k) o[k] = (a[k] + b[k]) / 2;  // barycenter and circumcenter agree
  }
  for (int t = 0; t < nt; ++t) {
    auto tv = m.tri_vertices(t);
    tri_center_point(&m.pts[3 * (size_t)tv[0]], &m.pts[3 * (size_t)tv[1]], &m.pts[3 * (size_t)tv[2]],
                     center, &d.dual_point[3 * (size_t)d.tri_center(t)]);
  }
  // precompute_volumes_1d!, :403-422 and set_volumes_2d! / set_dual_volumes_2d!, :963-990.
  d.length.resize(ne);
  for (int e = 0; e < ne; ++e) d.length[e] = vol1(&m.pts[3 * (size_t)m.ev0[e]], &m.pts[3 * (size_t)m.ev1[e]]);
  d.dual_length.resize(nde);
  for (size_t de = 0; de < nde; ++de)
    d.dual_length[de] = vol1(&d.dual_point[3 * (size_t)d.dv0[de]], &d.dual_point[3 * (size_t)d.dv1[de]]);
  d.area.resize(nt);
  for (int t = 0; t < nt; ++t) {
    auto tv = m.tri_vertices(t);
    d.area[t] = vol2(&m.pts[3 * (size_t)tv[0]], &m.pts[3 * (size_t)tv[1]], &m.pts[3 * (size_t)tv[2]]);
  }
  d.dual_area.resize(ndt);
  for (size_t dt = 0; dt < ndt; ++dt) {
    auto dv = d.dual_tri_vertices((int)dt);
    d.dual_area[dt] = vol2(&d.dual_point[3 * (size_t)dv[0]], &d.dual_point[3 * (size_t)dv[1]],
                           &d.dual_point[3 * (size_t)dv[2]]);
  }
  return d;
}

// ----------------------------------------------------------------------------------------
// Sparse matrices
// ----------------------------------------------------------------------------------------
CSC sparse_coo(int m, int n, const std::vector<i32>& I, const std::vector<i32>& J,
               const std::vector<double>& V) {
  CSC a;
  a.m = m;
  a.n = n;
  a.colptr.assign(n + 1, 0);
  for (auto j : J) a.colptr[j + 1]++;
  for (int j = 0; j < n; ++j) a.colptr[j + 1] += a.colptr[j];
  std::vector<i32> pos(a.colptr.begin(), a.colptr.end() - 1);
  std::vector<i32> r(I.size());
  std::vector<double> v(I.size());
  for (size_t k = 0; k < I.size(); ++k) {
    int p = pos[J[k]]++;
    r[p] = I[k];
    v[p] = V[k];
  }
  // sort rows within each column and sum duplicates (in input order)
  CSC out;
  out.m = m;
  out.n = n;
  out.colptr.assign(n + 1, 0);
  std::vector<std::pair<i32, double>> buf;
  for (int j = 0; j < n; ++j) {
    buf.clear();
    for (int p = a.colptr[j]; p < a.colptr[j + 1]; ++p) buf.emplace_back(r[p], v[p]);
    std::stable_sort(buf.begin(), buf.end(),
                     [](const auto& x, const auto& y) { return x.first < y.first; });
    for (size_t k = 0; k < buf.size(); ++k) {
      if (k > 0 && buf[k].first == out.rowval.back()) {
        out.nzval.back() += buf[k].second;
      } else {
        out.rowval.push_back(buf[k].first);
        out.nzval.push_back(buf[k].second);
      }
    }
    out.colptr[j + 1] = (i32)out.rowval.size();
  }
  return out;
}

CSC transpose(const CSC& a) {
  CSC t;
  t.m = a.n;
  t.n = a.m;
  t.colptr.assign(a.m + 1, 0);
  for (auto r : a.rowval) t.colptr[r + 1]++;
  for (int i = 0; i < a.m; ++i) t.colptr[i + 1] += t.colptr[i];
  t.rowval.resize(a.rowval.size());
  t.nzval.resize(a.nzval.size());
  std::vector<i32> pos(t.colptr.begin(), t.colptr.end() - 1);
  for (int j = 0; j < a.n; ++j)
    for (int p = a.colptr[j]; p < a.colptr[j + 1]; ++p) {
      int q = pos[a.rowval[p]]++;
      t.rowval[q] = j;
      t.nzval[q] = a.nzval[p];
    }
  return t;
}

CSC scale_rows(const std::vector<double>& d, const CSC& a) {
  CSC o = a;
  for (size_t p = 0; p < o.nzval.size(); ++p) o.nzval[p] = d[o.rowval[p]] * o.nzval[p];
  return o;
}

CSC scale_cols(const CSC& a, const std::vector<double>& d) {
  CSC o = a;
  for (int j = 0; j < a.n; ++j)
    for (int p = a.colptr[j]; p < a.colptr[j + 1]; ++p) o.nzval[p] = o.nzval[p] * d[j];
  return o;
}

// C = A * B column by column (SparseArrays spmatmul): the pattern of column j is the union
// of the columns of A selected by B[:, j], rows sorted.
CSC spgemm(const CSC& a, const CSC& b) {
  if (a.n != b.m) throw std::runtime_error("spgemm: dimension mismatch");
  CSC c;
  c.m = a.m;
  c.n = b.n;
  c.colptr.assign(b.n + 1, 0);
  std::vector<double> acc(a.m, 0.0);
  std::vector<char> mark(a.m, 0);
  std::vector<i32> rows;
  for (int j = 0; j < b.n; ++j) {
    rows.clear();
    for (int q = b.colptr[j]; q < b.colptr[j + 1]; ++q) {
      int k = b.rowval[q];
      double bv = b.nzval[q];
      for (int p = a.colptr[k]; p < a.colptr[k + 1]; ++p) {
        int i = a.rowval[p];
        if (!mark[i]) {
          mark[i] = 1;
          rows.push_back(i);
          acc[i] = 0.0;
        }
        acc[i] += a.nzval[p] * bv;
      }
    }
    std::sort(rows.begin(), rows.end());
    for (int i : rows) {
      c.rowval.push_back(i);
      c.nzval.push_back(acc[i]);
      mark[i] = 0;
    }
    c.colptr[j + 1] = (i32)c.rowval.size();
  }
  return c;
}

CSC add_identity(const CSC& a, double cshift) {
  std::vector<i32> I, J;
  std::vector<double> V;
  for (int j = 0; j < a.n; ++j)
    for (int p = a.colptr[j]; p < a.colptr[j + 1]; ++p) {
      I.push_back(a.rowval[p]);
      J.push_back(j);
      V.push_back(a.nzval[p]);
    }
  for (int i = 0; i < std::min(a.m, a.n); ++i) {
    I.push_back(i);
    J.push_back(i);
    V.push_back(cshift);
  }
  return sparse_coo(a.m, a.n, I, J, V);
}

void spmv(const CSC& a, const double* x, double* y) {
  std::fill(y, y + a.m, 0.0);
  for (int j = 0; j < a.n; ++j) {
    double xj = x[j];
    for (int p = a.colptr[j]; p < a.colptr[j + 1]; ++p) y[a.rowval[p]] += a.nzval[p] * xj;
  }
}

void apply(const CSC& A, const CSC* At, const double* x, double* y) {
  if (At == nullptr || g_threads <= 1) {
    spmv(A, x, y);
    return;
  }
  parallel_for(A.m, [&](int i) {  // row i of A = column i of Aᵀ
    double s = 0.0;
    for (int p = At->colptr[i]; p < At->colptr[i + 1]; ++p) s += At->nzval[p] * x[At->rowval[p]];
    y[i] = s;
  });
}

void spmv_t(const CSC& a, const double* x, double* y) {
  for (int j = 0; j < a.n; ++j) {
    double s = 0.0;
    for (int p = a.colptr[j]; p < a.colptr[j + 1]; ++p) s += a.nzval[p] * x[a.rowval[p]];
    y[j] = s;
  }
}

// ----------------------------------------------------------------------------------------
// FastDEC operators
// ----------------------------------------------------------------------------------------
static inline double nsign(int8_t o) { return o ? 1.0 : -1.0; }  // numeric_sign(::Bool)

// dec_p_derivbound(Val(0)), FastDEC.jl:471-494: row e has +σ at ∂v0 and -σ at ∂v1.
static void derivbound0(const Dual& d, std::vector<i32>& I, std::vector<i32>& J, std::vector<double>& V) {
  const Mesh& m = d.mesh;
  for (int e = 0; e < d.ne; ++e) {
    double s = nsign(m.eo[e]);
    I.push_back(e);
    J.push_back(m.ev0[e]);
    V.push_back(s);
    I.push_back(e);
    J.push_back(m.ev1[e]);
    V.push_back(-1 * s);
  }
}

// dec_p_derivbound(Val(1)), FastDEC.jl:496-524: row t = τ(σ(∂e0), -σ(∂e1), σ(∂e2)).
static void derivbound1(const Dual& d, std::vector<i32>& I, std::vector<i32>& J, std::vector<double>& V) {
  const Mesh& m = d.mesh;
  for (int t = 0; t < d.nt; ++t) {
    double ts = nsign(m.to[t]);
    int e[3] = {m.te0[t], m.te1[t], m.te2[t]};
    double v[3] = {nsign(m.eo[e[0]]) * ts, -1 * nsign(m.eo[e[1]]) * ts, nsign(m.eo[e[2]]) * ts};
    for (int k = 0; k < 3; ++k) {
      I.push_back(t);
      J.push_back(e[k]);
      V.push_back(v[k]);
    }
  }
}

static CSC derivbound(const Dual& d, int n, bool transpose_, bool negate) {
  std::vector<i32> I, J;
  std::vector<double> V;
  int rows, cols;
  if (n == 0) {
    derivbound0(d, I, J, V);
    rows = d.ne;
    cols = d.nv;
  } else if (n == 1) {
    derivbound1(d, I, J, V);
    rows = d.nt;
    cols = d.ne;
  } else {
    throw std::runtime_error("derivbound: n must be 0 or 1 in 2D");
  }
  if (transpose_) {
    std::swap(I, J);
    std::swap(rows, cols);
  }
  if (negate)
    for (auto& v : V) v = -1 * v;
  return sparse_coo(rows, cols, I, J, V);
}

CSC dec_differential(const Dual& d, int n) { return derivbound(d, n, false, false); }
// dec_boundary(n) = derivbound(n-1, transpose), FastDEC.jl:433-437.
CSC dec_boundary(const Dual& d, int n) { return derivbound(d, n - 1, true, false); }
// dec_dual_derivative in 2D, FastDEC.jl:449-453: (0) -> ∂2 = d1', (1) -> -∂1 = -d0'.
CSC dec_dual_derivative(const Dual& d, int n) {
  if (n == 0) return derivbound(d, 1, true, false);
  if (n == 1) return derivbound(d, 0, true, true);
  throw std::runtime_error("dual derivative: n must be 0 or 1 in 2D");
}

// dec_p_hodge_diag, FastDEC.jl:580-604 (accumulation in the reference's loop order).
std::vector<double> hodge_diag(const Dual& d, int k) {
  if (k == 0) {
    std::vector<double> h(d.nv, 0.0);
    for (size_t dt = 0; dt < d.dual_area.size(); ++dt) {
      int v = d.dv1[d.dte1[dt]];
      h[v] += d.dual_area[dt];
    }
    return h;
  }
  if (k == 1) {
    std::vector<double> h(d.ne, 0.0);
    for (size_t de = 0; de < d.dual_length.size(); ++de) {
      int e = d.dv1[de] - d.nv;
      if (e >= 0 && e < d.ne) h[e] += d.dual_length[de] / d.length[e];
    }
    return h;
  }
  if (k == 2) {
    std::vector<double> h(d.nt);
    for (int t = 0; t < d.nt; ++t) h[t] = 1 / d.area[t];
    return h;
  }
  throw std::runtime_error("hodge_diag: k must be 0, 1 or 2");
}

// dec_inv_hodge_star(Val(k), DiagonalHodge), FastDEC.jl:732-737: sign (-1)^(k(2-k)).
std::vector<double> inv_hodge_diag(const Dual& d, int k) {
  auto h = hodge_diag(d, k);
  double mult = ((k * (2 - k)) % 2 == 0) ? 1.0 : -1.0;
  for (auto& x : h) x = (1 / x) * mult;
  return h;
}

// fast_laplace_beltrami(sd) = -1 * ⋆0⁻¹ * dual_d(1) * ⋆1 * d(0), test/Multigrid.jl:46-48,
// evaluated left to right as Julia does.
CSC laplace_beltrami0(const Dual& d) {
  auto ih0 = inv_hodge_diag(d, 0);
  for (auto& x : ih0) x = -1 * x;  // -1 * Diagonal
  CSC a = scale_rows(ih0, dec_dual_derivative(d, 1));
  a = scale_cols(a, hodge_diag(d, 1));
  return spgemm(a, dec_differential(d, 0));
}

// ----------------------------------------------------------------------------------------
// Wedge products
// ----------------------------------------------------------------------------------------
// wedge_kernel_coeffs(Val(0), Val(2)), FastDEC.jl:50-62.
Wedge02Cache wedge02_cache(const Dual& d) {
  Wedge02Cache c;
  const int nt = d.nt;
  c.verts.resize(6 * (size_t)nt);
  c.coeffs.resize(6 * (size_t)nt);
  for (int t = 0; t < nt; ++t)
    for (int dt = 0; dt < 6; ++dt) {
      size_t real = (size_t)t + (size_t)dt * nt;
      c.verts[6 * (size_t)t + dt] = d.dv1[d.dte2[real]];
      c.coeffs[6 * (size_t)t + dt] = d.dual_area[real] / d.area[t];
    }
  return c;
}

// wedge_kernel_coeffs(Val(1), Val(1)), FastDEC.jl:78-93.
Wedge11Cache wedge11_cache(const Dual& d) {
  Wedge11Cache c;
  const int nt = d.nt;
  const Mesh& m = d.mesh;
  c.e.resize(3 * (size_t)nt);
  c.coeffs.resize(3 * (size_t)nt);
  const double* da = d.dual_area.data();
  for (int i = 0; i < nt; ++i) {
    double area = nsign(m.to[i]) * 2 * d.area[i];
    int e0 = m.te0[i], e1 = m.te1[i], e2 = m.te2[i];
    c.e[3 * (size_t)i] = e0;
    c.e[3 * (size_t)i + 1] = e1;
    c.e[3 * (size_t)i + 2] = e2;
    c.coeffs[3 * (size_t)i] = nsign(m.eo[e1]) * nsign(m.eo[e2]) * (da[i] + da[i + nt]) / area;
    c.coeffs[3 * (size_t)i + 1] =
        nsign(m.eo[e0]) * nsign(m.eo[e2]) * (da[i + 2 * (size_t)nt] + da[i + 3 * (size_t)nt]) / area;
    c.coeffs[3 * (size_t)i + 2] =
        nsign(m.eo[e0]) * nsign(m.eo[e1]) * (da[i + 4 * (size_t)nt] + da[i + 5 * (size_t)nt]) / area;
  }
  return c;
}

// wedge_kernel_01!, FastDEC.jl:159-163 (p = [∂v0 ∂v1], :42-47).
template <class T>
void wedge01(const Dual& d, const T* f, const T* a, T* out) {
  const Mesh& m = d.mesh;
  const T half = T(0.5);
  parallel_for(d.ne, [&](int i) { out[i] = half * a[i] * (f[m.ev0[i]] + f[m.ev1[i]]); });
}

// wedge_kernel_02!, FastDEC.jl:165-170.
template <class T>
void wedge02(const Dual& d, const Wedge02Cache& c, const T* f, const T* a, T* out) {
  parallel_for(d.nt, [&](int i) {
    const i32* p = &c.verts[6 * (size_t)i];
    T cc[6];
    for (int k = 0; k < 6; ++k) cc[k] = (T)c.coeffs[6 * (size_t)i + k];
    out[i] = a[i] * (cc[0] * f[p[0]] + cc[1] * f[p[1]] + cc[2] * f[p[2]] + cc[3] * f[p[3]] +
                     cc[4] * f[p[4]] + cc[5] * f[p[5]]);
  });
}

// wedge_kernel_11!, FastDEC.jl:184-191.
template <class T>
void wedge11(const Dual& d, const Wedge11Cache& c, const T* a, const T* b, T* out) {
  parallel_for(d.nt, [&](int i) {
    int e0 = c.e[3 * (size_t)i], e1 = c.e[3 * (size_t)i + 1], e2 = c.e[3 * (size_t)i + 2];
    T c1 = (T)c.coeffs[3 * (size_t)i], c2 = (T)c.coeffs[3 * (size_t)i + 1], c3 = (T)c.coeffs[3 * (size_t)i + 2];
    T ae0 = a[e0], ae1 = a[e1], ae2 = a[e2];
    T be0 = b[e0], be1 = b[e1], be2 = b[e2];
    out[i] = (c1 * (ae2 * be1 - ae1 * be2) + c2 * (ae2 * be0 - ae0 * be2) + c3 * (ae1 * be0 - ae0 * be1));
  });
}

template void wedge01<double>(const Dual&, const double*, const double*, double*);
template void wedge01<float>(const Dual&, const float*, const float*, float*);
template void wedge02<double>(const Dual&, const Wedge02Cache&, const double*, const double*, double*);
template void wedge02<float>(const Dual&, const Wedge02Cache&, const float*, const float*, float*);
template void wedge11<double>(const Dual&, const Wedge11Cache&, const double*, const double*, double*);
template void wedge11<float>(const Dual&, const Wedge11Cache&, const float*, const float*, float*);

// dec_c_wedge_product!(Val(j), Val(k), res, α, β, p, c) (FastDEC.jl:217-232) on caller caches in
// the reference's column-major layout, 0-based indices: wedge_kernel_01! (:159-163, p n x 2),
// _02! (:165-170, p, c 6 x n), _03! (:172-182, p, c 24 x n), _11! (:184-191, p, c 3 x n) and
// _21! (:193-205, p 10 x n, c 12 x n).  Same expressions, same order.
template <class T>
void c_wedge(int j, int k, int64_t n, const i32* p, const T* c, const T* a, const T* b, T* res) {
  for (int64_t i = 0; i < n; ++i) {
    if (j == 0 && k == 1) {
      const T half = T(0.5);
      res[i] = half * b[i] * (a[p[i]] + a[p[n + i]]);
    } else if (j == 0 && k == 2) {
      const i32* q = p + 6 * i;
      const T* w = c + 6 * i;
      res[i] = b[i] * (w[0] * a[q[0]] + w[1] * a[q[1]] + w[2] * a[q[2]] + w[3] * a[q[3]] + w[4] * a[q[4]] +
                       w[5] * a[q[5]]);
    } else if (j == 0 && k == 3) {
      T tmp = T(0);
      for (int r = 0; r < 24; ++r) tmp += b[i] * c[24 * i + r] * a[p[24 * i + r]];
      res[i] = tmp;
    } else if (j == 1 && k == 1) {
      const i32 e0 = p[3 * i], e1 = p[3 * i + 1], e2 = p[3 * i + 2];
      const T c1 = c[3 * i], c2 = c[3 * i + 1], c3 = c[3 * i + 2];
      res[i] = (c1 * (a[e2] * b[e1] - a[e1] * b[e2]) + c2 * (a[e2] * b[e0] - a[e0] * b[e2]) +
                c3 * (a[e1] * b[e0] - a[e0] * b[e1]));
    } else if (j == 2 && k == 1) {
      const i32* q = p + 10 * i;
      const T* w = c + 12 * i;
      const T be0 = b[q[0]], be1 = b[q[1]], be2 = b[q[2]], be3 = b[q[3]], be4 = b[q[4]], be5 = b[q[5]];
      const T at0 = a[q[6]], at1 = a[q[7]], at2 = a[q[8]], at3 = a[q[9]];
      res[i] = w[0] * be3 * at3 - w[1] * be4 * at2 + w[2] * be5 * at1 + w[3] * be1 * at3 - w[4] * be2 * at2 +
               w[5] * be5 * at0 + w[6] * be0 * at3 - w[7] * be2 * at1 + w[8] * be4 * at0 + w[9] * be0 * at2 -
               w[10] * be1 * at1 + w[11] * be3 * at0;
    } else {
      throw std::runtime_error("c_wedge: unsupported degrees");
    }
  }
}
template void c_wedge<double>(int, int, int64_t, const i32*, const double*, const double*, const double*, double*);
template void c_wedge<float>(int, int, int64_t, const i32*, const float*, const float*, const float*, float*);

// elementary_duals(1, s, e) = dual edges whose D_∂v1 is the center of e, in index order
// (DiscreteExteriorCalculus.jl:478-479).  In a 2D dual complex they are the D_edges12 entries.
static std::vector<std::vector<i32>> elementary_duals_1(const Dual& d) {
  std::vector<std::vector<i32>> out(d.ne);
  for (size_t de = 0; de < d.dv1.size(); ++de) {
    int e = d.dv1[de] - d.nv;
    if (e >= 0 && e < d.ne) out[e].push_back((i32)de);
  }
  return out;
}

static inline int tri_of_center(const Dual& d, int dv) { return dv - d.nv - d.ne; }

// wedge_dd_01_mat, FastDEC.jl:293-305.
CSC wedge_dd_01_mat(const Dual& d) {
  auto eds = elementary_duals_1(d);
  std::vector<i32> I, J;
  std::vector<double> V;
  for (int e = 0; e < d.ne; ++e) {
    double sum = 0;
    for (auto de : eds[e]) sum += d.dual_length[de];
    for (auto de : eds[e]) {
      I.push_back(e);
      J.push_back(tri_of_center(d, d.dv0[de]));
      V.push_back(d.dual_length[de] / sum);
    }
  }
  return sparse_coo(d.ne, d.nt, I, J, V);
}

// wedge_pd_01_mat, FastDEC.jl:329-347.
CSC wedge_pd_01_mat(const Dual& d) {
  const Mesh& m = d.mesh;
  auto eds = elementary_duals_1(d);
  std::vector<i32> I, J;
  std::vector<double> V;
  for (int e = 0; e < d.ne; ++e) {
    int a = m.ev0[e], b = m.ev1[e];
    double sum = 0;
    for (auto de : eds[e]) sum += d.dual_length[de];
    for (auto de : eds[e]) {
      int t = tri_of_center(d, d.dv0[de]);
      auto tv = m.tri_vertices(t);
      int l = -1;
      for (int k = 0; k < 3; ++k)
        if (tv[k] != a && tv[k] != b) l = tv[k];
      double w = d.dual_length[de] / sum;
      I.push_back(e); J.push_back(a); V.push_back(w * 5 / 12);
      I.push_back(e); J.push_back(b); V.push_back(w * 5 / 12);
      I.push_back(e); J.push_back(l); V.push_back(w * 2 / 12);
    }
  }
  return sparse_coo(d.ne, d.nv, I, J, V);
}

// ♭♯_mat = ♭_mat(DPPFlat) * ♯_mat(LLSDDSharp), DiscreteExteriorCalculus.jl:687-714,
// :876-909, :1992.  pinv(X) of the 3x3 matrix of dual-edge vectors (which span the triangle's
// plane, so X has rank 2 and pinv drops its third singular value) is written as
// B (YᵀY)⁻¹ Yᵀ with B an orthonormal basis of the plane and Y = X B.
// ⋆(Val(1), s, GeometricHodge()), DiscreteExteriorCalculus.jl:1680-1731.  Per triangle, with
// e = (∂e2, ∂e1, ∂e0), ev_i = p∂v0 - p∂v1 of e_i and dv_i = ±(triangle center - edge center)
// (minus for the middle edge): diagonal entries σ_t crossdot(ev_i, dv_i) / |ev_i|² times the
// triangle's relative orientation (the sign of its first nonzero one), and off-diagonal
// entries for the six ordered triples (p1, p2, p3):
// rel σ_t (ev_p1·dv_p1 / |ev_p1|²) (ev_p1·ev_p3) / crossdot(ev_p2, ev_p3); zero values are
// skipped and duplicates summed in input order.  crossdot(a, b) = |a × b| · sign((a × b)_z)
// (+1 when that component is 0), :1667-1670.
static double crossdot3(const double* a, const double* b) {
  const double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
  const double nrm = std::sqrt(c0 * c0 + c1 * c1 + c2 * c2);
  return nrm * (c2 == 0 ? 1.0 : (c2 > 0 ? 1.0 : -1.0));
}

CSC hodge_geometric1(const Dual& d) {
  const Mesh& m = d.mesh;
  std::vector<i32> I, J;
  std::vector<double> V;
  auto dot3 = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  for (int t = 0; t < d.nt; ++t) {
    const int e[3] = {m.te2[t], m.te1[t], m.te0[t]};
    double ev[3][3], dv[3][3];
    const double* tc = &d.dual_point[3 * (size_t)d.tri_center(t)];
    for (int i = 0; i < 3; ++i) {
      const double* ec = &d.dual_point[3 * (size_t)d.edge_center(e[i])];
      for (int k = 0; k < 3; ++k) {
        ev[i][k] = m.pts[3 * (size_t)m.ev0[e[i]] + k] - m.pts[3 * (size_t)m.ev1[e[i]] + k];
        dv[i][k] = (tc[k] - ec[k]) * (i == 1 ? -1.0 : 1.0);
      }
    }
    double diag_dot[3];
    for (int i = 0; i < 3; ++i) diag_dot[i] = dot3(ev[i], dv[i]) / dot3(ev[i], ev[i]);
    const double st = nsign(m.to[t]);
    double rel = 0.0;
    for (int i = 0; i < 3; ++i) {
      const double dc = st * crossdot3(ev[i], dv[i]) / dot3(ev[i], ev[i]);
      if (dc != 0.0) {
        if (rel == 0.0) rel = dc > 0 ? 1.0 : (dc < 0 ? -1.0 : 0.0);
        I.push_back(e[i]);
        J.push_back(e[i]);
        V.push_back(dc * rel);
      }
    }
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (const auto& p : perms) {
      const double val = rel * st * diag_dot[p[0]] * dot3(ev[p[0]], ev[p[2]]) / crossdot3(ev[p[1]], ev[p[2]]);
      if (val != 0.0) {
        I.push_back(e[p[0]]);
        J.push_back(e[p[1]]);
        V.push_back(val);
      }
    }
  }
  return sparse_coo(d.ne, d.ne, I, J, V);
}

// FastDEC.jl:660-716.  Per triangle, edges (∂e2, ∂e1, ∂e0); ev_i = p∂v0 - p∂v1, dv_i = triangle
// center - edge center with dv_2 negated; rel = sign of (ev_1 × dv_1)_z (1 when 0).  Entries in
// this order: diagonal rel crossdot(ev_i, dv_i) / |ev_i|² where crossdot ≠ 0, then for the six
// triples (p1, p2, p3) where val = (ev_p1·dv_p1 / |ev_p1|²) (ev_p1·ev_p3) ≠ 0 the entry
// (e_p1, e_p2) = rel val / crossdot(ev_p2, ev_p3); duplicates summed in input order.
CSC hodge_geometric1_fast(const Dual& d) {
  const Mesh& m = d.mesh;
  std::vector<i32> I, J;
  std::vector<double> V;
  auto dot3 = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  for (int t = 0; t < d.nt; ++t) {
    const int e[3] = {m.te2[t], m.te1[t], m.te0[t]};
    double ev[3][3], dv[3][3];
    const double* tc = &d.dual_point[3 * (size_t)d.tri_center(t)];
    for (int i = 0; i < 3; ++i) {
      const double* ec = &d.dual_point[3 * (size_t)d.edge_center(e[i])];
      for (int k = 0; k < 3; ++k) {
        ev[i][k] = d.dual_point[3 * (size_t)m.ev0[e[i]] + k] - d.dual_point[3 * (size_t)m.ev1[e[i]] + k];
        dv[i][k] = tc[k] - ec[k];
      }
    }
    for (int k = 0; k < 3; ++k) dv[1][k] *= -1;
    const double cz = ev[0][0] * dv[0][1] - ev[0][1] * dv[0][0];
    const double rel = cz == 0 ? 1.0 : (cz > 0 ? 1.0 : -1.0);
    for (int i = 0; i < 3; ++i) {
      const double dc = crossdot3(ev[i], dv[i]);
      if (dc != 0.0) {
        I.push_back(e[i]);
        J.push_back(e[i]);
        V.push_back(rel * dc / dot3(ev[i], ev[i]));
      }
    }
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (const auto& p : perms) {
      const double diag_dot = dot3(ev[p[0]], dv[p[0]]) / dot3(ev[p[0]], ev[p[0]]);
      const double val = diag_dot * dot3(ev[p[0]], ev[p[2]]);
      if (val != 0.0) {
        I.push_back(e[p[0]]);
        J.push_back(e[p[1]]);
        V.push_back(rel * val / crossdot3(ev[p[1]], ev[p[2]]));
      }
    }
  }
  return sparse_coo(d.ne, d.ne, I, J, V);
}

CSC flat_sharp_mat(const Dual& d) {
  const Mesh& m = d.mesh;
  auto eds = elementary_duals_1(d);
  const int nt = d.nt, ne = d.ne;
  std::vector<double> sumlen(ne, 0.0);
  for (int e = 0; e < ne; ++e)
    for (auto de : eds[e]) sumlen[e] += d.dual_length[de];
  // ♯ entries per triangle: 3 edges (sorted) x 3-vectors.
  std::vector<std::array<i32, 3>> tedges(nt);
  std::vector<std::array<double, 9>> sharp(nt);
  for (int t = 0; t < nt; ++t) {
    std::array<i32, 3> es = {m.te0[t], m.te1[t], m.te2[t]};
    std::sort(es.begin(), es.end());
    tedges[t] = es;
    int tc = d.tri_center(t);
    double X[3][3], w[3];
    for (int i = 0; i < 3; ++i) {
      int sel = -1;
      for (auto de : eds[es[i]])
        if (d.dv0[de] == tc) sel = de;
      double sg = d.de_orient[sel] ? 1.0 : -1.0;  // de_sign
      const double* p0 = &d.dual_point[3 * (size_t)d.dv0[sel]];
      const double* p1 = &d.dual_point[3 * (size_t)d.dv1[sel]];
      for (int k = 0; k < 3; ++k) X[i][k] = sg * (p0[k] - p1[k]);
      w[i] = d.dual_length[sel] / sumlen[es[i]];
    }
    // Orthonormal basis of the triangle's plane.
    auto tv = m.tri_vertices(t);
    const double* q0 = &m.pts[3 * (size_t)tv[0]];
    const double* q1 = &m.pts[3 * (size_t)tv[1]];
    const double* q2 = &m.pts[3 * (size_t)tv[2]];
    double u[3] = {q1[0] - q0[0], q1[1] - q0[1], q1[2] - q0[2]};
    double v[3] = {q2[0] - q0[0], q2[1] - q0[1], q2[2] - q0[2]};
    double nu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (auto& x : u) x /= nu;
    double uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
    for (int k = 0; k < 3; ++k) v[k] -= uv * u[k];
    double nvv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (auto& x : v) x /= nvv;
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
    double det = g00 * g11 - g01 * g01;
    double i00 = g11 / det, i01 = -g01 / det, i11 = g00 / det;
    for (int i = 0; i < 3; ++i) {
      // column i of pinv(X) = B (YᵀY)⁻¹ Y[i,:]ᵀ
      double c0 = i00 * Y[i][0] + i01 * Y[i][1];
      double c1 = i01 * Y[i][0] + i11 * Y[i][1];
      for (int k = 0; k < 3; ++k) sharp[t][3 * i + k] = w[i] * (c0 * u[k] + c1 * v[k]);
    }
  }
  // ♭ rows: e -> triangles incident to e (increasing), weight del * e_vec / sum(del).
  std::vector<std::vector<i32>> etris(ne);
  for (int t = 0; t < nt; ++t) {
    etris[m.te0[t]].push_back(t);
    etris[m.te1[t]].push_back(t);
    etris[m.te2[t]].push_back(t);
  }
  std::vector<i32> I, J;
  std::vector<double> V;
  for (int e = 0; e < ne; ++e) {
    auto& tris = etris[e];
    std::sort(tris.begin(), tris.end());
    tris.erase(std::unique(tris.begin(), tris.end()), tris.end());
    double sg = nsign(m.eo[e]);
    double ev[3];
    for (int k = 0; k < 3; ++k) ev[k] = (m.pts[3 * (size_t)m.ev0[e] + k] - m.pts[3 * (size_t)m.ev1[e] + k]) * sg;
    std::vector<double> dels;
    double dsum = 0;
    for (int t : tris) {
      int tc = d.tri_center(t), sel = -1;
      for (auto de : eds[e])
        if (d.dv0[de] == tc) sel = de;
      dels.push_back(d.dual_length[sel]);
      dsum += d.dual_length[sel];
    }
    for (size_t q = 0; q < tris.size(); ++q) {
      int t = tris[q];
      double fl[3];
      for (int k = 0; k < 3; ++k) fl[k] = dels[q] * ev[k] / dsum;
      for (int i = 0; i < 3; ++i) {
        const double* s = &sharp[t][3 * i];
        I.push_back(e);
        J.push_back(tedges[t][i]);
        V.push_back(fl[0] * s[0] + fl[1] * s[1] + fl[2] * s[2]);
      }
    }
  }
  return sparse_coo(ne, ne, I, J, V);
}

// ----------------------------------------------------------------------------------------
// Multigrid
// ----------------------------------------------------------------------------------------
Topo topo_of(const Mesh& m) {
  Topo t;
  t.nv = m.nv();
  t.ne = m.ne();
  t.nt = m.nt();
  t.ev0 = m.ev0;
  t.ev1 = m.ev1;
  t.te0 = m.te0;
  t.te1 = m.te1;
  t.te2 = m.te2;
  return t;
}

// refine(::BinarySubdivision, topo), Multigrid.jl:130-183, in 0-based numbering: coarse
// edge e splits into fine edges 2e and 2e+1 (midpoint nv+e); triangle t adds interior
// edges 2ne+3t .. 2ne+3t+2 and children 4t .. 4t+3.
Topo refine_binary(const Topo& c) {
  Topo f;
  f.nv = c.nv + c.ne;
  f.ne = 2 * c.ne + 3 * c.nt;
  f.nt = 4 * c.nt;
  f.ev0.resize(f.ne);
  f.ev1.resize(f.ne);
  for (int e = 0; e < c.ne; ++e) {
    int mm = c.nv + e;
    f.ev0[2 * e] = mm;
    f.ev1[2 * e] = c.ev0[e];
    f.ev0[2 * e + 1] = mm;
    f.ev1[2 * e + 1] = c.ev1[e];
  }
  f.te0.resize(f.nt);
  f.te1.resize(f.nt);
  f.te2.resize(f.nt);
  for (int t = 0; t < c.nt; ++t) {
    int e0 = c.te0[t], e1 = c.te1[t], e2 = c.te2[t];
    int m0 = e0 + c.nv, m1 = e1 + c.nv, m2 = e2 + c.nv;
    int m0_m1 = 2 * c.ne + 3 * t, m1_m2 = m0_m1 + 1, m0_m2 = m0_m1 + 2;
    f.ev0[m0_m1] = m1; f.ev1[m0_m1] = m0;
    f.ev0[m1_m2] = m2; f.ev1[m1_m2] = m1;
    f.ev0[m0_m2] = m2; f.ev1[m0_m2] = m0;
    int m0_v1 = 2 * e0 + 1, v2_m0 = 2 * e0;
    int m1_v0 = 2 * e1 + 1, v2_m1 = 2 * e1;
    int m2_v0 = 2 * e2 + 1, v1_m2 = 2 * e2;
    int b = 4 * t;
    f.te0[b] = m1_m2;     f.te1[b] = m0_m2;     f.te2[b] = m0_m1;
    f.te0[b + 1] = m1_m2; f.te1[b + 1] = m2_v0; f.te2[b + 1] = m1_v0;
    f.te0[b + 2] = m0_m2; f.te1[b + 2] = v1_m2; f.te2[b + 2] = m0_v1;
    f.te0[b + 3] = m0_m1; f.te1[b + 3] = v2_m1; f.te2[b + 3] = v2_m0;
  }
  return f;
}

// propagate_points(::BinarySubdivision), Multigrid.jl:111-122: midpoint of each edge.  A
// positive radius then projects the new points onto the sphere of that radius (the
// icosphere construction; the reference expresses it with a custom subdivider).
std::vector<double> propagate_points_binary(const Topo& t, const std::vector<double>& pts,
                                            double radius) {
  std::vector<double> f(3 * (size_t)(t.nv + t.ne));
  std::copy(pts.begin(), pts.begin() + 3 * (size_t)t.nv, f.begin());
  for (int e = 0; e < t.ne; ++e) {
    double* o = &f[3 * ((size_t)t.nv + e)];
    for (int k = 0; k < 3; ++k) o[k] = (pts[3 * (size_t)t.ev0[e] + k] + pts[3 * (size_t)t.ev1[e] + k]) / 2;
    if (radius > 0) {
      double n = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
      for (int k = 0; k < 3; ++k) o[k] = o[k] / n * radius;
    }
  }
  return f;
}

// subdivision_matrix(::BinarySubdivision), Multigrid.jl:191-219.
CSC subdivision_matrix_binary(const Topo& t) {
  CSC s;
  s.m = t.nv;
  s.n = t.nv + t.ne;
  s.colptr.resize(s.n + 1);
  s.rowval.resize(t.nv + 2 * (size_t)t.ne);
  s.nzval.resize(s.rowval.size());
  for (int i = 0; i < t.nv; ++i) {
    s.colptr[i] = i;
    s.rowval[i] = i;
    s.nzval[i] = 1.0;
  }
  for (int e = 0; e < t.ne; ++e) {
    int k = t.nv + 2 * e;
    s.colptr[t.nv + e] = k;
    int r0 = t.ev0[e], r1 = t.ev1[e];
    if (r0 > r1) std::swap(r0, r1);
    s.rowval[k] = r0;
    s.nzval[k] = 0.5;
    s.rowval[k + 1] = r1;
    s.nzval[k + 1] = 0.5;
  }
  s.colptr[s.n] = (i32)s.rowval.size();
  return s;
}

// make_restriction, Multigrid.jl:595-612: S with each row divided by its row sum.
CSC make_restriction(const CSC& s) {
  std::vector<double> rs(s.m, 0.0);
  for (size_t k = 0; k < s.nzval.size(); ++k) rs[s.rowval[k]] += s.nzval[k];
  CSC r = s;
  for (size_t k = 0; k < r.nzval.size(); ++k) r.nzval[k] = s.nzval[k] / rs[s.rowval[k]];
  return r;
}

// topo_to_mesh, Multigrid.jl:49-64 (orientations left unset).
Mesh topo_to_mesh(const Topo& t, const std::vector<double>& pts) {
  Mesh m;
  m.pts = pts;
  m.ev0 = t.ev0;
  m.ev1 = t.ev1;
  m.te0 = t.te0;
  m.te1 = t.te1;
  m.te2 = t.te2;
  m.eo.assign(t.ne, -1);
  m.to.assign(t.nt, -1);
  m.rebuild_edge_map();
  return m;
}

static CSC level_op(const Mesh& m, int center, double shift, Mesh* oriented) {
  Dual d = dualize(m, center);
  if (oriented) *oriented = d.mesh;
  CSC L = laplace_beltrami0(d);
  return shift != 0.0 ? add_identity(L, shift) : L;
}

// _build_multigrid(DirectMode(), s, BinarySubdivision(), levels, op, steps, alg),
// Multigrid.jl:752-797.
MGData build_mg(const Mesh& coarse, int levels, int center, double shift, double radius, int steps, bool galerkin) {
  MGData md;
  std::vector<CSC> ops;
  std::vector<Mesh> meshes;
  Mesh om;
  ops.push_back(level_op(coarse, center, shift, &om));
  meshes.push_back(om);
  md.ps.resize(levels);
  md.rs.resize(levels);
  Topo topo = topo_of(coarse);
  std::vector<double> pts = coarse.pts;
  for (int i = 1; i <= levels; ++i) {
    CSC mat = subdivision_matrix_binary(topo);
    pts = propagate_points_binary(topo, pts, radius);
    topo = refine_binary(topo);
    int idx = levels - i;
    md.ps[idx] = transpose(mat);
    md.rs[idx] = make_restriction(mat);
    ops.push_back(level_op(topo_to_mesh(topo, pts), center, shift, &om));
    meshes.push_back(om);
  }
  std::reverse(ops.begin(), ops.end());
  std::reverse(meshes.begin(), meshes.end());
  if (galerkin)  // _finalize_ops(::GalerkinMode), Multigrid.jl:740-748: ops[i+1] = rs[i] * ops[i] * ps[i]
    for (int i = 0; i < levels; ++i) ops[i + 1] = spgemm(spgemm(md.rs[i], ops[i]), md.ps[i]);
  md.ops = std::move(ops);
  md.meshes = std::move(meshes);
  md.steps.assign(levels + 1, steps);
  for (auto& a : md.ops) md.ops_t.push_back(transpose(a));
  for (auto& a : md.rs) md.rs_t.push_back(transpose(a));
  for (auto& a : md.ps) md.ps_t.push_back(transpose(a));
  return md;
}

// Krylov.jl cg(A, b, x0; itmax) with M = I, atol = rtol = sqrt(eps): warm start solves for
// Δx from r0 = b - A x0 and returns x0 + Δx.
std::vector<double> krylov_cg(const CSC& A, const std::vector<double>& b,
                              const std::vector<double>& x0, int itmax, const CSC* At) {
  const int n = A.m;
  const double eps = std::numeric_limits<double>::epsilon();
  const double atol = std::sqrt(eps), rtol = std::sqrt(eps);
  std::vector<double> x(n, 0.0), r(n), p(n), Ap(n);
  apply(A, At, x0.data(), r.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  p = r;
  double gamma = 0;
  for (int i = 0; i < n; ++i) gamma += r[i] * r[i];
  if (gamma == 0) return x0;
  double rNorm = std::sqrt(gamma);
  if (itmax == 0) itmax = 2 * n;
  double pNorm2 = gamma;
  const double eps_tol = atol + rtol * rNorm;
  bool solved = rNorm <= eps_tol;
  int iter = 0;
  bool zero_curvature = false;
  while (!(solved || iter >= itmax || zero_curvature)) {
    apply(A, At, p.data(), Ap.data());
    double pAp = 0;
    for (int i = 0; i < n; ++i) pAp += p[i] * Ap[i];
    if (pAp <= eps * pNorm2 && std::fabs(pAp) <= eps * pNorm2) {
      zero_curvature = true;
      continue;
    }
    double alpha = gamma / pAp;
    for (int i = 0; i < n; ++i) x[i] += alpha * p[i];
    for (int i = 0; i < n; ++i) r[i] += -alpha * Ap[i];
    double gamma_next = 0;
    for (int i = 0; i < n; ++i) gamma_next += r[i] * r[i];
    rNorm = std::sqrt(gamma_next);
    bool resid_decrease_mach = (rNorm + 1.0 <= 1.0);
    solved = (rNorm <= eps_tol) || resid_decrease_mach;
    if (!solved) {
      double beta = gamma_next / gamma;
      pNorm2 = gamma_next + beta * beta * pNorm2;
      gamma = gamma_next;
      for (int i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
    }
    ++iter;
  }
  for (int i = 0; i < n; ++i) x[i] += x0[i];
  return x;
}

std::vector<double> mu_cycle(const std::vector<double>& u0, const std::vector<double>& b,
                             const MGData& md, int lvl, int mu) {
  const CSC& A = md.ops[lvl];
  const CSC* At = md.ops_t.empty() ? nullptr : &md.ops_t[lvl];
  const int steps = md.steps[lvl];
  std::vector<double> u = steps == 0 ? u0 : krylov_cg(A, b, u0, steps, At);
  if (lvl >= (int)md.ops.size() - 1) return u;
  const CSC& R = md.rs[lvl];
  const CSC& P = md.ps[lvl];  // transpose(S): P*z = S' z
  std::vector<double> Au(A.m), rf(A.m), rc(R.m);
  apply(A, At, u.data(), Au.data());
  for (int i = 0; i < A.m; ++i) rf[i] = b[i] - Au[i];
  apply(R, md.rs_t.empty() ? nullptr : &md.rs_t[lvl], rf.data(), rc.data());
  std::vector<double> z = mu_cycle(std::vector<double>(rc.size(), 0.0), rc, md, lvl + 1, mu);
  if (mu > 1) z = mu_cycle(z, rc, md, lvl + 1, mu - 1);
  std::vector<double> pz(A.m);
  apply(P, md.ps_t.empty() ? nullptr : &md.ps_t[lvl], z.data(), pz.data());
  for (int i = 0; i < A.m; ++i) u[i] = u[i] + pz[i];
  return steps == 0 ? u : krylov_cg(A, b, u, steps, At);
}

std::vector<double> mu_cycles(std::vector<double> u, const std::vector<double>& b, const MGData& md,
                              int cycles, int mu) {
  for (int c = 0; c < cycles; ++c) u = mu_cycle(u, b, md, 0, mu);
  return u;
}

static std::vector<double> fmg_rec(const std::vector<double>& b, const MGData& md, int lvl, int cycles,
                                   int mu) {
  std::vector<double> z(b.size(), 0.0);
  if (lvl < (int)md.ops.size() - 1) {
    std::vector<double> bc(md.rs[lvl].m);
    spmv(md.rs[lvl], b.data(), bc.data());
    auto zc = fmg_rec(bc, md, lvl + 1, cycles, mu);
    spmv(md.ps[lvl], zc.data(), z.data());
  }
  for (int c = 0; c < cycles; ++c) z = mu_cycle(z, b, md, lvl, mu);
  return z;
}

// full_multigrid, Multigrid.jl:830-855.
std::vector<double> full_multigrid(const std::vector<double>& b, const MGData& md, int cycles, int mu) {
  std::vector<double> z(b.size(), 0.0);
  if (md.ops.size() > 1) {
    std::vector<double> bc(md.rs[0].m);
    spmv(md.rs[0], b.data(), bc.data());
    auto zc = fmg_rec(bc, md, 1, cycles, mu);
    spmv(md.ps[0], zc.data(), z.data());
  }
  return mu_cycles(z, b, md, cycles, mu);
}

// Dense LU with partial pivoting.
std::vector<double> dense_solve(const CSC& A, const std::vector<double>& b) {
  const int n = A.m;
  std::vector<double> M((size_t)n * n, 0.0), x = b;
  for (int j = 0; j < A.n; ++j)
    for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) M[(size_t)A.rowval[p] * n + j] += A.nzval[p];
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int best = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(M[(size_t)i * n + k]) > std::fabs(M[(size_t)best * n + k])) best = i;
    if (best != k) {
      for (int j = 0; j < n; ++j) std::swap(M[(size_t)k * n + j], M[(size_t)best * n + j]);
      std::swap(x[k], x[best]);
    }
    double pv = M[(size_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double f = M[(size_t)i * n + k] / pv;
      if (f == 0) continue;
      for (int j = k; j < n; ++j) M[(size_t)i * n + j] -= f * M[(size_t)k * n + j];
      x[i] -= f * x[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int j = i + 1; j < n; ++j) s -= M[(size_t)i * n + j] * x[j];
    x[i] = s / M[(size_t)i * n + i];
  }
  return x;
}

static std::vector<double> diag_of(const CSC& A) {
  std::vector<double> d(A.m, 0.0);
  for (int j = 0; j < A.n; ++j)
    for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p)
      if (A.rowval[p] == j) d[j] += A.nzval[p];
  return d;
}

// Stationary smoothing: damped Jacobi x += ω D⁻¹(b - A x), or Chebyshev iteration of the given
// degree on D⁻¹A over [λ/ratio, λ] (three-term recurrence).
static std::vector<double> smooth(const CSC& A, const std::vector<double>& b, std::vector<double> x,
                                  int sweeps, const PlainOpts& o, double lmax) {
  const int n = A.m;
  auto D = diag_of(A);
  std::vector<double> Ax(n), r(n), dvec(n, 0.0);
  if (o.smoother == 0) {
    for (int s = 0; s < sweeps; ++s) {
      spmv(A, x.data(), Ax.data());
      for (int i = 0; i < n; ++i) x[i] = x[i] + o.omega * ((b[i] - Ax[i]) / D[i]);
    }
    return x;
  }
  const double hi = lmax, lo = lmax / o.cheb_ratio;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2, sigma = theta / delta;
  double rho = 1 / sigma;
  for (int s = 0; s < sweeps; ++s) {
    spmv(A, x.data(), Ax.data());
    if (s == 0) {
      for (int i = 0; i < n; ++i) {
        dvec[i] = ((b[i] - Ax[i]) / D[i]) / theta;
        x[i] = x[i] + dvec[i];
      }
    } else {
      double rho_new = 1 / (2 * sigma - rho);
      double c1 = rho_new * rho, c2 = 2 * rho_new / delta;
      for (int i = 0; i < n; ++i) {
        dvec[i] = c1 * dvec[i] + c2 * ((b[i] - Ax[i]) / D[i]);
        x[i] = x[i] + dvec[i];
      }
      rho = rho_new;
    }
  }
  return x;
}

std::vector<double> plain_vcycle(const std::vector<double>& u0, const std::vector<double>& b,
                                 const MGData& md, const PlainOpts& o, int lvl) {
  const CSC& A = md.ops[lvl];
  if (lvl == (int)md.ops.size() - 1) return dense_solve(A, b);
  std::vector<double> u = smooth(A, b, u0, o.pre, o, o.lmax.at(lvl));
  const int n = A.m;
  std::vector<double> Au(n), rf(n), rc(md.rs[lvl].m);
  spmv(A, u.data(), Au.data());
  for (int i = 0; i < n; ++i) rf[i] = b[i] - Au[i];
  spmv(md.rs[lvl], rf.data(), rc.data());
  auto z = plain_vcycle(std::vector<double>(rc.size(), 0.0), rc, md, o, lvl + 1);
  std::vector<double> pz(n);
  spmv(md.ps[lvl], z.data(), pz.data());
  for (int i = 0; i < n; ++i) u[i] = u[i] + pz[i];
  return smooth(A, b, u, o.post, o, o.lmax.at(lvl));
}

}  // namespace orc

namespace orc {

float round_bf16(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

namespace {
struct MlpView {
  const float *W1, *b1, *W2, *b2, *w3, *b3;
  explicit MlpView(const std::vector<float>& p) {
    W1 = p.data();
    b1 = W1 + MLP_H * MLP_IN;
    W2 = b1 + MLP_H;
    b2 = W2 + MLP_H * MLP_H;
    w3 = b2 + MLP_H;
    b3 = w3 + MLP_H;
  }
};
// One sample: returns y and fills x0 (rounded), z1, h1 (rounded), z2.
// With bf16 = false every rounding is skipped and the network is evaluated in FP64 (used to
// check the backward pass against finite differences).
double mlp_one(const MlpView& v, const float* x, double* x0, double* z1, double* h1, double* z2, bool bf16) {
  auto rd = [bf16](float a) { return bf16 ? (double)round_bf16(a) : (double)a; };
  for (int k = 0; k < MLP_IN; ++k) x0[k] = rd(x[k]);
  for (int j = 0; j < MLP_H; ++j) {
    double s = v.b1[j];
    for (int k = 0; k < MLP_IN; ++k) s += rd(v.W1[j * MLP_IN + k]) * x0[k];
    z1[j] = s;
    h1[j] = bf16 ? (double)round_bf16((float)std::max(s, 0.0)) : std::max(s, 0.0);
  }
  double y = v.b3[0];
  for (int j = 0; j < MLP_H; ++j) {
    double s = v.b2[j];
    for (int i = 0; i < MLP_H; ++i) s += rd(v.W2[j * MLP_H + i]) * h1[i];
    z2[j] = s;
    y += (double)v.w3[j] * std::max(s, 0.0);
  }
  return y;
}
}  // namespace

void mlp_forward(const std::vector<float>& p, const float* x, int S, double* y, bool bf16) {
  MlpView v(p);
  double x0[MLP_IN], h1[MLP_H], z1[MLP_H], z2[MLP_H];
  for (int s = 0; s < S; ++s) y[s] = mlp_one(v, x + (size_t)s * MLP_IN, x0, z1, h1, z2, bf16);
}

void mlp_backward(const std::vector<float>& p, const float* x, const double* dy, int S, std::vector<double>& g,
                  bool bf16) {
  MlpView v(p);
  g.assign(MLP_NPARAM, 0.0);
  double* gW1 = g.data();
  double* gb1 = gW1 + MLP_H * MLP_IN;
  double* gW2 = gb1 + MLP_H;
  double* gb2 = gW2 + MLP_H * MLP_H;
  double* gw3 = gb2 + MLP_H;
  double* gb3 = gw3 + MLP_H;
  double x0[MLP_IN], h1[MLP_H], z1[MLP_H], z2[MLP_H], dz2[MLP_H];
  for (int s = 0; s < S; ++s) {
    mlp_one(v, x + (size_t)s * MLP_IN, x0, z1, h1, z2, bf16);
    const double d = dy[s];
    gb3[0] += d;
    for (int j = 0; j < MLP_H; ++j) {
      gw3[j] += d * std::max(z2[j], 0.0);
      dz2[j] = z2[j] > 0 ? d * v.w3[j] : 0.0;
      gb2[j] += dz2[j];
      for (int i = 0; i < MLP_H; ++i) gW2[j * MLP_H + i] += dz2[j] * h1[i];
    }
    for (int i = 0; i < MLP_H; ++i) {
      double dh = 0.0;
      for (int j = 0; j < MLP_H; ++j) dh += (bf16 ? (double)round_bf16(v.W2[j * MLP_H + i]) : v.W2[j * MLP_H + i]) * dz2[j];
      double dz1 = z1[i] > 0 ? dh : 0.0;
      gb1[i] += dz1;
      for (int k = 0; k < MLP_IN; ++k) gW1[i * MLP_IN + k] += dz1 * x0[k];
    }
  }
}

}  // namespace orc
