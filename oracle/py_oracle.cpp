// TEST INFRASTRUCTURE ONLY: Python bindings of the CPU oracle (dec_oracle.hpp).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <chrono>

#include "dec_oracle.hpp"

#include <cstring>

namespace py = pybind11;
using namespace orc;

template <class T>
static py::array_t<T> to_np(const std::vector<T>& v) {
  py::array_t<T> a(v.size());
  if (!v.empty()) std::memcpy(a.mutable_data(), v.data(), v.size() * sizeof(T));
  return a;
}

template <class T>
static std::vector<T> from_np(py::array_t<T, py::array::c_style | py::array::forcecast> a) {
  return std::vector<T>(a.data(), a.data() + a.size());
}

static py::tuple csc_tuple(const CSC& c) {
  return py::make_tuple(to_np(c.colptr), to_np(c.rowval), to_np(c.nzval), py::make_tuple(c.m, c.n));
}

static py::array_t<double> pts_np(const std::vector<double>& p) {
  py::array_t<double> a({(py::ssize_t)(p.size() / 3), (py::ssize_t)3});
  if (!p.empty()) std::memcpy(a.mutable_data(), p.data(), p.size() * sizeof(double));
  return a;
}

static Mesh mesh_from_arrays(py::array_t<double, py::array::c_style | py::array::forcecast> pts,
                             py::array_t<int32_t, py::array::c_style | py::array::forcecast> ev0,
                             py::array_t<int32_t, py::array::c_style | py::array::forcecast> ev1,
                             py::array_t<int32_t, py::array::c_style | py::array::forcecast> te0,
                             py::array_t<int32_t, py::array::c_style | py::array::forcecast> te1,
                             py::array_t<int32_t, py::array::c_style | py::array::forcecast> te2,
                             py::array_t<int8_t, py::array::c_style | py::array::forcecast> eo,
                             py::array_t<int8_t, py::array::c_style | py::array::forcecast> to) {
  Mesh m;
  m.pts = from_np(pts);
  m.ev0 = from_np(ev0);
  m.ev1 = from_np(ev1);
  m.te0 = from_np(te0);
  m.te1 = from_np(te1);
  m.te2 = from_np(te2);
  m.eo = from_np(eo);
  m.to = from_np(to);
  if (m.eo.size() != m.ev0.size() || m.to.size() != m.te0.size())
    throw std::runtime_error("orientation arrays do not match the edge / triangle counts");
  m.rebuild_edge_map();
  return m;
}

template <class T>
static py::array_t<T> run_wedge(const Dual& d, int kind, py::array_t<T, py::array::c_style> a,
                                py::array_t<T, py::array::c_style> b) {
  if (kind == 1) {  // (0,1): f on vertices, α on edges
    py::array_t<T> out(d.ne);
    wedge01<T>(d, a.data(), b.data(), out.mutable_data());
    return out;
  } else if (kind == 2) {  // (0,2)
    auto c = wedge02_cache(d);
    py::array_t<T> out(d.nt);
    wedge02<T>(d, c, a.data(), b.data(), out.mutable_data());
    return out;
  } else if (kind == 11) {
    auto c = wedge11_cache(d);
    py::array_t<T> out(d.nt);
    wedge11<T>(d, c, a.data(), b.data(), out.mutable_data());
    return out;
  }
  throw std::runtime_error("unsupported wedge kind");
}

PYBIND11_MODULE(dec_oracle, mod) {
  mod.doc() = "TEST INFRASTRUCTURE ONLY: CPU restatement of the CombinatorialSpaces.jl DEC hot path";
  mod.attr("BARYCENTER") = (int)BARYCENTER;
  mod.attr("CIRCUMCENTER") = (int)CIRCUMCENTER;

  mod.def("set_num_threads", &set_num_threads);
  mod.def("num_threads", &num_threads);

  py::class_<Mesh>(mod, "Mesh")
      .def(py::init<>())
      .def_property_readonly("nv", &Mesh::nv)
      .def_property_readonly("ne", &Mesh::ne)
      .def_property_readonly("nt", &Mesh::nt)
      .def_property_readonly("points", [](const Mesh& m) { return pts_np(m.pts); })
      .def_property_readonly("ev0", [](const Mesh& m) { return to_np(m.ev0); })
      .def_property_readonly("ev1", [](const Mesh& m) { return to_np(m.ev1); })
      .def_property_readonly("te0", [](const Mesh& m) { return to_np(m.te0); })
      .def_property_readonly("te1", [](const Mesh& m) { return to_np(m.te1); })
      .def_property_readonly("te2", [](const Mesh& m) { return to_np(m.te2); })
      .def_property_readonly("edge_orientation", [](const Mesh& m) { return to_np(m.eo); })
      .def_property_readonly("tri_orientation", [](const Mesh& m) { return to_np(m.to); })
      .def("add_vertex", &Mesh::add_vertex)
      .def("glue_triangle", &Mesh::glue_triangle, py::arg("v0"), py::arg("v1"), py::arg("v2"),
           py::arg("orientation") = -1)
      .def("glue_sorted_triangle", &Mesh::glue_sorted_triangle, py::arg("v0"), py::arg("v1"),
           py::arg("v2"), py::arg("orientation") = -1)
      .def("set_edge_orientation", [](Mesh& m, int v) { for (auto& o : m.eo) o = (int8_t)v; })
      .def("set_tri_orientation",
           [](Mesh& m, py::array_t<int8_t, py::array::c_style | py::array::forcecast> a) {
             m.to = from_np(a);
           })
      .def("tri_vertices", [](const Mesh& m) {
        py::array_t<int32_t> a({(py::ssize_t)m.nt(), (py::ssize_t)3});
        auto* p = a.mutable_data();
        for (int t = 0; t < m.nt(); ++t) {
          auto v = m.tri_vertices(t);
          p[3 * t] = v[0];
          p[3 * t + 1] = v[1];
          p[3 * t + 2] = v[2];
        }
        return a;
      })
      .def("copy", [](const Mesh& m) { return Mesh(m); });

  mod.def("mesh_from_arrays", &mesh_from_arrays);
  mod.def("orient", [](Mesh& m) { return orient2(m); });
  mod.def("triangulated_grid", &triangulated_grid, py::arg("lx"), py::arg("ly"), py::arg("dx"),
          py::arg("dy"), py::arg("compress") = true);
  mod.def("icosahedron", &icosahedron);
  mod.def("tri_345", &tri_345, py::arg("orientation") = true);
  mod.def("grid_345", &grid_345);

  py::class_<Dual>(mod, "Dual")
      .def_readonly("nv", &Dual::nv)
      .def_readonly("ne", &Dual::ne)
      .def_readonly("nt", &Dual::nt)
      .def_readonly("mesh", &Dual::mesh)
      .def_property_readonly("D_dv0", [](const Dual& d) { return to_np(d.dv0); })
      .def_property_readonly("D_dv1", [](const Dual& d) { return to_np(d.dv1); })
      .def_property_readonly("D_de0", [](const Dual& d) { return to_np(d.dte0); })
      .def_property_readonly("D_de1", [](const Dual& d) { return to_np(d.dte1); })
      .def_property_readonly("D_de2", [](const Dual& d) { return to_np(d.dte2); })
      .def_property_readonly("D_edge_orientation", [](const Dual& d) { return to_np(d.de_orient); })
      .def_property_readonly("dual_point", [](const Dual& d) { return pts_np(d.dual_point); })
      .def_property_readonly("length", [](const Dual& d) { return to_np(d.length); })
      .def_property_readonly("area", [](const Dual& d) { return to_np(d.area); })
      .def_property_readonly("dual_length", [](const Dual& d) { return to_np(d.dual_length); })
      .def_property_readonly("dual_area", [](const Dual& d) { return to_np(d.dual_area); })
      .def("dual_triangle_vertices", [](const Dual& d, int dt) {
        auto v = d.dual_tri_vertices(dt);
        return py::make_tuple(v[0], v[1], v[2]);
      });

  mod.def("dualize", &dualize, py::arg("mesh"), py::arg("center") = (int)BARYCENTER);
  mod.def("dec_differential", [](const Dual& d, int n) { return csc_tuple(dec_differential(d, n)); });
  mod.def("dec_boundary", [](const Dual& d, int n) { return csc_tuple(dec_boundary(d, n)); });
  mod.def("dec_dual_derivative", [](const Dual& d, int n) { return csc_tuple(dec_dual_derivative(d, n)); });
  mod.def("hodge_diag", [](const Dual& d, int k) { return to_np(hodge_diag(d, k)); });
  mod.def("inv_hodge_diag", [](const Dual& d, int k) { return to_np(inv_hodge_diag(d, k)); });
  mod.def("laplace_beltrami0", [](const Dual& d) { return csc_tuple(laplace_beltrami0(d)); });
  mod.def("wedge_dd_01_mat", [](const Dual& d) { return csc_tuple(wedge_dd_01_mat(d)); });
  mod.def("wedge_pd_01_mat", [](const Dual& d) { return csc_tuple(wedge_pd_01_mat(d)); });
  mod.def("flat_sharp_mat", [](const Dual& d) { return csc_tuple(flat_sharp_mat(d)); });
  mod.def("hodge_geometric1", [](const Dual& d) { return csc_tuple(hodge_geometric1(d)); });
  mod.def("hodge_geometric1_fast", [](const Dual& d) { return csc_tuple(hodge_geometric1_fast(d)); });
  mod.def("wedge02_cache", [](const Dual& d) {
    auto c = wedge02_cache(d);
    return py::make_tuple(to_np(c.verts), to_np(c.coeffs));
  });
  mod.def("wedge11_cache", [](const Dual& d) {
    auto c = wedge11_cache(d);
    return py::make_tuple(to_np(c.e), to_np(c.coeffs));
  });
  // kind: 1 = (0,1), 2 = (0,2), 11 = (1,1)
  mod.def("wedge", &run_wedge<double>);
  mod.def("wedge_f32", &run_wedge<float>);
  mod.def("c_wedge", [](int j, int k, int64_t n, py::array_t<int32_t, py::array::c_style | py::array::forcecast> p,
                        py::array_t<double, py::array::c_style | py::array::forcecast> c,
                        py::array_t<double, py::array::c_style | py::array::forcecast> a,
                        py::array_t<double, py::array::c_style | py::array::forcecast> b) {
    py::array_t<double> out(n);
    c_wedge<double>(j, k, n, p.data(), c.size() ? c.data() : nullptr, a.data(), b.data(), out.mutable_data());
    return out;
  });
  mod.def("c_wedge_f32", [](int j, int k, int64_t n, py::array_t<int32_t, py::array::c_style | py::array::forcecast> p,
                            py::array_t<float, py::array::c_style | py::array::forcecast> c,
                            py::array_t<float, py::array::c_style | py::array::forcecast> a,
                            py::array_t<float, py::array::c_style | py::array::forcecast> b) {
    py::array_t<float> out(n);
    c_wedge<float>(j, k, n, p.data(), c.size() ? c.data() : nullptr, a.data(), b.data(), out.mutable_data());
    return out;
  });
  mod.def("time_wedge", [](const Dual& d, int kind, py::array_t<double, py::array::c_style> a,
                           py::array_t<double, py::array::c_style> b, int reps) {
    // Seconds per evaluation of the cached kernel (caches built once, outside the timing).
    auto c02 = wedge02_cache(d);
    auto c11 = wedge11_cache(d);
    std::vector<double> out(std::max(d.ne, d.nt));
    auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < reps; ++r) {
      if (kind == 1) wedge01<double>(d, a.data(), b.data(), out.data());
      else if (kind == 2) wedge02<double>(d, c02, a.data(), b.data(), out.data());
      else wedge11<double>(d, c11, a.data(), b.data(), out.data());
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count() / reps;
  });

  mod.def("time_operators", [](const Dual& d, py::array_t<double, py::array::c_style | py::array::forcecast> f,
                                py::array_t<double, py::array::c_style | py::array::forcecast> a,
                                py::array_t<double, py::array::c_style | py::array::forcecast> b, int reps) {
    // Seconds per evaluation on the current thread count (caches and matrices built once, outside
    // the timing): ∧(0,1)(f, α), ∧(1,1)(α, β), ∧(0,2)(f, d1 α) (the d1 SpMV, then the wedge) and
    // Δ0 f = L f (the Laplacian SpMV: SparseArrays' column-order product on one thread, rows in
    // parallel on several).
    auto c02 = wedge02_cache(d);
    auto c11 = wedge11_cache(d);
    CSC d1 = dec_differential(d, 1), L = laplace_beltrami0(d);
    CSC d1t = transpose(d1), Lt = transpose(L);
    std::vector<double> oe(d.ne), ot(d.nt), ov(d.nv), t1(d.nt);
    auto time = [&](auto fn) {
      fn();
      auto t0 = std::chrono::steady_clock::now();
      for (int r = 0; r < reps; ++r) fn();
      auto t1c = std::chrono::steady_clock::now();
      return std::chrono::duration<double>(t1c - t0).count() / reps;
    };
    py::dict out;
    out["wedge01"] = time([&] { wedge01<double>(d, f.data(), a.data(), oe.data()); });
    out["wedge11"] = time([&] { wedge11<double>(d, c11, a.data(), b.data(), ot.data()); });
    out["wedge02_d1"] = time([&] {
      apply(d1, &d1t, a.data(), t1.data());
      wedge02<double>(d, c02, f.data(), t1.data(), ot.data());
    });
    out["laplacian"] = time([&] { apply(L, &Lt, f.data(), ov.data()); });
    return out;
  });
  mod.def("csc_matvec", [](py::tuple t, py::array_t<double, py::array::c_style | py::array::forcecast> x) {
    // y = A x in the column order of the reference's SparseMatrixCSC SpMV
    CSC a;
    a.colptr = from_np(t[0].cast<py::array_t<int32_t, py::array::c_style | py::array::forcecast>>());
    a.rowval = from_np(t[1].cast<py::array_t<int32_t, py::array::c_style | py::array::forcecast>>());
    a.nzval = from_np(t[2].cast<py::array_t<double, py::array::c_style | py::array::forcecast>>());
    auto shape = t[3].cast<py::tuple>();
    a.m = shape[0].cast<int>();
    a.n = shape[1].cast<int>();
    std::vector<double> y(a.m);
    spmv(a, x.data(), y.data());
    return to_np(y);
  });

  mod.attr("MLP_NPARAM") = MLP_NPARAM;
  mod.def("mlp_forward", [](py::array_t<float, py::array::c_style | py::array::forcecast> p,
                            py::array_t<float, py::array::c_style | py::array::forcecast> x, bool bf16) {
    std::vector<float> pv(p.data(), p.data() + p.size());
    int S = (int)(x.size() / MLP_IN);
    py::array_t<double> y(S);
    mlp_forward(pv, x.data(), S, y.mutable_data(), bf16);
    return y;
  }, py::arg("p"), py::arg("x"), py::arg("bf16") = true);
  mod.def("mlp_backward", [](py::array_t<float, py::array::c_style | py::array::forcecast> p,
                             py::array_t<float, py::array::c_style | py::array::forcecast> x,
                             py::array_t<double, py::array::c_style | py::array::forcecast> dy, bool bf16) {
    std::vector<float> pv(p.data(), p.data() + p.size());
    std::vector<double> g;
    mlp_backward(pv, x.data(), dy.data(), (int)dy.size(), g, bf16);
    return to_np(g);
  }, py::arg("p"), py::arg("x"), py::arg("dy"), py::arg("bf16") = true);

  // Multigrid
  mod.def("refine_binary", [](const Mesh& m, double radius) {
    Topo t = topo_of(m);
    auto pts = propagate_points_binary(t, m.pts, radius);
    return topo_to_mesh(refine_binary(t), pts);
  }, py::arg("mesh"), py::arg("radius") = 0.0);
  mod.def("subdivision_matrix", [](const Mesh& m) { return csc_tuple(subdivision_matrix_binary(topo_of(m))); });

  py::class_<MGData>(mod, "MGData")
      .def_property_readonly("nlevels", [](const MGData& md) { return (int)md.ops.size(); })
      .def("op", [](const MGData& md, int k) { return csc_tuple(md.ops.at(k)); })
      .def("restriction", [](const MGData& md, int k) { return csc_tuple(md.rs.at(k)); })
      .def("prolongation", [](const MGData& md, int k) { return csc_tuple(md.ps.at(k)); })
      .def("mesh", [](const MGData& md, int k) { return md.meshes.at(k); })
      .def("set_steps", [](MGData& md, int s) { for (auto& x : md.steps) x = s; })
      .def("set_level_steps", [](MGData& md, std::vector<int> s) {
        if (s.size() != md.steps.size()) throw std::runtime_error("set_level_steps: one entry per level");
        md.steps = s;
      });

  mod.def("mgdata_from_csc", [](py::list ops, py::list rs, py::list ps, std::vector<int> steps) {
    // MultigridData(g, r, p, s) (Multigrid.jl:538-546) from CSC tuples (0-based), finest first
    auto csc_of = [](py::handle h) {
      auto t = h.cast<py::tuple>();
      CSC a;
      a.colptr = from_np(t[0].cast<py::array_t<int32_t, py::array::c_style | py::array::forcecast>>());
      a.rowval = from_np(t[1].cast<py::array_t<int32_t, py::array::c_style | py::array::forcecast>>());
      a.nzval = from_np(t[2].cast<py::array_t<double, py::array::c_style | py::array::forcecast>>());
      auto shape = t[3].cast<py::tuple>();
      a.m = shape[0].cast<int>();
      a.n = shape[1].cast<int>();
      return a;
    };
    MGData md;
    for (auto h : ops) md.ops.push_back(csc_of(h));
    for (auto h : rs) md.rs.push_back(csc_of(h));
    for (auto h : ps) md.ps.push_back(csc_of(h));
    if (md.rs.size() + 1 != md.ops.size() || md.ps.size() + 1 != md.ops.size() || steps.size() != md.ops.size())
      throw std::runtime_error("mgdata_from_csc: level counts do not match");
    md.steps = steps;
    for (auto& a : md.ops) md.ops_t.push_back(transpose(a));
    for (auto& a : md.rs) md.rs_t.push_back(transpose(a));
    for (auto& a : md.ps) md.ps_t.push_back(transpose(a));
    return md;
  });
  mod.def("build_mg", &build_mg, py::arg("coarse"), py::arg("levels"), py::arg("center"),
          py::arg("shift"), py::arg("radius"), py::arg("steps") = 3, py::arg("galerkin") = false);
  mod.def("krylov_cg", [](const MGData& md, int lvl, py::array_t<double, py::array::c_style | py::array::forcecast> b,
                          py::array_t<double, py::array::c_style | py::array::forcecast> x0, int itmax) {
    return to_np(krylov_cg(md.ops.at(lvl), from_np(b), from_np(x0), itmax));
  });
  mod.def("mu_cycles", [](const MGData& md, py::array_t<double, py::array::c_style | py::array::forcecast> u,
                          py::array_t<double, py::array::c_style | py::array::forcecast> b, int cycles, int mu) {
    return to_np(mu_cycles(from_np(u), from_np(b), md, cycles, mu));
  });
  mod.def("full_multigrid", [](const MGData& md, py::array_t<double, py::array::c_style | py::array::forcecast> b,
                               int cycles, int mu) { return to_np(full_multigrid(from_np(b), md, cycles, mu)); });
  mod.def("plain_vcycles", [](const MGData& md, py::array_t<double, py::array::c_style | py::array::forcecast> u,
                              py::array_t<double, py::array::c_style | py::array::forcecast> b, int cycles,
                              int smoother, int pre, int post, double omega, double ratio,
                              std::vector<double> lmax) {
    PlainOpts o;
    o.smoother = smoother;
    o.pre = pre;
    o.post = post;
    o.omega = omega;
    o.cheb_ratio = ratio;
    o.lmax = lmax;
    auto x = from_np(u);
    auto bb = from_np(b);
    for (int c = 0; c < cycles; ++c) x = plain_vcycle(x, bb, md, o, 0);
    return to_np(x);
  });
}
