// TEST INFRASTRUCTURE ONLY.
//
// CPU (FP64) restatement of the CombinatorialSpaces.jl (v0.10.1) DEC hot path: mesh
// construction, the dual complex and its geometry, the FastDEC wedge caches and kernels,
// d / boundary / dual d, the diagonal Hodge stars, the Laplace-Beltrami operator, the
// primal-dual and dual-dual wedge matrices, binary subdivision and the Multigrid.jl
// mu-cycles with a Krylov.jl-style CG smoother.  Every function names the reference
// file:line it restates.  It is the checker for the sm_100a library: only the test suite,
// the smoke check and the CPU-baseline leg of the benchmark may load it; the product
// library never links it.
//
// Indices are 0-based here; the reference is 1-based.  Orientation flags use
// 1 = true, 0 = false, -1 = unset (the reference's `nothing`).
#pragma once
#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

using i32 = int32_t;

enum Center { BARYCENTER = 0, CIRCUMCENTER = 1 };

void set_num_threads(int n);  // host threads for the wedge loops (default 1)
int num_threads();

// ---------------------------------------------------------------------------------------
// Primal 2D delta set (EmbeddedDeltaSet2D{Bool, Point3d}); src/SimplicialSets.jl:221-411.
// ---------------------------------------------------------------------------------------
struct Mesh {
  std::vector<double> pts;            // 3 * nv
  std::vector<i32> ev0, ev1;          // edge faces: ∂v0 (target), ∂v1 (source)
  std::vector<i32> te0, te1, te2;     // triangle faces ∂e0, ∂e1, ∂e2
  std::vector<int8_t> eo, to;         // edge / triangle orientation (1, 0, -1 = unset)
  std::unordered_map<uint64_t, i32> emap;  // directed (src, tgt) -> first edge

  int nv() const { return (int)(pts.size() / 3); }
  int ne() const { return (int)ev0.size(); }
  int nt() const { return (int)te0.size(); }

  int add_vertex(double x, double y, double z);
  int add_edge(int src, int tgt);                  // SimplicialSets.jl:143
  int get_edge(int src, int tgt);                  // SimplicialSets.jl:348-351
  int add_triangle(int src2_first, int src2_last, int tgt2, int8_t o);  // :323-324
  int glue_triangle(int v0, int v1, int v2, int8_t o = -1);              // :343-346
  int glue_sorted_triangle(int v0, int v1, int v2, int8_t o = -1);       // :361-364
  // triangle_vertices, SimplicialSets.jl:305-309: (∂v1∂e1, ∂v0∂e2, ∂v0∂e1)
  std::array<i32, 3> tri_vertices(int t) const {
    return {ev1[te1[t]], ev0[te2[t]], ev0[te1[t]]};
  }
  void rebuild_edge_map();
};

// orient!(s, Val(2)), SimplicialSets.jl:812-852.  Returns false (and leaves `to`
// untouched) when the check in the reference's DFS fails.
bool orient2(Mesh& m);

// Mesh generators.
Mesh triangulated_grid(double lx, double ly, double dx, double dy, bool compress);  // CombMeshes.jl:79-133
Mesh icosahedron();             // unit icosahedron, glue_sorted_triangle! + orient!
Mesh tri_345(bool orientation); // CombMeshes.jl:348-370
Mesh grid_345();                // CombMeshes.jl:378-398

// ---------------------------------------------------------------------------------------
// Embedded dual complex; src/DiscreteExteriorCalculus.jl:301-328, :545-608, :935-990.
// ---------------------------------------------------------------------------------------
struct Dual {
  Mesh mesh;                            // primal, with orientations filled in
  int nv = 0, ne = 0, nt = 0;
  std::vector<i32> dv0, dv1;            // dual edges D_∂v0, D_∂v1  (2ne + 6nt)
  std::vector<i32> dte0, dte1, dte2;    // dual triangles D_∂e0..2  (6nt)
  std::vector<int8_t> de_orient;        // D_edge_orientation
  std::vector<int8_t> dt_orient;        // D_tri_orientation
  std::vector<double> dual_point;       // 3 * (nv + ne + nt)
  std::vector<double> length, area, dual_length, dual_area;
  int vertex_center(int v) const { return v; }
  int edge_center(int e) const { return nv + e; }
  int tri_center(int t) const { return nv + ne + t; }
  // dual_triangle_vertices, DiscreteExteriorCalculus.jl:224-228
  std::array<i32, 3> dual_tri_vertices(int dt) const {
    return {dv1[dte1[dt]], dv1[dte0[dt]], dv0[dte0[dt]]};
  }
};

Dual dualize(const Mesh& m, int center);

// ---------------------------------------------------------------------------------------
// Sparse matrices in the reference's SparseMatrixCSC layout.
// ---------------------------------------------------------------------------------------
struct CSC {
  int m = 0, n = 0;
  std::vector<i32> colptr, rowval;
  std::vector<double> nzval;
};
CSC sparse_coo(int m, int n, const std::vector<i32>& I, const std::vector<i32>& J,
               const std::vector<double>& V);  // SparseArrays.sparse (duplicates summed)
CSC transpose(const CSC& a);
CSC scale_rows(const std::vector<double>& d, const CSC& a);   // Diagonal * sparse
CSC scale_cols(const CSC& a, const std::vector<double>& d);   // sparse * Diagonal
CSC spgemm(const CSC& a, const CSC& b);                        // sparse * sparse
CSC add_identity(const CSC& a, double c);                      // A + c*I
void spmv(const CSC& a, const double* x, double* y);           // y = A x
void spmv_t(const CSC& a, const double* x, double* y);         // y = A' x

// FastDEC operators, src/FastDEC.jl:426-557 and :559-757.
CSC dec_differential(const Dual& d, int n);       // :468-469, derivbound :471-524
CSC dec_boundary(const Dual& d, int n);           // :433-437
CSC dec_dual_derivative(const Dual& d, int n);    // :443-453
std::vector<double> hodge_diag(const Dual& d, int k);      // :580-604
std::vector<double> inv_hodge_diag(const Dual& d, int k);  // :732-737
// fast_laplace_beltrami, test/Multigrid.jl:46-48 (= ∇²(0), DiscreteExteriorCalculus.jl:1889)
CSC laplace_beltrami0(const Dual& d);

// Wedge caches (FastDEC.jl:42-93) and kernels (:159-191), evaluated in T with the
// coefficients computed in FP64 and then cast to T (cache_wedge cast_float, :147-155).
struct Wedge02Cache { std::vector<i32> verts; std::vector<double> coeffs; };  // 6 x nt
struct Wedge11Cache { std::vector<i32> e; std::vector<double> coeffs; };      // 3 x nt
Wedge02Cache wedge02_cache(const Dual& d);
Wedge11Cache wedge11_cache(const Dual& d);
template <class T> void wedge01(const Dual& d, const T* f, const T* a, T* out);
template <class T> void wedge02(const Dual& d, const Wedge02Cache& c, const T* f, const T* a, T* out);
template <class T> void wedge11(const Dual& d, const Wedge11Cache& c, const T* a, const T* b, T* out);
template <class T>
void c_wedge(int j, int k, int64_t n, const i32* p, const T* c, const T* a, const T* b, T* res);

// Primal-dual / dual-dual wedge matrices, FastDEC.jl:293-347, and ♭♯ (DEC.jl:1992).
CSC wedge_dd_01_mat(const Dual& d);
CSC wedge_pd_01_mat(const Dual& d);
CSC flat_sharp_mat(const Dual& d);
// ⋆1 with GeometricHodge (the reference default for 1-forms in 2D), DiscreteExteriorCalculus.jl:1680-1731.
CSC hodge_geometric1(const Dual& d);
// FastDEC's dec_hodge_star(Val(1), sd, GeometricHodge()), FastDEC.jl:660-716 (the GPU's formulation).
CSC hodge_geometric1_fast(const Dual& d);

// ---------------------------------------------------------------------------------------
// Multigrid.jl
// ---------------------------------------------------------------------------------------
struct Topo {  // MeshTopology, Multigrid.jl:27-42
  int nv = 0, ne = 0, nt = 0;
  std::vector<i32> ev0, ev1, te0, te1, te2;
};
Topo topo_of(const Mesh& m);
Topo refine_binary(const Topo& t);                       // :130-183
std::vector<double> propagate_points_binary(const Topo& t, const std::vector<double>& pts,
                                            double project_radius);  // :111-122 (+ projection)
CSC subdivision_matrix_binary(const Topo& t);           // :191-219
CSC make_restriction(const CSC& s);                      // :595-612
Mesh topo_to_mesh(const Topo& t, const std::vector<double>& pts);    // :49-64

struct MGData {  // MultigridData, :538-553 (finest level first)
  std::vector<CSC> ops, rs, ps;
  std::vector<CSC> ops_t, rs_t, ps_t;  // transposes: row access for the threaded CPU baseline
  std::vector<int> steps;
  std::vector<Mesh> meshes;  // finest first, orientations as dualize left them
};
// _build_multigrid(DirectMode or GalerkinMode, BinarySubdivision), :740-797, with op = L + shift*I.
MGData build_mg(const Mesh& coarse, int levels, int center, double shift, double project_radius,
                int steps, bool galerkin = false);

// Krylov.jl cg(A, b, x0; itmax) (warm start, atol = rtol = sqrt(eps)).
std::vector<double> krylov_cg(const CSC& A, const std::vector<double>& b,
                              const std::vector<double>& x0, int itmax, const CSC* At = nullptr);
// y = A x; with more than one host thread and At (the CSC of Aᵀ) given, rows run in parallel.
void apply(const CSC& A, const CSC* At, const double* x, double* y);
std::vector<double> mu_cycle(const std::vector<double>& u, const std::vector<double>& b,
                             const MGData& md, int lvl, int mu);  // :857-872
std::vector<double> mu_cycles(std::vector<double> u, const std::vector<double>& b,
                              const MGData& md, int cycles, int mu);  // :819-824
std::vector<double> full_multigrid(const std::vector<double>& b, const MGData& md, int cycles,
                                   int mu);  // :830-855

// The project's plain V-cycle (stationary smoother + dense coarsest solve): the CPU
// statement of the GPU "plain" algorithm, used to check it.
struct PlainOpts {
  int smoother = 1;       // 0 = damped Jacobi, 1 = Chebyshev-Jacobi
  int pre = 3, post = 3;  // sweeps / Chebyshev degree
  double omega = 0.8;
  double cheb_ratio = 4.0;            // lower bound = upper / ratio
  std::vector<double> lmax;           // per level upper eigenvalue bound of D^-1 A
};
std::vector<double> plain_vcycle(const std::vector<double>& u, const std::vector<double>& b,
                                 const MGData& md, const PlainOpts& o, int lvl = 0);
std::vector<double> dense_solve(const CSC& A, const std::vector<double>& b);  // LU, partial pivot

}  // namespace orc

namespace orc {
// ---------------------------------------------------------------------------------------------
// The learned smoother's per-vertex MLP 16 -> 64 -> 64 -> 1 (ReLU), as the library evaluates it:
// features, W1 and W2 rounded to BF16 (round to nearest even), the first hidden layer rounded
// to BF16 before the second product, FP32-or-wider accumulation.  Parameters are one flat vector:
// W1[64][16] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3.  Gradients flow to the FP32 master
// parameters through the rounding (straight-through).
// ---------------------------------------------------------------------------------------------
constexpr int MLP_IN = 16, MLP_H = 64;
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1;
float round_bf16(float x);
// bf16 = false: no rounding, FP64 throughout (for finite-difference checks of the backward pass)
void mlp_forward(const std::vector<float>& p, const float* x, int S, double* y, bool bf16 = true);
// grad += d(Σ_s dy_s y_s)/dp
void mlp_backward(const std::vector<float>& p, const float* x, const double* dy, int S, std::vector<double>& grad,
                  bool bf16 = true);
}  // namespace orc
