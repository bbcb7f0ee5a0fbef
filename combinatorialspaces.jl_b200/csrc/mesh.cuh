// Device-resident mesh: flattened topology (SoA int32, 0-based), orientation signs,
// dual-complex geometry and the diagonal Hodge stars.
#pragma once
#include "common.cuh"

namespace decb {

struct Mesh {
  int nv = 0, ne = 0, nt = 0, center = 0;

  // Host copies of the (0-based) topology and points, for CSR exports and host-side products:
  // filled by build(); a level refined on the device fills them on first use (ensure_host).
  mutable std::vector<int32_t> h_ev0, h_ev1, h_te0, h_te1, h_te2;
  mutable std::vector<int8_t> h_eo, h_to;  // 1 / 0
  mutable std::vector<double> h_pts;       // 3 * nv
  mutable bool host_ready = false;

  // Topology.
  DArr<int32_t> ev0, ev1;            // ∂v0, ∂v1 per edge
  DArr<int32_t> te0, te1, te2;       // ∂e0, ∂e1, ∂e2 per triangle
  DArr<int32_t> tv0, tv1, tv2;       // triangle vertices (∂v1∂e1, ∂v0∂e2, ∂v0∂e1)
  DArr<int8_t> esign;                // edge orientation as ±1
  DArr<int8_t> tsign;                // triangle orientation as ±1

  // d1 rows with the three edges sorted by index (the CSC column order of the reference's
  // SpMV) and their ±1 coefficients packed in bits 0..2 (set = negative).
  DArr<int32_t> d1c0, d1c1, d1c2;
  DArr<uint8_t> d1neg;

  // Incidence (CSR over vertices / edges).
  //  v2t: vertex -> 3t+k for every triangle t whose k-th vertex it is, sorted by (k, t)
  //  e2t: edge   -> 3t+k for every triangle t whose ∂e_k it is, sorted by (k, t)
  //  v2e: vertex -> signed entry ±(e+1) of d0ᵀ (sign of d0[e, v]), sorted by e
  //  e2ts: edge  -> signed entry ±(t+1) of d1ᵀ, sorted by t
  DArr<int32_t> v2t_ptr, v2t, e2t_ptr, e2t, v2e_ptr, v2e, e2ts_ptr, e2ts;
  int max_v2e = 0;  // max vertex degree

  // Geometry (FP64), the reference's arrays.
  DArr<double> pts;          // 3 * nv
  DArr<double> length;       // ne
  DArr<double> area;         // nt
  DArr<double> tri_center;   // 3 * nt
  DArr<double> dual_area;    // 6 * nt, dual-triangle order (block i = schema i)
  DArr<double> dual_len_te;  // 3 * nt, |tri center - edge center of ∂e_k|, block k
  DArr<double> star0, star1, star2;  // diagonal Hodge stars

  void build(const dec_mesh_desc& desc);
  // The binary subdivision of coarse mesh c, built on the device (refine + propagate_points, new
  // vertices projected onto the sphere of `radius` when it is positive); dflip: device per coarse
  // triangle, nonzero where the children's orientation follows the flipped coarse one (or null).
  void refine_from(const Mesh& c, double radius, const int8_t* dflip, int center);
  void ensure_host() const;

 private:
  void derive();

 public:
};

}  // namespace decb

// The opaque handle of the C ABI.
struct dec_mesh {
  decb::Mesh m;
};
