// Operator handle shared by ops.cu, mg.cu and the C ABI.
#pragma once
#include "mesh.cuh"

struct dec_op {
  decb::Mesh* m = nullptr;
  int kind = 0;
  dec_dtype dtype = DEC_F64;
  double shift = 0.0;
  int64_t rows = 0, cols = 0;
  decb::DArr<double> diag64;  // diagonal operators
  decb::DArr<float> diag32;
  int W = 0;                  // slot-major ELL width (Laplacian / Helmholtz / geometric ⋆1 / ♭♯)
  decb::DArr<int32_t> col;
  decb::DArr<double> val64;
  decb::DArr<float> val32;
  decb::DArr<double> kry;     // inverse geometric ⋆1: Krylov vectors, 1/diag and reduction scratch
  mutable unsigned tuned_at = 0;  // tuning-table version of ell_rows
  mutable int ell_rows = 1;       // rows per thread of the ELL apply (autotuned)
};

namespace decb {
void hodge_into(const Mesh& m, int k, bool inverse, DArr<double>& out);
void assemble_laplacian(const Mesh& m, double shift, int& W, DArr<int32_t>& col, DArr<double>& val);
int assemble_flat_sharp(const Mesh& m, DArr<int32_t>& idx, DArr<double>& val);  // wedge.cu
template <class T>
void cast_array(const DArr<double>& a, DArr<T>& b);

// Blocks of the residual-norm reduction (each block reduces a strided set of rows).
constexpr int kResidBlocks = DEC_RESIDUAL_BLOCKS;
constexpr int kResidThreads = 256;
// Residual-norm kernels on caller-provided scratch: partial holds 2 * kResidBlocks * nrhs doubles,
// dnorms 2 * nrhs.  Every partial slot is written before it is read, so the scratch needs no
// clearing between calls.
void launch_residual_norms(const dec_op& op, const double* x, const double* b, int nrhs, double* partial,
                           double* dnorms, cudaStream_t s);
}  // namespace decb
