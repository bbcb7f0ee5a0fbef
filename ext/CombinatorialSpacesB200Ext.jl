"""
    CombinatorialSpacesB200Ext

The `Val(:B200)` backend of CombinatorialSpaces.jl: the entry points of
`ext/CombinatorialSpacesCUDAExt.jl` (cache_wedge, dec_boundary, dec_dual_derivative,
dec_differential, dec_hodge_star, dec_inv_hodge_star) and of the wedge products and multigrid
solvers, each `ccall`ing `libdec_b200.so` (declared in `include/dec_b200.h`) on CUDA.jl device
arrays.  The library path comes from the environment variable `DEC_B200_LIB` (default:
`libdec_b200.so` on the loader path).

Load it as a package extension with the weak dependency CUDA (Project.toml: `[extensions]
CombinatorialSpacesB200Ext = "CUDA"`).  Forms are CuArrays in the reference's element order, indices
1-based: the library takes the Julia arrays as they are.  Every call is enqueued on CUDA.jl's
task-local stream.  Device handles are released by finalizers.
"""
module CombinatorialSpacesB200Ext

using CombinatorialSpaces
using CombinatorialSpaces.DiscreteExteriorCalculus: DiscreteHodge, DiagonalHodge, GeometricHodge
using CUDA
using LinearAlgebra
using SparseArrays
import CombinatorialSpaces: cache_wedge, dec_wedge_product, dec_wedge_product_pd, dec_wedge_product_dp,
  dec_wedge_product_dd, dec_boundary, dec_differential, dec_dual_derivative, dec_hodge_star,
  dec_inv_hodge_star, multigrid_vcycles, multigrid_wcycles, full_multigrid

const lib = get(ENV, "DEC_B200_LIB", "libdec_b200.so")

# ---- C structs (include/dec_b200.h) --------------------------------------------------------

struct DecMeshDesc
  nv::Int32; ne::Int32; nt::Int32; index_base::Int32
  points::Ptr{Float64}
  e_v0::Ptr{Int32}; e_v1::Ptr{Int32}
  t_e0::Ptr{Int32}; t_e1::Ptr{Int32}; t_e2::Ptr{Int32}
  edge_orientation::Ptr{Int8}; tri_orientation::Ptr{Int8}
  center::Int32
end

struct DecCsc
  m::Int32; n::Int32; index_base::Int32
  colptr::Ptr{Int32}; rowval::Ptr{Int32}; nzval::Ptr{Float64}
end

mutable struct DecMGOptions
  levels::Int32; center::Int32; project_radius::Float64; shift::Float64
  smoother::Int32; pre::Int32; post::Int32; omega::Float64; cheb_ratio::Float64
  coarse_solver::Int32; precision::Int32; rhs_block::Int32; mu::Int32; inner_cycles::Int32
  reorder::Int32; coarse_max::Int32; fallback_rho::Float64; galerkin::Int32; device_loop::Int32
  DecMGOptions() = new()
end

mutable struct DecSolveReport
  iterations::Int32; converged::Int32; max_rel_residual::Float64; seconds::Float64
  launches::Int64; rhs_block::Int32; fallback_iteration::Int32
  DecSolveReport() = new(0, 0, 0.0, 0.0, 0, 0, -1)
end

const DEC_F64, DEC_F32 = Int32(0), Int32(1)
const DEC_BARYCENTER, DEC_CIRCUMCENTER = Int32(0), Int32(1)
const DEC_WEDGE_PP, DEC_WEDGE_PD, DEC_WEDGE_DP, DEC_WEDGE_DD = Int32(0), Int32(1), Int32(2), Int32(3)
const DEC_OP_D0, DEC_OP_D1, DEC_OP_BOUNDARY1, DEC_OP_BOUNDARY2 = Int32(0), Int32(1), Int32(2), Int32(3)
const DEC_OP_DUAL_D0, DEC_OP_DUAL_D1 = Int32(4), Int32(5)
const DEC_OP_STAR0, DEC_OP_INV_STAR0 = Int32(6), Int32(9)
const DEC_OP_STAR1_GEOMETRIC, DEC_OP_INV_STAR1_GEOMETRIC = Int32(14), Int32(15)
const DEC_SMOOTH_JACOBI, DEC_SMOOTH_CHEBYSHEV, DEC_SMOOTH_CG = Int32(0), Int32(1), Int32(2)

check(st) = st == 0 || error("libdec_b200: " * unsafe_string(ccall((:dec_last_error, lib), Cstring, ())))
dtype_code(::Type{Float64}) = DEC_F64
dtype_code(::Type{Float32}) = DEC_F32
stream_ptr() = reinterpret(Ptr{Cvoid}, CUDA.stream().handle)

# ---- device meshes -------------------------------------------------------------------------

mutable struct B200Mesh
  h::Ptr{Cvoid}
  nv::Int; ne::Int; nt::Int
end

# One device mesh per (dual complex, centre): the flattened SoA topology, the dual geometry and
# FastDEC's coefficient caches live on the device for as long as the complex does.
const MESHES = WeakKeyDict{Any, Dict{Int32, B200Mesh}}()

function b200_mesh(sd::HasDeltaSet, center::Int32=DEC_BARYCENTER)
  per = get!(() -> Dict{Int32, B200Mesh}(), MESHES, sd)
  haskey(per, center) && return per[center]
  pts = zeros(Float64, 3, nv(sd))
  for (i, p) in enumerate(sd[:point])
    for k in 1:min(3, length(p)); pts[k, i] = p[k]; end
  end
  v0, v1 = Int32.(sd[:∂v0]), Int32.(sd[:∂v1])
  t0, t1, t2 = Int32.(sd[:∂e0]), Int32.(sd[:∂e1]), Int32.(sd[:∂e2])
  eo, to = Int8.(sd[:edge_orientation]), Int8.(sd[:tri_orientation])
  h = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve pts v0 v1 t0 t1 t2 eo to begin
    d = DecMeshDesc(nv(sd), ne(sd), ntriangles(sd), 1, pointer(pts), pointer(v0), pointer(v1),
                    pointer(t0), pointer(t1), pointer(t2), pointer(eo), pointer(to), center)
    check(ccall((:dec_mesh_create, lib), Cint, (Ref{DecMeshDesc}, Ref{Ptr{Cvoid}}), d, h))
  end
  m = B200Mesh(h[], nv(sd), ne(sd), ntriangles(sd))
  finalizer(x -> ccall((:dec_mesh_destroy, lib), Cint, (Ptr{Cvoid},), x.h), m)
  per[center] = m
end

# ---- operators ----------------------------------------------------------------------------

"""A DEC operator on the device: `op * x` and `mul!(y, op, x)` on CuVectors."""
mutable struct B200Operator{T}
  h::Ptr{Cvoid}
  rows::Int; cols::Int
  owner::Any  # keeps the mesh alive
end

function B200Operator{T}(mesh::B200Mesh, kind::Int32, shift::Float64=0.0) where T
  h = Ref{Ptr{Cvoid}}(C_NULL)
  check(ccall((:dec_op_create, lib), Cint, (Ptr{Cvoid}, Int32, Float64, Int32, Ref{Ptr{Cvoid}}),
              mesh.h, kind, shift, dtype_code(T), h))
  wrap_op(T, h[], mesh)
end

function wrap_op(::Type{T}, h::Ptr{Cvoid}, owner) where T
  r, c = Ref{Int64}(0), Ref{Int64}(0)
  check(ccall((:dec_op_shape, lib), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}), h, r, c))
  op = B200Operator{T}(h, r[], c[], owner)
  finalizer(x -> ccall((:dec_op_destroy, lib), Cint, (Ptr{Cvoid},), x.h), op)
  op
end

"""A caller's SparseMatrixCSC as a device operator (dec_op_create_csc)."""
function B200Operator{T}(A::SparseMatrixCSC) where T
  cp, rv, nz = Int32.(A.colptr), Int32.(A.rowval), Float64.(A.nzval)
  h = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve cp rv nz begin
    c = DecCsc(size(A, 1), size(A, 2), 1, pointer(cp), pointer(rv), pointer(nz))
    check(ccall((:dec_op_create_csc, lib), Cint, (Ref{DecCsc}, Int32, Ref{Ptr{Cvoid}}), c, dtype_code(T), h))
  end
  wrap_op(T, h[], nothing)
end

Base.size(op::B200Operator) = (op.rows, op.cols)
Base.size(op::B200Operator, k::Int) = size(op)[k]
Base.eltype(::B200Operator{T}) where T = T

function LinearAlgebra.mul!(y::CuVector{T}, op::B200Operator{T}, x::CuVector{T}, α::Number=true, β::Number=false) where T
  length(x) == op.cols && length(y) == op.rows || throw(DimensionMismatch("operator $(size(op)) on $(length(x))"))
  check(ccall((:dec_op_apply, lib), Cint, (Ptr{Cvoid}, CuPtr{T}, CuPtr{T}, Float64, Float64, Ptr{Cvoid}),
              op.h, x, y, Float64(α), Float64(β), stream_ptr()))
  y
end
Base.:*(op::B200Operator{T}, x::CuVector{T}) where T = mul!(CUDA.zeros(T, op.rows), op, x)

float_type_of(::EmbeddedDeltaDualComplex2D{Bool, F, P}) where {F, P} = F
center_of(sd) = DEC_BARYCENTER  # dualize(s, Barycenter()) unless the complex says otherwise

# dec_differential / dec_boundary / dec_dual_derivative(n, sd, Val(:CUDA)), CUDAExt.jl:30-61
dec_differential(n::Int, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}) =
  B200Operator{float_type_of(sd)}(b200_mesh(sd, center_of(sd)), n == 0 ? DEC_OP_D0 : DEC_OP_D1)
dec_boundary(n::Int, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}) =
  B200Operator{float_type_of(sd)}(b200_mesh(sd, center_of(sd)), n == 1 ? DEC_OP_BOUNDARY1 : DEC_OP_BOUNDARY2)
dec_dual_derivative(n::Int, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}) =
  B200Operator{float_type_of(sd)}(b200_mesh(sd, center_of(sd)), n == 0 ? DEC_OP_DUAL_D0 : DEC_OP_DUAL_D1)

# dec_hodge_star / dec_inv_hodge_star(n, sd, h, Val(:CUDA)), CUDAExt.jl:70-96: the diagonal stars
# are CuArrays, the geometric ⋆1 an operator, its inverse a closure (a BiCGSTAB solve to 1e-14
# in the library where the CUDA extension runs Krylov.gmres)
dec_hodge_star(n::Int, sd::HasDeltaSet, h::DiscreteHodge, ::Val{:B200}) = dec_hodge_star(Val(n), sd, h, Val(:B200))
function dec_hodge_star(::Val{n}, sd::EmbeddedDeltaDualComplex2D, ::DiagonalHodge, ::Val{:B200}) where n
  T = float_type_of(sd)
  m = b200_mesh(sd, center_of(sd))
  out = CUDA.zeros(T, n == 0 ? m.nv : n == 1 ? m.ne : m.nt)
  check(ccall((:dec_hodge_diag, lib), Cint, (Ptr{Cvoid}, Int32, Int32, Int32, CuPtr{T}, Ptr{Cvoid}),
              m.h, n, 0, dtype_code(T), out, stream_ptr()))
  out
end
dec_hodge_star(::Val{1}, sd::EmbeddedDeltaDualComplex2D, ::GeometricHodge, ::Val{:B200}) =
  B200Operator{float_type_of(sd)}(b200_mesh(sd, center_of(sd)), DEC_OP_STAR1_GEOMETRIC)
dec_hodge_star(::Val{n}, sd::EmbeddedDeltaDualComplex2D, ::GeometricHodge, ::Val{:B200}) where n =
  dec_hodge_star(Val(n), sd, DiagonalHodge(), Val(:B200))

dec_inv_hodge_star(n::Int, sd::HasDeltaSet, h::DiscreteHodge, ::Val{:B200}) =
  dec_inv_hodge_star(Val(n), sd, h, Val(:B200))
function dec_inv_hodge_star(::Val{n}, sd::EmbeddedDeltaDualComplex2D, ::DiagonalHodge, ::Val{:B200}) where n
  T = float_type_of(sd)
  m = b200_mesh(sd, center_of(sd))
  out = CUDA.zeros(T, n == 0 ? m.nv : n == 1 ? m.ne : m.nt)
  check(ccall((:dec_hodge_diag, lib), Cint, (Ptr{Cvoid}, Int32, Int32, Int32, CuPtr{T}, Ptr{Cvoid}),
              m.h, n, 1, dtype_code(T), out, stream_ptr()))
  out
end
function dec_inv_hodge_star(::Val{1}, sd::EmbeddedDeltaDualComplex2D, ::GeometricHodge, ::Val{:B200})
  op = B200Operator{Float64}(b200_mesh(sd, center_of(sd)), DEC_OP_INV_STAR1_GEOMETRIC)
  x -> op * x
end
dec_inv_hodge_star(::Val{n}, sd::EmbeddedDeltaDualComplex2D, ::GeometricHodge, ::Val{:B200}) where n =
  dec_inv_hodge_star(Val(n), sd, DiagonalHodge(), Val(:B200))

# ---- wedge products -------------------------------------------------------------------------

# cache_wedge(Val(m), Val(n), sd, Val(:CUDA)) (CUDAExt.jl:16-21): the same caches, on the device
cache_wedge(::Val{m}, ::Val{n}, sd::EmbeddedDeltaDualComplex2D{Bool, float_type, _p}, ::Val{:B200},
            arr_cons=CuArray, cast_float=nothing) where {float_type, _p, m, n} =
  cache_wedge(m, n, sd, float_type, arr_cons, cast_float)

mutable struct B200WedgePlan{T}
  h::Ptr{Cvoid}
  len_a::Int; len_b::Int; len_out::Int
  mesh::B200Mesh
end

function wedge_plan(::Type{T}, sd, kind::Int32, m::Int, n::Int) where T
  mesh = b200_mesh(sd, center_of(sd))
  h = Ref{Ptr{Cvoid}}(C_NULL)
  check(ccall((:dec_wedge_plan_create, lib), Cint, (Ptr{Cvoid}, Int32, Int32, Int32, Int32, Ref{Ptr{Cvoid}}),
              mesh.h, kind, m, n, dtype_code(T), h))
  la, lb, lo = Ref{Int64}(0), Ref{Int64}(0), Ref{Int64}(0)
  check(ccall((:dec_wedge_lengths, lib), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}, Ref{Int64}), h[], la, lb, lo))
  p = B200WedgePlan{T}(h[], la[], lb[], lo[], mesh)
  finalizer(x -> ccall((:dec_wedge_plan_destroy, lib), Cint, (Ptr{Cvoid},), x.h), p)
  p
end

function apply!(res::CuVector{T}, p::B200WedgePlan{T}, a::CuVector{T}, b::CuVector{T}) where T
  length(a) == p.len_a && length(b) == p.len_b && length(res) == p.len_out ||
    throw(DimensionMismatch("wedge product on forms of lengths $(length(a)), $(length(b))"))
  check(ccall((:dec_wedge_apply, lib), Cint, (Ptr{Cvoid}, CuPtr{T}, CuPtr{T}, CuPtr{T}, Ptr{Cvoid}),
              p.h, a, b, res, stream_ptr()))
  res
end

# dec_wedge_product(m, n, sd, Val(:CUDA), arr_cons, cast_float) (FastDEC.jl:255-289): a closure
# (α, β) -> α ∧ β on CuArrays, (0,1) (1,0) (0,2) (2,0) (1,1)
function dec_wedge_product(::Val{m}, ::Val{n}, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}, arr_cons=CuArray,
                           cast_float=nothing) where {m, n}
  T = cast_float === nothing ? float_type_of(sd) : cast_float
  p = wedge_plan(T, sd, DEC_WEDGE_PP, m, n)
  (α, β) -> apply!(CUDA.zeros(T, p.len_out), p, α, β)
end
dec_wedge_product(m::Int, n::Int, sd::EmbeddedDeltaDualComplex2D, b::Val{:B200}, args...) =
  dec_wedge_product(Val(m), Val(n), sd, b, args...)

# dec_wedge_product_pd / _dp / _dd (FastDEC.jl:293-401)
dec_wedge_product_pd(m::Int, n::Int, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}) =
  (p = wedge_plan(float_type_of(sd), sd, DEC_WEDGE_PD, m, n); (α, β) -> apply!(CUDA.zeros(eltype(α), p.len_out), p, α, β))
dec_wedge_product_dp(m::Int, n::Int, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}) =
  (p = wedge_plan(float_type_of(sd), sd, DEC_WEDGE_DP, m, n); (α, β) -> apply!(CUDA.zeros(eltype(α), p.len_out), p, α, β))
dec_wedge_product_dd(m::Int, n::Int, sd::EmbeddedDeltaDualComplex2D, ::Val{:B200}) =
  (p = wedge_plan(float_type_of(sd), sd, DEC_WEDGE_DD, m, n); (α, β) -> apply!(CUDA.zeros(eltype(α), p.len_out), p, α, β))

"""
    b200_c_wedge_product!(Val(j), Val(k), res, α, β, p, c)

dec_c_wedge_product!(Val(j), Val(k), res, α, β, p, c) (FastDEC.jl:217-232) on a `cache_wedge`
output on the device, (j, k) = (0,1), (0,2), (0,3), (1,1), (2,1): the Julia matrices go in as they
are (column-major, 1-based).
"""
function b200_c_wedge_product!(::Val{j}, ::Val{k}, res::CuVector{T}, α::CuVector{T}, β::CuVector{T},
                               p::CuMatrix{Int32}, c) where {j, k, T}
  cptr = c === nothing ? CuPtr{T}(0) : pointer(c)
  check(ccall((:dec_c_wedge_apply, lib), Cint,
              (Int32, Int32, Int64, CuPtr{Int32}, CuPtr{T}, Int32, CuPtr{T}, CuPtr{T}, CuPtr{T}, Int32, Ptr{Cvoid}),
              j, k, length(res), p, cptr, dtype_code(T), α, β, res, 1, stream_ptr()))
  res
end

# ---- multigrid ------------------------------------------------------------------------------

"""A multigrid hierarchy on the device; `steps`, smoother and cycle options as `dec_mg_options`."""
mutable struct B200MultigridData
  h::Ptr{Cvoid}
  n::Int
  nlevels::Int
end

function options(; kw...)
  o = DecMGOptions()
  ccall((:dec_mg_default_options, lib), Cvoid, (Ref{DecMGOptions},), o)
  for (k, v) in kw
    setfield!(o, k, convert(fieldtype(DecMGOptions, k), v))
  end
  o
end

function wrap_mg(h::Ptr{Cvoid}, nlevels::Int)
  nv = Ref{Int64}(0)
  check(ccall((:dec_mg_level_info, lib), Cint, (Ptr{Cvoid}, Int32, Ref{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}),
              h, 0, nv, C_NULL, C_NULL, C_NULL))
  md = B200MultigridData(h, nv[], nlevels)
  finalizer(x -> ccall((:dec_mg_destroy, lib), Cint, (Ptr{Cvoid},), x.h), md)
  md
end

function csc_desc(A::SparseMatrixCSC, keep::Vector{Any})
  cp, rv, nz = Int32.(A.colptr), Int32.(A.rowval), Float64.(A.nzval)
  push!(keep, cp, rv, nz)
  DecCsc(size(A, 1), size(A, 2), 1, pointer(cp), pointer(rv), pointer(nz))
end
csc_desc(A::Transpose{<:Any, <:SparseMatrixCSC}, keep::Vector{Any}) = csc_desc(SparseMatrixCSC(A), keep)
csc_desc(A::AbstractMatrix, keep::Vector{Any}) = csc_desc(sparse(A), keep)

"""
    B200MultigridData(md::MultigridData; smoother=DEC_SMOOTH_CG, kw...)

MultigridData(g, r, p, s) (src/Multigrid.jl:538-546) on the device: the reference's operators,
restrictions, prolongations and per-level steps, whatever `op` or scheme built them
(dec_mg_create_from_csc).  The default smoother is the reference's Krylov cg.
"""
function B200MultigridData(md::MultigridData; smoother=DEC_SMOOTH_CG, kw...)
  nl = length(md.operators)
  keep = Any[]
  GC.@preserve keep begin
    ops = [csc_desc(A, keep) for A in md.operators]
    rs = [csc_desc(R, keep) for R in md.restrictions]
    ps = [csc_desc(P, keep) for P in md.prolongations]
    steps = Int32.(md.steps)
    o = options(; smoother=smoother, kw...)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:dec_mg_create_from_csc, lib), Cint,
                (Int32, Ptr{DecCsc}, Ptr{DecCsc}, Ptr{DecCsc}, Ptr{Int32}, Ref{DecMGOptions}, Ref{Ptr{Cvoid}}),
                nl, ops, rs, ps, steps, o, h))
  end
  wrap_mg(h[], nl)
end

"""
    b200_multigrid(s, levels; shift=0.0, project_radius=0.0, kw...)

MultigridData(s, BinarySubdivision(), levels, s -> ∇²(0, s) + shift I, steps) with the hierarchy built
on the device from the coarse mesh `s` (dec_mg_create): refinement, circumcentric duals (the
reference's default), operators, transfers.
"""
function b200_multigrid(s::HasDeltaSet, levels::Int; shift=0.0, project_radius=0.0, kw...)
  pts = zeros(Float64, 3, nv(s))
  for (i, p) in enumerate(s[:point])
    for k in 1:min(3, length(p)); pts[k, i] = p[k]; end
  end
  v0, v1 = Int32.(s[:∂v0]), Int32.(s[:∂v1])
  t0, t1, t2 = Int32.(s[:∂e0]), Int32.(s[:∂e1]), Int32.(s[:∂e2])
  o = options(; levels=levels, shift=shift, project_radius=project_radius, kw...)
  h = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve pts v0 v1 t0 t1 t2 begin
    d = DecMeshDesc(nv(s), ne(s), ntriangles(s), 1, pointer(pts), pointer(v0), pointer(v1),
                    pointer(t0), pointer(t1), pointer(t2), C_NULL, C_NULL, o.center)
    check(ccall((:dec_mg_create, lib), Cint, (Ref{DecMeshDesc}, Ref{DecMGOptions}, Ref{Ptr{Cvoid}}), d, o, h))
  end
  wrap_mg(h[], levels + 1)
end

"""MultigridData.steps per level (pre = post = steps[k]); dec_mg_set_level_steps."""
function set_steps!(md::B200MultigridData, steps::AbstractVector{<:Integer})
  length(steps) == md.nlevels || throw(ArgumentError("one steps entry per level"))
  s = Int32.(steps)
  check(ccall((:dec_mg_set_level_steps, lib), Cint, (Ptr{Cvoid}, Ptr{Int32}), md.h, s))
  md
end

function cycles!(md::B200MultigridData, u::CuVecOrMat{Float64}, b::CuVecOrMat{Float64}, cycles::Int)
  nrhs = size(b, 2)
  size(u) == size(b) && size(b, 1) == md.n || throw(DimensionMismatch("multigrid on $(size(b))"))
  check(ccall((:dec_mg_cycles, lib), Cint, (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int32, Int32, Ptr{Cvoid}),
              md.h, u, b, nrhs, cycles, stream_ptr()))
  u
end

# multigrid_vcycles / multigrid_wcycles (src/Multigrid.jl:814-824): the cycle type is the hierarchy's
# `mu` option (1 = V, 2 = W); `alg` is the smoother chosen when the hierarchy was built
multigrid_vcycles(u::CuVecOrMat{Float64}, b::CuVecOrMat{Float64}, md::B200MultigridData, cycles, alg=nothing) =
  cycles!(md, copy(u), b, cycles)
multigrid_wcycles(u::CuVecOrMat{Float64}, b::CuVecOrMat{Float64}, md::B200MultigridData, cycles, alg=nothing) =
  cycles!(md, copy(u), b, cycles)

# full_multigrid(b, md, cycles, alg, μ) (src/Multigrid.jl:826-855)
function full_multigrid(b::CuVecOrMat{Float64}, md::B200MultigridData, cycles, alg=nothing, μ=1)
  u = similar(b)
  check(ccall((:dec_mg_full_multigrid, lib), Cint, (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int32, Int32, Ptr{Cvoid}),
              md.h, u, b, size(b, 2), cycles, stream_ptr()))
  u
end

"""
    b200_solve!(md, u, b; rtol=1e-8, max_iters=100, from_zero=false)

V-cycles inside FP64 iterative refinement to ‖b - A u‖ / ‖b‖ ≤ rtol for every column of b
(dec_mg_solve / dec_mg_solve_from_zero); returns (u, report).
"""
function b200_solve!(md::B200MultigridData, u::CuVecOrMat{Float64}, b::CuVecOrMat{Float64};
                     rtol=1e-8, max_iters=100, from_zero=false)
  rep = DecSolveReport()
  f = from_zero ? :dec_mg_solve_from_zero : :dec_mg_solve
  st = ccall((f, lib), Cint,
             (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int32, Float64, Int32, Ref{DecSolveReport}, Ptr{Cvoid}),
             md.h, u, b, size(b, 2), rtol, max_iters, rep, stream_ptr())
  st == 4 || check(st)  # DEC_ERR_NOT_CONVERGED leaves the report to say how far it got
  u, rep
end

end
