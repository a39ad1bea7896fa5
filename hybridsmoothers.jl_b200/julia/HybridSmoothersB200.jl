# Julia binding of libhsb200 (include/hsb200.h): the drop-in for
# HybridSmoothers.jl's L1GS / Chebyshev apply path on a B200.
#
# It keeps the reference's user-facing calls
#     L1GSPrecBuilder(CUDABackend(); threads, blocks)(A, partsize; isSymA, η, sweep, cache_strategy)
#     LinearSolve.ldiv!(y, P, x),  P \ x
#     _build_smoother(ChebyshevFourth(; degree, backend), A),  smooth!(x, s, b)
# and reaches the GPU only through `ccall` into libhsb200.so.  CuArray
# arguments pass their raw device pointers (no copies); host Vectors take the
# library's host entry point (copy in, sweep, copy out), like the reference's
# generic ldiv! (src/l1_gauss_seidel.jl:367-384).
#
# Not exercised in this repository's test suite: Julia is not installed in the
# build image.  The same C entry points are exercised from Python
# (tests/test_*_gpu.py).
module HybridSmoothersB200

using SparseArrays: SparseMatrixCSC, getcolptr, rowvals, nonzeros
using LinearAlgebra: Symmetric, SingularException
import LinearSolve
using CUDA: CuArray, CuPtr, CUDABackend, stream

const libhsb200 = joinpath(@__DIR__, "..", "hsb200", "libhsb200.so")

const HS_F64, HS_F32 = Int32(0), Int32(1)
const HS_CSC, HS_CSR = Int32(0), Int32(1)

struct HsSparse
    n::Int32
    nnz::Int64
    format::Int32
    dtype::Int32
    ptr::Ptr{Int32}
    idx::Ptr{Int32}
    val::Ptr{Cvoid}
end

abstract type AbstractSweep end
struct ForwardSweep <: AbstractSweep end
struct BackwardSweep <: AbstractSweep end
struct SymmetricSweep <: AbstractSweep end
code(::ForwardSweep) = Int32(0)
code(::BackwardSweep) = Int32(1)
code(::SymmetricSweep) = Int32(2)

abstract type AbstractCacheStrategy end
struct PackedBufferCache <: AbstractCacheStrategy end
struct MatrixViewCache <: AbstractCacheStrategy end
code(::PackedBufferCache) = Int32(0)
code(::MatrixViewCache) = Int32(1)

function check(status::Cint)
    status == 0 && return nothing
    msg = unsafe_string(ccall((:hs_last_error, libhsb200), Cstring, ()))
    if status == 4
        col = ccall((:hs_last_singular_col, libhsb200), Int32, ())
        throw(SingularException(Int(col)))
    end
    error(msg)
end

dtcode(::Type{Float64}) = HS_F64
dtcode(::Type{Float32}) = HS_F32

# 0-based int32 copies of a SparseMatrixCSC, kept alive during the call.
function with_desc(f, A::SparseMatrixCSC{Tv}) where {Tv}
    ptr = Int32.(getcolptr(A) .- 1)
    idx = Int32.(rowvals(A) .- 1)
    val = nonzeros(A)
    GC.@preserve ptr idx val begin
        d = Ref(HsSparse(size(A, 1), length(val), HS_CSC, dtcode(Tv), pointer(ptr), pointer(idx),
                         Ptr{Cvoid}(pointer(val))))
        return f(d)
    end
end

struct GPUConfig
    threads::Int32
    blocks::Int32
    function GPUConfig(threads::Integer, blocks::Integer)
        threads > 0 || error("`threads` must be greater than 0")
        blocks > 0 || error("`blocks` must be greater than 0")
        new(threads, blocks)
    end
end

struct L1GSPrecBuilder
    backend::CUDABackend
    device_config::GPUConfig
end
L1GSPrecBuilder(backend::CUDABackend; threads::Integer, blocks::Integer) =
    L1GSPrecBuilder(backend, GPUConfig(threads, blocks))

mutable struct L1GSPreconditioner{T}
    handle::Ptr{Cvoid}
    n::Int
end

struct HsL1gsOptions
    threads_per_part::Int32   # 0: the library's choice; 1: thread per partition; 4/8/16/32 lanes
    order::Int32              # 0: the library's choice; 1: the reference's summation order; 2: reordered
end

function (b::L1GSPrecBuilder)(A::SparseMatrixCSC{T}, partsize::Integer = b.device_config.blocks;
                              isSymA::Bool = false, η = 1.5, sweep::AbstractSweep = SymmetricSweep(),
                              cache_strategy::AbstractCacheStrategy = PackedBufferCache(),
                              precision::Type = T, threads_per_part::Integer = 0,
                              order::Symbol = :auto) where {T}
    partsize == 0 && error("partsize must be greater than 0")
    h = Ref{Ptr{Cvoid}}(C_NULL)
    opts = HsL1gsOptions(threads_per_part, order === :reference ? 1 : order === :any ? 2 : 0)
    with_desc(A) do d
        check(ccall((:hs_l1gs_create_opts, libhsb200), Cint,
                    (Ref{HsSparse}, Int32, Int32, Cdouble, Int32, Int32, Int32, Int32, Int32, Ref{HsL1gsOptions},
                     Ptr{Cvoid}, Ref{Ptr{Cvoid}}),
                    d, partsize, isSymA, η, code(sweep), code(cache_strategy), dtcode(precision),
                    b.device_config.threads, b.device_config.blocks, opts, stream().handle, h))
    end
    P = L1GSPreconditioner{precision}(h[], size(A, 1))
    finalizer(p -> ccall((:hs_l1gs_destroy, libhsb200), Cint, (Ptr{Cvoid},), p.handle), P)
    return P
end

# Symmetric(A): materialised like get_data (src/l1_gauss_seidel.jl:602-610), isSymA = true.
(b::L1GSPrecBuilder)(A::Symmetric{T, <:SparseMatrixCSC}, partsize::Integer = b.device_config.blocks; kwargs...) where {T} =
    b(SparseMatrixCSC(A), partsize; isSymA = true, kwargs...)

# ldiv! on device vectors: raw pointers, no copies.
function LinearSolve.ldiv!(y::CuArray{T}, P::L1GSPreconditioner, x::CuArray{T}) where {T <: Union{Float64, Float32}}
    check(ccall((:hs_l1gs_apply, libhsb200), Cint, (Ptr{Cvoid}, CuPtr{T}, CuPtr{T}, Int32, Ptr{Cvoid}),
                P.handle, x, y, dtcode(T), stream().handle))
    return nothing
end

# ldiv! on host vectors: the generic path (copy to the device, sweep, copy back).
function LinearSolve.ldiv!(y::Vector{T}, P::L1GSPreconditioner, x::Vector{T}) where {T <: Union{Float64, Float32}}
    GC.@preserve x y check(ccall((:hs_l1gs_apply_host, libhsb200), Cint,
                                 (Ptr{Cvoid}, Ptr{T}, Ptr{T}, Int32, Ptr{Cvoid}),
                                 P.handle, x, y, dtcode(T), stream().handle))
    return nothing
end

Base.:\(P::L1GSPreconditioner, x::AbstractVector) = (y = similar(x); LinearSolve.ldiv!(y, P, x); y)

# ---- Chebyshev -------------------------------------------------------------
struct ChebyshevFourth
    degree::Int
end
ChebyshevFourth(; degree = 4, backend = CUDABackend()) = ChebyshevFourth(degree)
struct ChebyshevFirst
    degree::Int
end
ChebyshevFirst(; degree = 4, backend = CUDABackend()) = ChebyshevFirst(degree)
kind(::ChebyshevFourth) = Int32(4)
kind(::ChebyshevFirst) = Int32(1)

mutable struct ChebyshevSmoother{T}
    handle::Ptr{Cvoid}
end

function _build_smoother(cfg::Union{ChebyshevFourth, ChebyshevFirst}, A::SparseMatrixCSC{Float64};
                         precision::Type = Float64, lanczos::Bool = false)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    with_desc(A) do d
        check(ccall((:hs_cheb_create, libhsb200), Cint,
                    (Ref{HsSparse}, Int32, Int32, Int32, Int32, Ptr{Cvoid}, Ref{Ptr{Cvoid}}),
                    d, kind(cfg), cfg.degree, Int32(lanczos), dtcode(precision), stream().handle, h))
    end
    S = ChebyshevSmoother{precision}(h[])
    finalizer(s -> ccall((:hs_cheb_destroy, libhsb200), Cint, (Ptr{Cvoid},), s.handle), S)
    return S
end

function smooth!(x::CuArray{T}, s::ChebyshevSmoother{T}, b::CuArray{T}) where {T}
    check(ccall((:hs_cheb_smooth, libhsb200), Cint, (Ptr{Cvoid}, CuPtr{T}, CuPtr{T}, Ptr{Cvoid}),
                s.handle, x, b, stream().handle))
    return nothing
end

# ldiv!(z, S, r) := (z .= 0; smooth!(z, S, r)) — the smoother as a PCG preconditioner.
function LinearSolve.ldiv!(z::CuArray{T}, s::ChebyshevSmoother, r::CuArray{T}) where {T}
    check(ccall((:hs_cheb_apply, libhsb200), Cint, (Ptr{Cvoid}, CuPtr{T}, CuPtr{T}, Int32, Ptr{Cvoid}),
                s.handle, r, z, dtcode(T), stream().handle))
    return nothing
end

export L1GSPrecBuilder, ForwardSweep, BackwardSweep, SymmetricSweep, PackedBufferCache, MatrixViewCache,
       ChebyshevFourth, ChebyshevFirst, smooth!

end # module

# The callers of ldiv!: Krylov.jl's cg and gmres as LinearSolve runs them with
# Pl = P, on the device (hs_cg_krylovjl / hs_gmres_krylovjl).  A device matrix
# handle comes from hs_matrix_create; the solvers apply P once per iteration.
struct HsSolveInfo
    iterations::Int32
    converged::Int32
    relres::Cdouble
    ms::Cdouble
    rnorm::Cdouble
end

prec_code(::Nothing) = (Int32(0), C_NULL)
prec_code(P::L1GSPreconditioner) = (Int32(1), P.handle)
prec_code(S::ChebyshevSmoother) = (Int32(2), S.handle)

function krylov_cg!(x::CuArray{Float64}, A::Ptr{Cvoid}, b::CuArray{Float64}, Pl = nothing;
                    atol = sqrt(eps(Float64)), rtol = sqrt(eps(Float64)), itmax::Integer = 0)
    t, h = prec_code(Pl)
    info = Ref{HsSolveInfo}()
    st = ccall((:hs_cg_krylovjl, libhsb200), Cint,
               (Ptr{Cvoid}, Int32, Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Cdouble, Cdouble, Int32, Ptr{Cvoid},
                Ref{HsSolveInfo}), A, t, h, b, x, atol, rtol, itmax, stream().handle, info)
    st == 6 || check(st)   # 6: not converged, reported in info
    return info[]
end

function krylov_gmres!(x::CuArray{Float64}, A::Ptr{Cvoid}, b::CuArray{Float64}, Pl = nothing; memory::Integer = 20,
                       atol = sqrt(eps(Float64)), rtol = sqrt(eps(Float64)), itmax::Integer = 0)
    t, h = prec_code(Pl)
    info = Ref{HsSolveInfo}()
    st = ccall((:hs_gmres_krylovjl, libhsb200), Cint,
               (Ptr{Cvoid}, Int32, Ptr{Cvoid}, Int32, CuPtr{Float64}, CuPtr{Float64}, Cdouble, Cdouble, Int32,
                Ptr{Cvoid}, Ref{HsSolveInfo}), A, t, h, memory, b, x, atol, rtol, itmax, stream().handle, info)
    st == 6 || check(st)
    return info[]
end
