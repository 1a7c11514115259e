# Julia binding of libcsipm.so (include/csipm.h) for CompressedSensingIPM.jl.
#
# `include` this file from the package (or a script that has loaded it) to
# run the hot path on the B200 library instead of the package's CUDA backend:
# the structs mirror the C ABI field by field, the wrappers keep the
# reference's names and argument order, and every vector is a CuArray passed
# by pointer (column-major, the reference's beta packing).  Julia is not
# installed where this library is built, so this file is not exercised by the
# library's tests; the Python mirror (csipm/) is the tested host side.

module CsipmBackend

using CUDA
using LinearAlgebra
import NLPModels
import MadNLP

const libcsipm = get(ENV, "CSIPM_LIB", joinpath(@__DIR__, "..", "csipm", "libcsipm.so"))

# ----------------------------------------------------------------- C structs
struct CsipmProblem                      # csipm_problem
    dim::Cint
    size::NTuple{3,Cint}
    lambda::Cdouble
    z0::CuPtr{Cdouble}
    host_missing::Ptr{Int64}
    n_missing::Int64
end

mutable struct CsipmOptions              # csipm_options
    rdft::Cint
    precision::Cint                      # 0 FP64, 1 mixed
    preconditioner::Cint
    tol::Cdouble
    max_iter::Cint
    cg_atol::Cdouble
    cg_rtol::Cdouble
    cg_maxit::Cint
    ipm_cg_rtol::Cdouble
    ir_max::Cint
    verbose::Cint
    stream::Ptr{Cvoid}
    layout::Cint
    cuda_graphs::Cint
    autotune::Cint
end

mutable struct CsipmStats                # csipm_stats
    status::Cint
    ipm_iter::Cint
    cg_iter::Cint
    matvecs::Cint
    refinements::Cint
    gap::Cdouble
    obj::Cdouble
    lasso_obj::Cdouble
    mu::Cdouble
    dual_inf::Cdouble
    solve_ms::Cdouble
    launches::Clonglong
    fallbacks::Cint
    resid_pass_ms::Cdouble
    resid_pass_bytes::Cdouble
    resid_pass_launches::Cint
end
CsipmStats() = CsipmStats(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)

function csipm_check(st, h=C_NULL)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:csipm_last_error, libcsipm), Cstring, (Ptr{Cvoid},), h))
    error("libcsipm status $st: $msg")
end

function default_options(; rdft=true, mixed=false, tol=1e-8, ipm_cg_rtol=1e-8)
    o = CsipmOptions(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, C_NULL, 0, 0, 0)
    csipm_check(ccall((:csipm_default_options, libcsipm), Cint, (Ref{CsipmOptions},), o))
    o.rdft = rdft
    o.precision = mixed ? 1 : 0
    o.tol = tol
    o.ipm_cg_rtol = ipm_cg_rtol
    o.stream = CUDA.stream().handle      # the task-local CUDA.jl stream
    return o
end

# ------------------------------------------------- FFTOperator / FFTNLPModel
# FFTOperator{VT}(...) + FFTNLPModel constructor (src/fft_utils.jl:16-54,
# src/fft_model.jl:12-64): one library handle owns plans, mask, spectrum and
# the cached A^T z0.
mutable struct CsipmHandle
    ptr::Ptr{Cvoid}
    N::Int
    z0::CuVector{Float64}                # kept alive: the handle reads it at create
end

function CsipmHandle(DFTdim::Int, DFTsize, z0::CuVector{Float64}, lambda::Real, index_missing;
                     options=default_options())
    N = prod(DFTsize)
    missing = Int64[LinearIndices(Tuple(DFTsize))[i] - 1 for i in index_missing]    # 0-based
    sz = ntuple(d -> d <= DFTdim ? Cint(DFTsize[d]) : Cint(1), 3)
    prob = CsipmProblem(DFTdim, sz, lambda, pointer(z0), pointer(missing), length(missing))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve missing z0 begin
        csipm_check(ccall((:csipm_create, libcsipm), Cint,
                          (Ref{CsipmProblem}, Ref{CsipmOptions}, Ref{Ptr{Cvoid}}), prob, options, h))
    end
    obj = CsipmHandle(h[], N, z0)
    finalizer(x -> ccall((:csipm_destroy, libcsipm), Cint, (Ptr{Cvoid},), x.ptr), obj)
    return obj
end

# M_perp_beta / M_perpt_z / M_perpt_M_perp_vec (src/fft_utils.jl:67-123)
for (jl, c) in ((:M_perp_beta!, :csipm_apply_A), (:M_perpt_z!, :csipm_apply_At),
                (:M_perpt_M_perp_vec!, :csipm_apply_AtA))
    @eval function $jl(y::CuVector{Float64}, h::CsipmHandle, x::CuVector{Float64})
        csipm_check(ccall(($(QuoteNode(c)), libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}),
                          h.ptr, x, y), h.ptr)
        return y
    end
end

# beta_to_DFT! / DFT_to_beta! (src/fft_utils.jl:144-222)
function beta_to_DFT!(v::CuArray{ComplexF64}, DFTdim, DFTsize, beta::CuVector{Float64}; rdft=true)
    sz = Cint[DFTsize[d] for d in 1:DFTdim]
    csipm_check(ccall((:csipm_beta_to_dft, libcsipm), Cint,
                      (Cint, Ptr{Cint}, Cint, CuPtr{Cdouble}, CuPtr{ComplexF64}, Ptr{Cvoid}),
                      DFTdim, sz, rdft, beta, v, CUDA.stream().handle))
    return v
end

function DFT_to_beta!(beta::CuVector{Float64}, DFTdim, DFTsize, v::CuArray{ComplexF64})
    sz = Cint[DFTsize[d] for d in 1:DFTdim]
    csipm_check(ccall((:csipm_dft_to_beta, libcsipm), Cint,
                      (Cint, Ptr{Cint}, Cint, CuPtr{ComplexF64}, CuPtr{Cdouble}, Ptr{Cvoid}),
                      DFTdim, sz, size(v, 1), v, beta, CUDA.stream().handle))
    return beta
end

# ------------------------------------------------------------ NLPModels API
# obj / grad! / cons! (src/fft_model.jl:66-101) on x = [beta; c]
struct CsipmNLP{M} <: NLPModels.AbstractNLPModel{Float64,CuVector{Float64}}
    meta::M
    counters::NLPModels.Counters
    h::CsipmHandle
end

function NLPModels.obj(nlp::CsipmNLP, x::CuVector{Float64})
    f = Ref{Cdouble}()
    csipm_check(ccall((:csipm_obj, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Ref{Cdouble}), nlp.h.ptr, x, f),
                nlp.h.ptr)
    return f[]
end
function NLPModels.grad!(nlp::CsipmNLP, x::CuVector{Float64}, g::CuVector{Float64})
    csipm_check(ccall((:csipm_grad, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}), nlp.h.ptr, x, g),
                nlp.h.ptr)
    return g
end
function NLPModels.cons!(nlp::CsipmNLP, x::CuVector{Float64}, c::CuVector{Float64})
    csipm_check(ccall((:csipm_cons, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}), nlp.h.ptr, x, c),
                nlp.h.ptr)
    return c
end

# ------------------------------------------------------- MadNLP KKT plugin
# build_kkt! / mul! / jtprod! / solve_kkt! (src/fft_kkt.jl:213-354); the
# struct holds what the reference's FFTKKTSystem holds on the Julia side
# (pr_diag, l/u diagonals); the library holds the operator and CG workspace.
mutable struct CsipmKKT
    h::CsipmHandle
    pr_diag::CuVector{Float64}
    l_diag::CuVector{Float64}
    u_diag::CuVector{Float64}
    krylov_iterations::Vector{Int}
end

build_kkt!(kkt::CsipmKKT) =
    csipm_check(ccall((:csipm_kkt_build, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}), kkt.h.ptr, kkt.pr_diag),
                kkt.h.ptr)

function kkt_mul!(y::CuVector{Float64}, kkt::CsipmKKT, x::CuVector{Float64}, alpha, beta)
    csipm_check(ccall((:csipm_kkt_mul, libcsipm), Cint,
                      (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble, Cdouble), kkt.h.ptr, y, x, alpha, beta),
                kkt.h.ptr)
    return y
end

function jtprod!(y::CuVector{Float64}, kkt::CsipmKKT, x::CuVector{Float64})
    csipm_check(ccall((:csipm_jtprod, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}),
                      kkt.h.ptr, y, x), kkt.h.ptr)
    return y
end

# the full KKT vector w (MadNLP.full(w)) after MadNLP.reduce_rhs!
function solve_kkt!(kkt::CsipmKKT, w_full::CuVector{Float64})
    it = Ref{Cint}(0)
    csipm_check(ccall((:csipm_kkt_solve, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Ref{Cint}),
                      kkt.h.ptr, w_full, kkt.pr_diag, it), kkt.h.ptr)
    push!(kkt.krylov_iterations, it[])
    return w_full
end

# ---------------------------------------------------------------- ipm_solve!
# The device interior-point solve in place of MadNLP's loop
# (src/CompressedSensingIPM.jl:31-36): returns beta, c and the statistics.
function ipm_solve!(h::CsipmHandle)
    beta = CUDA.zeros(Float64, h.N)
    c = CUDA.zeros(Float64, h.N)
    stats = Ref(CsipmStats())
    st = ccall((:csipm_solve, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Ref{CsipmStats}),
               h.ptr, beta, c, stats)
    st in (0, -8) || csipm_check(st, h.ptr)   # -8: max_iter reached (result still returned)
    return beta, c, stats[]
end

end # module
