# Julia binding of libcsipm.so (include/csipm.h) for CompressedSensingIPM.jl:
# the MadNLP / NLPModels plugin surface of the package, backed by the B200
# library.
#
#   nlp = CsipmBackend.CsipmNLP(parameters; rdft=true)                 # FFTNLPModel
#   solver = MadNLP.MadNLPSolver(nlp; kkt_system=CsipmBackend.CsipmKKT, # FFTKKTSystem
#                                nlp_scaling=false, dual_initialized=true,
#                                richardson_max_iter=0, tol=1e-8, richardson_tol=Inf,
#                                max_iter=2000)
#   stats = CsipmBackend.ipm_solve!(solver)                           # MadNLP's loop
#   beta, c, st = CsipmBackend.device_ipm_solve!(nlp)                 # or the device IPM
#
# `parameters` is the package's FFTParameters (or anything with the fields
# DFTdim, DFTsize, z0, lambda, index_missing).  Every vector is a CuArray
# passed by pointer (column-major, the reference's beta packing); the C
# structs are mirrored field by field.  Gondzio's formulation has the same
# pair: CsipmGondzioNLP / CsipmGondzioKKT.
#
# Julia is not installed where the library is built, so this file is written
# against the header and MadNLP 0.8's plugin API but has not been run; the
# Python mirror (csipm/) is the tested host side.

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
    z0::CuPtr{Cdouble}                   # device pointer (const double*)
    host_missing::Ptr{Int64}
    n_missing::Int64
end

mutable struct CsipmOptions              # csipm_options (ABI version 2)
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
    ipm_cg_forcing::Cdouble
end
CsipmOptions() = CsipmOptions(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, C_NULL, 0, 0, 0, 0)

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
    graph_iters::Cint
end
CsipmStats() = CsipmStats(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)

# csipm_stats as an immutable (inline) row, for arrays of statistics
struct CsipmStatsRow
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
    graph_iters::Cint
end

function csipm_check(st, h=C_NULL)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:csipm_last_error, libcsipm), Cstring, (Ptr{Cvoid},), h))
    error("libcsipm status $st: $msg")
end

function default_options(; rdft=true, mixed=false, preconditioner=true, tol=1e-8, ipm_cg_rtol=1e-8)
    o = CsipmOptions()
    csipm_check(ccall((:csipm_default_options, libcsipm), Cint, (Ref{CsipmOptions},), o))
    o.rdft = rdft
    o.precision = mixed ? 1 : 0
    o.preconditioner = preconditioner
    o.tol = tol
    o.ipm_cg_rtol = ipm_cg_rtol
    o.stream = CUDA.stream().handle      # the task-local CUDA.jl stream
    return o
end

# ------------------------------------------------------------ the operator
# FFTOperator{VT}(nβ, DFTdim, DFTsize, index_missing, rdft) (src/fft_utils.jl:16-54):
# one library handle owns the plans, the mask, the spectrum, the cached
# A^T z0 and the CG workspace.
mutable struct CsipmHandle
    ptr::Ptr{Cvoid}
    N::Int
    z0::CuVector{Float64}                # kept alive: the Gondzio model reads it after create
end

function CsipmHandle(DFTdim::Integer, DFTsize, z0::CuVector{Float64}, lambda::Real, index_missing;
                     options=default_options())
    N = prod(DFTsize)
    missing = Int64[LinearIndices(Tuple(DFTsize))[i] - 1 for i in index_missing]    # 0-based
    sz = ntuple(d -> d <= DFTdim ? Cint(DFTsize[d]) : Cint(1), 3)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve missing z0 begin
        prob = CsipmProblem(DFTdim, sz, lambda, pointer(z0), pointer(missing), length(missing))
        csipm_check(ccall((:csipm_create, libcsipm), Cint,
                          (Ref{CsipmProblem}, Ref{CsipmOptions}, Ref{Ptr{Cvoid}}), prob, options, h))
    end
    obj = CsipmHandle(h[], N, z0)
    finalizer(x -> ccall((:csipm_destroy, libcsipm), Cint, (Ptr{Cvoid},), x.ptr), obj)
    return obj
end

function CsipmHandle(parameters; rdft=true, preconditioner=true, mixed=false, tol=1e-8, ipm_cg_rtol=1e-8)
    z0 = CuVector{Float64}(vec(parameters.z0))
    opt = default_options(; rdft, mixed, preconditioner, tol, ipm_cg_rtol)
    return CsipmHandle(parameters.DFTdim, parameters.DFTsize, z0, parameters.lambda,
                       parameters.index_missing; options=opt)
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

# ----------------------------------------------------------- the NLP model
# FFTNLPModel{VT}(parameters; krylov_solver, rdft, preconditioner)
# (src/fft_model.jl:1-64): variables [beta; c] (2nβ, free), constraints
# [-beta - c; beta - c] <= 0 (2nβ), no Jacobian / Hessian storage (the KKT
# plugin never asks for them).
mutable struct CsipmNLP{P} <: NLPModels.AbstractNLPModel{Float64,CuVector{Float64}}
    meta::NLPModels.NLPModelMeta{Float64,CuVector{Float64}}
    counters::NLPModels.Counters
    parameters::P
    nβ::Int
    h::CsipmHandle
    krylov_solver::Symbol
    preconditioner::Bool
end

function fft_meta(nβ, DFTdim)
    VT = CuVector{Float64}
    nvar = ncon = 2nβ
    return NLPModels.NLPModelMeta(
        nvar;
        x0=CUDA.zeros(Float64, nvar), lvar=fill!(VT(undef, nvar), -Inf), uvar=fill!(VT(undef, nvar), Inf),
        ncon=ncon, y0=CUDA.zeros(Float64, ncon), lcon=fill!(VT(undef, ncon), -Inf), ucon=CUDA.zeros(Float64, ncon),
        nnzj=0, nnzh=0, minimize=true, islp=false,
        variable_bounds_analysis=false, constraint_bounds_analysis=false,
        grad_available=true, jac_available=false, hess_available=false,
        jprod_available=false, jtprod_available=false, hprod_available=false,
        name="CompressedSensing-$(DFTdim)D")
end

function CsipmNLP(parameters; krylov_solver::Symbol=:cg, rdft::Bool=false, preconditioner::Bool=true,
                  mixed::Bool=false, tol=1e-8, ipm_cg_rtol=1e-8)
    nβ = prod(parameters.DFTsize)
    h = CsipmHandle(parameters; rdft, preconditioner, mixed, tol, ipm_cg_rtol)   # also computes A^T z0
    return CsipmNLP(fft_meta(nβ, parameters.DFTdim), NLPModels.Counters(), parameters, nβ, h,
                    krylov_solver, preconditioner)
end

# M_perpt_z0 (src/fft_model.jl:61-62), copied out of the handle
function M_perpt_z0(nlp::CsipmNLP)
    out = CuVector{Float64}(undef, nlp.nβ)
    csipm_check(ccall((:csipm_get_Atz0, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}), nlp.h.ptr, out), nlp.h.ptr)
    return out
end

# obj / grad! / cons! (src/fft_model.jl:66-101)
function NLPModels.obj(nlp::CsipmNLP, x::AbstractVector)
    NLPModels.increment!(nlp, :neval_obj)
    f = Ref{Cdouble}()
    csipm_check(ccall((:csipm_obj, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Ref{Cdouble}), nlp.h.ptr, x, f),
                nlp.h.ptr)
    return f[]
end
function NLPModels.grad!(nlp::CsipmNLP, x::AbstractVector, g::AbstractVector)
    NLPModels.increment!(nlp, :neval_grad)
    csipm_check(ccall((:csipm_grad, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}), nlp.h.ptr, x, g),
                nlp.h.ptr)
    return g
end
function NLPModels.cons!(nlp::CsipmNLP, x::AbstractVector, c::AbstractVector)
    NLPModels.increment!(nlp, :neval_cons)
    csipm_check(ccall((:csipm_cons, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}), nlp.h.ptr, x, c),
                nlp.h.ptr)
    return c
end
# the Lagrangian's Hessian action (obj_weight * [A^T A v_beta; 0]); the
# reference declares hprod unavailable and keeps this product inside its KKT
# plugin, so MadNLP never calls it with CsipmKKT
function NLPModels.hprod!(nlp::CsipmNLP, x::AbstractVector, y::AbstractVector, v::AbstractVector,
                          hv::AbstractVector; obj_weight=1.0)
    NLPModels.increment!(nlp, :neval_hprod)
    csipm_check(ccall((:csipm_hprod, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble),
                      nlp.h.ptr, v, hv, obj_weight), nlp.h.ptr)
    return hv
end

# ------------------------------------------------ condensed operator and P
# CondensedFFTKKTSystem (src/fft_kkt.jl:9-44) and FFTPreconditioner
# (src/fft_kkt.jl:54-85): the library holds Λ1, Λ2, P11, P12, P22 (written by
# build_kkt!); these wrappers give them the reference's mul! methods.
struct CsipmCondensed
    h::CsipmHandle
    nβ::Int
end
struct CsipmPreconditioner
    h::CsipmHandle
    nβ::Int
end
Base.size(K::CsipmCondensed) = (2K.nβ, 2K.nβ)
Base.size(P::CsipmPreconditioner) = (2P.nβ, 2P.nβ)
Base.eltype(::CsipmCondensed) = Float64
Base.eltype(::CsipmPreconditioner) = Float64

function LinearAlgebra.mul!(y::CuVector{Float64}, K::CsipmCondensed, x::CuVector{Float64}, alpha::Number, beta::Number)
    csipm_check(ccall((:csipm_condensed_mul, libcsipm), Cint,
                      (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble, Cdouble), K.h.ptr, y, x, alpha, beta),
                K.h.ptr)
    return y
end
function LinearAlgebra.mul!(y::CuVector{Float64}, P::CsipmPreconditioner, x::CuVector{Float64}, alpha::Number,
                            beta::Number)
    csipm_check(ccall((:csipm_precond_mul, libcsipm), Cint,
                      (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble, Cdouble), P.h.ptr, y, x, alpha, beta),
                P.h.ptr)
    return y
end
LinearAlgebra.mul!(y::CuVector{Float64}, K::Union{CsipmCondensed,CsipmPreconditioner}, x::CuVector{Float64}) =
    mul!(y, K, x, 1.0, 0.0)

# -------------------------------------------------- the linear "solver"
# MadNLP asks its KKT system's linear solver for inertia, a name and
# refinement; the condensed system is solved by the library's PCG (Krylov
# cg semantics: atol 1e-12, rtol 0), which needs no factorisation and has no
# inertia to report (src/fft_kkt.jl:163-167 say the same of Krylov's workspace).
struct CsipmPCG end
MadNLP.is_inertia(::CsipmPCG) = true
MadNLP.inertia(::CsipmPCG) = (0, 0, 0)
MadNLP.introduce(::CsipmPCG) = "libcsipm PCG (B200)"
MadNLP.improve!(::CsipmPCG) = true
MadNLP.factorize!(::CsipmPCG) = nothing

# --------------------------------------------------------- the KKT plugin
# FFTKKTSystem (src/fft_kkt.jl:91-111): MadNLP's diagonals stay on the Julia
# side (they are MadNLP's to fill); the operator, the preconditioner and the
# CG workspace are the handle's.
struct CsipmKKT{T,VI,VT,NLP} <: MadNLP.AbstractReducedKKTSystem{T,VT,CsipmCondensed,MadNLP.ExactHessian{T,VT}}
    nlp::NLP
    K::CsipmCondensed
    P::CsipmPreconditioner
    reg::VT
    pr_diag::VT
    du_diag::VT
    l_diag::VT
    u_diag::VT
    l_lower::VT
    u_lower::VT
    ind_lb::VI
    ind_ub::VI
    linear_solver::CsipmPCG
    krylov_iterations::Vector{Int}
    krylov_timer::Vector{Float64}
end

# create_kkt_system (src/fft_kkt.jl:113-156)
function MadNLP.create_kkt_system(
    ::Type{CsipmKKT},
    cb::MadNLP.AbstractCallback{T,VT},
    linear_solver::Type;
    opt_linear_solver=nothing,
    hessian_approximation=MadNLP.ExactHessian,
    qn_options=MadNLP.QuasiNewtonOptions(),
) where {T,VT}
    nlp = cb.nlp
    nβ = nlp.nβ
    nlb, nub = length(cb.ind_lb), length(cb.ind_ub)
    n = NLPModels.get_nvar(nlp) + length(cb.ind_ineq)     # variables and slacks
    m = NLPModels.get_ncon(nlp)
    VI = typeof(cb.ind_lb)
    return CsipmKKT{T,VI,VT,typeof(nlp)}(
        nlp, CsipmCondensed(nlp.h, nβ), CsipmPreconditioner(nlp.h, nβ),
        VT(undef, n), VT(undef, n), VT(undef, m),
        VT(undef, nlb), VT(undef, nub), VT(undef, nlb), VT(undef, nub),
        cb.ind_lb, cb.ind_ub, CsipmPCG(), Int[], Float64[])
end

# the stubs of src/fft_kkt.jl:158-211 and :277-283: no Jacobian or Hessian is
# ever formed, inertia is always accepted, nothing to compress or factorise
MadNLP.num_variables(kkt::CsipmKKT) = 2 * kkt.nlp.nβ
MadNLP.get_hessian(kkt::CsipmKKT) = nothing
MadNLP.get_jacobian(kkt::CsipmKKT) = nothing
MadNLP.is_inertia_correct(kkt::CsipmKKT, p, n, z) = true
Base.eltype(kkt::CsipmKKT{T}) where {T} = T
function Base.size(kkt::CsipmKKT)
    n = NLPModels.get_nvar(kkt.nlp)
    m = NLPModels.get_ncon(kkt.nlp)
    N = n + 2m + length(kkt.l_diag) + length(kkt.u_diag)
    return (N, N)
end
function MadNLP.initialize!(kkt::CsipmKKT{T}) where {T}
    fill!(kkt.reg, one(T))
    fill!(kkt.pr_diag, one(T))
    fill!(kkt.du_diag, zero(T))
    fill!(kkt.l_lower, zero(T))
    fill!(kkt.u_lower, zero(T))
    fill!(kkt.l_diag, one(T))
    fill!(kkt.u_diag, one(T))
    return
end
MadNLP.eval_jac_wrapper!(solver::MadNLP.MadNLPSolver, kkt::CsipmKKT, x::MadNLP.PrimalVector) = nothing
MadNLP.eval_lag_hess_wrapper!(solver::MadNLP.MadNLPSolver, kkt::CsipmKKT, x::MadNLP.PrimalVector,
                              l::AbstractVector; is_resto=false) = nothing
MadNLP.compress_jacobian!(kkt::CsipmKKT) = nothing
MadNLP.compress_hessian!(kkt::CsipmKKT) = nothing

# mul! (src/fft_kkt.jl:213-251): the 6nβ block product on the device, then
# MadNLP's own diagonal terms
function MadNLP.mul!(y::VT, kkt::CsipmKKT, x::VT, alpha::Number, beta::Number) where {VT<:MadNLP.AbstractKKTVector}
    csipm_check(ccall((:csipm_kkt_mul, libcsipm), Cint,
                      (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble, Cdouble),
                      kkt.nlp.h.ptr, MadNLP.full(y), MadNLP.full(x), alpha, beta), kkt.nlp.h.ptr)
    MadNLP._kktmul!(y, x, kkt.reg, kkt.du_diag, kkt.l_lower, kkt.u_lower, kkt.l_diag, kkt.u_diag, alpha, beta)
    return y
end

# jtprod! (src/fft_kkt.jl:253-275)
function MadNLP.jtprod!(y::AbstractVector, kkt::CsipmKKT, x::AbstractVector)
    csipm_check(ccall((:csipm_jtprod, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}),
                      kkt.nlp.h.ptr, y, x), kkt.nlp.h.ptr)
    return y
end

# build_kkt! (src/fft_kkt.jl:285-307): Λ1, Λ2 and the preconditioner from
# the slack block of pr_diag
function MadNLP.build_kkt!(kkt::CsipmKKT)
    csipm_check(ccall((:csipm_kkt_build, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}), kkt.nlp.h.ptr,
                      kkt.pr_diag), kkt.nlp.h.ptr)
    return
end

# solve_kkt! (src/fft_kkt.jl:309-354): MadNLP's reduction of the bound rows,
# then right-hand side, PCG and back-substitution on the device, then
# MadNLP's completion of the bound rows
function MadNLP.solve_kkt!(kkt::CsipmKKT, w::MadNLP.AbstractKKTVector)
    MadNLP.reduce_rhs!(w.xp_lr, MadNLP.dual_lb(w), kkt.l_diag, w.xp_ur, MadNLP.dual_ub(w), kkt.u_diag)
    it = Ref{Cint}(0)
    t = @elapsed csipm_check(ccall((:csipm_kkt_solve, libcsipm), Cint,
                                   (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Ref{Cint}),
                                   kkt.nlp.h.ptr, MadNLP.full(w), kkt.pr_diag, it), kkt.nlp.h.ptr)
    push!(kkt.krylov_iterations, it[])
    push!(kkt.krylov_timer, t)
    MadNLP.finish_aug_solve!(kkt, w)
    return true
end

# factorize_wrapper! (src/fft_kkt.jl:356-362): assembling is all there is
function MadNLP.factorize_wrapper!(solver::MadNLP.MadNLPSolver{T,VT,IT,KKT}) where {T,VT,IT,KKT<:CsipmKKT}
    MadNLP.build_kkt!(solver.kkt)
    return true
end

# ---------------------------------------------------------------- ipm_solve!
# ipm_solve!(solver) (src/CompressedSensingIPM.jl:31-36): MadNLP's loop over
# the plugin above
function ipm_solve!(solver::MadNLP.MadNLPSolver)
    MadNLP.print_init(solver)
    MadNLP.initialize!(solver)
    MadNLP.regular!(solver)
    return MadNLP.MadNLPExecutionStats(solver)
end

# The whole interior-point solve on the device instead of MadNLP's loop
# (csipm_solve): beta, c and the statistics.
function device_ipm_solve!(nlp::CsipmNLP)
    beta = CUDA.zeros(Float64, nlp.nβ)
    c = CUDA.zeros(Float64, nlp.nβ)
    stats = Ref(CsipmStats())
    st = ccall((:csipm_solve, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Ref{CsipmStats}),
               nlp.h.ptr, beta, c, stats)
    st in (0, -8) || csipm_check(st, nlp.h.ptr)   # -8: max_iter reached (the iterate is still returned)
    return beta, c, stats[]
end

# Several recoveries solved together on the device (csipm_solve_batch): one
# kernel launch per step for all of them, FP64.  The models share the
# dimension count, the long-row 1D passes and the presence of missing
# samples; sizes, lambda and options are their own.  Returns each beta and
# its statistics (status per instance: 0 converged, -8 max_iter, ...).
function device_ipm_solve_batch!(nlps::AbstractVector{<:CsipmNLP})
    n = length(nlps)
    betas = [CUDA.zeros(Float64, nlp.nβ) for nlp in nlps]
    handles = Ptr{Cvoid}[nlp.h.ptr for nlp in nlps]
    outs = Ptr{Cdouble}[Ptr{Cdouble}(reinterpret(UInt, pointer(b))) for b in betas]
    stats = Vector{CsipmStatsRow}(undef, n)
    st = GC.@preserve betas ccall((:csipm_solve_batch, libcsipm), Cint,
                                  (Ptr{Ptr{Cvoid}}, Cint, Ptr{Ptr{Cdouble}}, Ptr{CsipmStatsRow}),
                                  handles, n, outs, stats)
    st in (0, -6, -7, -8) || csipm_check(st, C_NULL)   # per-instance failures are in stats[k].status
    return betas, stats
end

# ============================================================ Gondzio pair
# GondzioNLPModel (src/gondzio_model.jl:1-65): x = [p; q; r], p, q >= 0,
# z0 - A(p - q) - r = 0.  The handle keeps z0 (FFTParameters.z0 outlives it).
mutable struct CsipmGondzioNLP{P} <: NLPModels.AbstractNLPModel{Float64,CuVector{Float64}}
    meta::NLPModels.NLPModelMeta{Float64,CuVector{Float64}}
    counters::NLPModels.Counters
    parameters::P
    nβ::Int
    h::CsipmHandle
    krylov_solver::Symbol
    preconditioner::Bool
end

function CsipmGondzioNLP(parameters; krylov_solver::Symbol=:cg, rdft::Bool=false, preconditioner::Bool=true)
    VT = CuVector{Float64}
    nβ = prod(parameters.DFTsize)
    m = nβ
    nvar = 2nβ + m
    lvar = fill!(VT(undef, nvar), -Inf)
    fill!(view(lvar, 1:2nβ), 0.0)
    meta = NLPModels.NLPModelMeta(
        nvar; x0=CUDA.zeros(Float64, nvar), lvar=lvar, uvar=fill!(VT(undef, nvar), Inf),
        ncon=m, y0=CUDA.zeros(Float64, m), lcon=CUDA.zeros(Float64, m), ucon=CUDA.zeros(Float64, m),
        nnzj=0, nnzh=0, minimize=true, islp=false,
        grad_available=true, jac_available=false, hess_available=false,
        jprod_available=false, jtprod_available=false, hprod_available=false,
        name="CompressedSensing-Gondzio-$(parameters.DFTdim)D")
    h = CsipmHandle(parameters; rdft, preconditioner)
    return CsipmGondzioNLP(meta, NLPModels.Counters(), parameters, nβ, h, krylov_solver, preconditioner)
end

for (f, c) in ((:grad!, :csipm_gondzio_grad), (:cons!, :csipm_gondzio_cons))
    @eval function NLPModels.$f(nlp::CsipmGondzioNLP, x::AbstractVector, out::AbstractVector)
        NLPModels.increment!(nlp, $(QuoteNode(f == :grad! ? :neval_grad : :neval_cons)))
        csipm_check(ccall(($(QuoteNode(c)), libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}),
                          nlp.h.ptr, x, out), nlp.h.ptr)
        return out
    end
end
function NLPModels.obj(nlp::CsipmGondzioNLP, x::AbstractVector)
    NLPModels.increment!(nlp, :neval_obj)
    f = Ref{Cdouble}()
    csipm_check(ccall((:csipm_gondzio_obj, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Ref{Cdouble}),
                      nlp.h.ptr, x, f), nlp.h.ptr)
    return f[]
end

# GondzioKKTSystem (src/gondzio_kkt.jl:98-362): the same plugin shape over a
# 4nβ KKT vector [p; q; r; y]
struct CsipmGondzioKKT{T,VI,VT,NLP} <: MadNLP.AbstractReducedKKTSystem{T,VT,CsipmCondensed,MadNLP.ExactHessian{T,VT}}
    nlp::NLP
    K::CsipmCondensed
    reg::VT
    pr_diag::VT
    du_diag::VT
    l_diag::VT
    u_diag::VT
    l_lower::VT
    u_lower::VT
    ind_lb::VI
    ind_ub::VI
    linear_solver::CsipmPCG
    krylov_iterations::Vector{Int}
    krylov_timer::Vector{Float64}
end

function MadNLP.create_kkt_system(::Type{CsipmGondzioKKT}, cb::MadNLP.AbstractCallback{T,VT}, linear_solver::Type;
                                  opt_linear_solver=nothing, hessian_approximation=MadNLP.ExactHessian,
                                  qn_options=MadNLP.QuasiNewtonOptions()) where {T,VT}
    nlp = cb.nlp
    nlb, nub = length(cb.ind_lb), length(cb.ind_ub)
    n = NLPModels.get_nvar(nlp) + length(cb.ind_ineq)
    m = NLPModels.get_ncon(nlp)
    VI = typeof(cb.ind_lb)
    return CsipmGondzioKKT{T,VI,VT,typeof(nlp)}(
        nlp, CsipmCondensed(nlp.h, nlp.nβ), VT(undef, n), VT(undef, n), VT(undef, m),
        VT(undef, nlb), VT(undef, nub), VT(undef, nlb), VT(undef, nub),
        cb.ind_lb, cb.ind_ub, CsipmPCG(), Int[], Float64[])
end

MadNLP.num_variables(kkt::CsipmGondzioKKT) = 2 * kkt.nlp.nβ
MadNLP.get_hessian(kkt::CsipmGondzioKKT) = nothing
MadNLP.get_jacobian(kkt::CsipmGondzioKKT) = nothing
MadNLP.is_inertia_correct(kkt::CsipmGondzioKKT, p, n, z) = true
Base.eltype(kkt::CsipmGondzioKKT{T}) where {T} = T
function Base.size(kkt::CsipmGondzioKKT)
    N = NLPModels.get_nvar(kkt.nlp) + NLPModels.get_ncon(kkt.nlp) + length(kkt.l_diag) + length(kkt.u_diag)
    return (N, N)
end
function MadNLP.initialize!(kkt::CsipmGondzioKKT{T}) where {T}
    fill!(kkt.reg, one(T)); fill!(kkt.pr_diag, one(T)); fill!(kkt.du_diag, zero(T))
    fill!(kkt.l_lower, zero(T)); fill!(kkt.u_lower, zero(T))
    fill!(kkt.l_diag, one(T)); fill!(kkt.u_diag, one(T))
    return
end
MadNLP.eval_jac_wrapper!(solver::MadNLP.MadNLPSolver, kkt::CsipmGondzioKKT, x::MadNLP.PrimalVector) = nothing
MadNLP.eval_lag_hess_wrapper!(solver::MadNLP.MadNLPSolver, kkt::CsipmGondzioKKT, x::MadNLP.PrimalVector,
                              l::AbstractVector; is_resto=false) = nothing
MadNLP.compress_jacobian!(kkt::CsipmGondzioKKT) = nothing
MadNLP.compress_hessian!(kkt::CsipmGondzioKKT) = nothing

function MadNLP.mul!(y::VT, kkt::CsipmGondzioKKT, x::VT, alpha::Number, beta::Number) where {VT<:MadNLP.AbstractKKTVector}
    csipm_check(ccall((:csipm_gondzio_kkt_mul, libcsipm), Cint,
                      (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble, Cdouble),
                      kkt.nlp.h.ptr, MadNLP.full(y), MadNLP.full(x), alpha, beta), kkt.nlp.h.ptr)
    MadNLP._kktmul!(y, x, kkt.reg, kkt.du_diag, kkt.l_lower, kkt.u_lower, kkt.l_diag, kkt.u_diag, alpha, beta)
    return y
end
function MadNLP.jtprod!(y::AbstractVector, kkt::CsipmGondzioKKT, x::AbstractVector)
    csipm_check(ccall((:csipm_gondzio_jtprod, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}),
                      kkt.nlp.h.ptr, y, x), kkt.nlp.h.ptr)
    return y
end
function MadNLP.build_kkt!(kkt::CsipmGondzioKKT)
    csipm_check(ccall((:csipm_gondzio_kkt_build, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}), kkt.nlp.h.ptr,
                      kkt.pr_diag), kkt.nlp.h.ptr)
    return
end
function MadNLP.solve_kkt!(kkt::CsipmGondzioKKT, w::MadNLP.AbstractKKTVector)
    MadNLP.reduce_rhs!(w.xp_lr, MadNLP.dual_lb(w), kkt.l_diag, w.xp_ur, MadNLP.dual_ub(w), kkt.u_diag)
    it = Ref{Cint}(0)
    t = @elapsed csipm_check(ccall((:csipm_gondzio_kkt_solve, libcsipm), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Ref{Cint}),
                                   kkt.nlp.h.ptr, MadNLP.full(w), it), kkt.nlp.h.ptr)
    push!(kkt.krylov_iterations, it[])
    push!(kkt.krylov_timer, t)
    MadNLP.finish_aug_solve!(kkt, w)
    return true
end
function MadNLP.factorize_wrapper!(solver::MadNLP.MadNLPSolver{T,VT,IT,KKT}) where {T,VT,IT,KKT<:CsipmGondzioKKT}
    MadNLP.build_kkt!(solver.kkt)
    return true
end

# CompressedSensingADMM(parameters, operator; rho, maxt, tol) (src/admm.jl:8-61)
mutable struct CsipmAdmmStats            # csipm_admm_stats
    status::Cint
    iterations::Cint
    cg_iter::Cint
    err::Cdouble
    solve_ms::Cdouble
end
CsipmAdmmStats() = CsipmAdmmStats(0, 0, 0, 0, 0)

function CompressedSensingADMM(nlp::CsipmNLP; rho=1.0, maxt=1000, tol=1e-6)
    z = CUDA.zeros(Float64, nlp.nβ)
    stats = Ref(CsipmAdmmStats())
    st = ccall((:csipm_admm, libcsipm), Cint, (Ptr{Cvoid}, Cdouble, Cint, Cdouble, CuPtr{Cdouble}, Ref{CsipmAdmmStats}),
               nlp.h.ptr, rho, maxt, tol, z, stats)
    st in (0, -8) || csipm_check(st, nlp.h.ptr)   # -8: maxt reached before tol
    return z, stats[]
end

end # module
