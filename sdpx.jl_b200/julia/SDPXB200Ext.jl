# SDPX package extension binding libsdpx_b200.so (sm_100a) through ccall.
#
# This file is the reference-side glue a maintainer adds as ext/SDPXB200Ext.jl
# (with `[weakdeps] CUDA, ChainRulesCore` / `[extensions] SDPXB200Ext =
# ["CUDA", "ChainRulesCore"]` in Project.toml) together with the small core
# patch shown in INTEGRATION.md (the `:b200` provider symbol, the plan branch,
# the instantiate / route / whole-loop hooks this file overloads).
# It is written against SDPX's seams but is not executed in this repository's
# tests: the build environment has no Julia.  Every ccall below matches a
# declaration in include/sdpx_b200.h or include/sdpx_b200_normal.h.
module SDPXB200Ext

using SDPX
using LinearAlgebra
import ChainRulesCore

const libsdpx = get(ENV, "SDPX_B200_LIB", joinpath(@__DIR__, "..", "libsdpx_b200.so"))

# ---------------------------------------------------------------- handle ---
struct B200Problem
    m::Int64
    nblocks::Int32
    block_order::Ptr{Int32}
    Av::Ptr{Ptr{Float64}}
    C::Ptr{Ptr{Float64}}
    c::Ptr{Float64}
end

mutable struct B200Handle
    ptr::Ptr{Cvoid}
end

function _check(h::B200Handle, status::Cint, what)
    status == 0 && return 0
    status > 0 && return Int(status)
    msg = unsafe_string(ccall((:sdpx_b200_last_error, libsdpx), Cstring, (Ptr{Cvoid},), h.ptr))
    error("libsdpx_b200 $what failed ($status): $msg")
end

"""Upload a dense SDPProblem (DenseCons; equality rows B, b when n > 0) to the
B200 (src/workspace.jl:779)."""
function B200Handle(prob::SDPX.SDPProblem{Float64}; device::Integer=0)
    cons = prob.cons::SDPX.DenseCons{Float64}
    orders = Int32[prob.dims.k[l] for l in 1:prob.dims.L]
    Avs = [Matrix{Float64}(cons.Av[l]) for l in 1:prob.dims.L]   # k² × m, column i = vec(A_i)
    Cs = [Matrix{Float64}(prob.C[l]) for l in 1:prob.dims.L]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve orders Avs Cs prob begin
        p = B200Problem(prob.dims.m, Int32(prob.dims.L), pointer(orders),
                        pointer([pointer(a) for a in Avs]), pointer([pointer(c) for c in Cs]),
                        pointer(prob.c))
        status = ccall((:sdpx_b200_create, libsdpx), Cint,
                       (Ref{B200Problem}, Cint, Ref{Ptr{Cvoid}}), p, device, out)
        status == 0 || error(unsafe_string(ccall((:sdpx_b200_create_error, libsdpx), Cstring, ())))
    end
    h = B200Handle(out[])
    finalizer(h) do x
        x.ptr == C_NULL || ccall((:sdpx_b200_destroy, libsdpx), Cvoid, (Ptr{Cvoid},), x.ptr)
        x.ptr = C_NULL
    end
    if prob.dims.n > 0
        # SDPProblem.B (m×n, column-major) and .b; the KKT factor then carries the
        # equality block of src/kkt.jl:1466-1680 (FP64 precision mode only).
        B = Matrix{Float64}(prob.B)
        b = Vector{Float64}(prob.b)
        _check(h, ccall((:sdpx_b200_set_equality, libsdpx), Cint,
                        (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}), h.ptr,
                        Int32(prob.dims.n), B, b), "set_equality")
    end
    return h
end

"""Rank tolerance input `_requested_accuracy(opts)` (src/kkt.jl:518-521) and
`opts.equality_solver` (:auto → 0, :qr → 1)."""
set_equality_options!(h::B200Handle, requested::Float64, solver::Symbol) =
    _check(h, ccall((:sdpx_b200_set_equality_options, libsdpx), Cint,
                    (Ptr{Cvoid}, Float64, Cint), h.ptr, requested, solver === :qr ? 1 : 0),
           "set_equality_options")

"""Multipliers y (and dy, p = b − Bᵀx) of the equality rows."""
function multipliers(h::B200Handle, n::Integer)
    y, dy, p = zeros(n), zeros(n), zeros(n)
    _check(h, ccall((:sdpx_b200_get_multipliers, libsdpx), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), h.ptr, y, dy, p),
           "get_multipliers")
    return y, dy, p
end

set_precision!(h::B200Handle, mixed::Bool) =
    _check(h, ccall((:sdpx_b200_set_precision, libsdpx), Cint, (Ptr{Cvoid}, Cint), h.ptr, mixed ? 1 : 0),
           "set_precision")

# ------------------------------------------------- whole solve in one call ---
"""`sdpx_b200_solve_options`: SDPX's `SolverOptions{Float64}` fields the dense
core reads (src/types/workspaces.jl:101-185), enums as in include/sdpx_b200.h."""
mutable struct B200SolveOptions
    beta::Float64; gamma::Float64; omega_p::Float64; omega_d::Float64
    eps_gap::Float64; eps_primal::Float64; eps_dual::Float64
    iter_max::Int32; restart::Int32; min_step::Float64; omega_step::Float64
    max_restarts::Int32; max_centering::Int32; stall_iterations::Int32
    stall_tolerance::Float64; step_rule::Int32; refine_steps::Int32
    refine_policy::Int32; refine_max_steps::Int32; refine_tol::Float64
    max_time::Float64; parameter_policy::Int32; parameter_strategy::Int32
    adaptive_sigma_max::Float64; scaling::Int32; precision::Int32
    equality_solver::Int32
    B200SolveOptions() = new()
end

struct B200SolveResult
    status::Int32; iterations::Int32; restarts::Int32
    mixed_iterations::Int32; fp64_iterations::Int32
    p_obj::Float64; d_obj::Float64; p_res::Float64; d_res::Float64; seconds::Float64
    message::NTuple{256,UInt8}
end

"""`_solve_pipeline!` for the dense route run inside the library
(sdpx_b200_optimize): returns the result record and the solution (x, X, y, Y)
in the original coordinates."""
function optimize(h::B200Handle, prob::SDPX.SDPProblem{Float64}, tolerance::Float64;
                  mixed::Bool=false)
    o = B200SolveOptions()
    ccall((:sdpx_b200_default_options, libsdpx), Cvoid, (Ref{B200SolveOptions},), o)
    o.eps_gap = o.eps_primal = o.eps_dual = tolerance
    o.precision = mixed ? Int32(1) : Int32(0)
    res = Ref{B200SolveResult}()
    _check(h, ccall((:sdpx_b200_optimize, libsdpx), Cint,
                    (Ptr{Cvoid}, Ref{B200SolveOptions}, Ref{B200SolveResult}), h.ptr, o, res),
           "optimize")
    m, n = prob.dims.m, prob.dims.n
    stacked = sum(k -> k * k, prob.dims.k)
    x, X, y, Y = zeros(m), zeros(stacked), zeros(n), zeros(stacked)
    _check(h, ccall((:sdpx_b200_get_solution, libsdpx), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                    h.ptr, x, X, n > 0 ? y : C_NULL, Y), "get_solution")
    return res[], (x, X, y, Y)
end

# ------------------------------------------------------ KKT backend seam ---
"""`KKTBackend` whose methods run on the B200 (src/kkt_backend.jl:115-552)."""
struct B200DenseBackend <: SDPX.KKTBackend
    handle::B200Handle
end

SDPX.backend_name(::B200DenseBackend) = :b200_dense

# factorize! → (ok, reg_attempts, q_pivoted) shape of src/kkt.jl:1448-1463
function SDPX.factorize!(b::B200DenseBackend, ws, prob, opts)
    _check(b.handle, ccall((:sdpx_b200_schur_build, libsdpx), Cint, (Ptr{Cvoid}, Cint), b.handle.ptr, 0),
           "schur_build")
    ok = Ref{Cint}(0); attempts = Ref{Cint}(0); quality = Ref{Float64}(0)
    _check(b.handle, ccall((:sdpx_b200_factorize, libsdpx), Cint,
                           (Ptr{Cvoid}, Ref{Cint}, Ref{Cint}, Ref{Float64}),
                           b.handle.ptr, ok, attempts, quality), "factorize")
    return (ok[] == 1, Int(attempts[]), false)
end

function SDPX.solve_direction!(b::B200DenseBackend, ws, prob, opts, r)
    _check(b.handle, ccall((:sdpx_b200_solve, libsdpx), Cint, (Ptr{Cvoid},), b.handle.ptr), "solve")
    return true
end

function SDPX.refine!(b::B200DenseBackend, ws, prob, opts, r)
    steps = Ref{Cint}(0); resid = Ref{Float64}(0)
    _check(b.handle, ccall((:sdpx_b200_refine, libsdpx), Cint,
                           (Ptr{Cvoid}, Cint, Float64, Cint, Cint, Ref{Cint}, Ref{Float64}),
                           b.handle.ptr, 1, 0.0, 8, 0, steps, resid), "refine")  # auto policy, 64-ulp tol, cap 8
    return resid[]
end

# ------------------------------------------------------ provider seams ---
# Capabilities the B200 core executes for the dense Cholesky route
# (src/la_backend.jl:75-90 `_la_route_requirements(:dense_cholesky, …)`): the
# Schur Cholesky and its solves, the triangular solves, the Schur SYRK, owned
# products, iterative refinement against the FP64 operator and (mixed mode)
# the low-precision factor with higher-precision residuals.
const _B200_CAPABILITIES = SDPX.LAProviderCapabilities(
    cholesky=true, rank_revealing_qr=true, factor_solve=true, multi_rhs=true,
    iterative_refinement=true, higher_precision_residual=true,
    refinement_correction=true, mixed_precision_residual=true, dot=true,
    norminf=true, mul=true, mul_owned=true, syrk=true, triangular_solve=true,
    axpby=true)

_b200_library_ready() =
    Libc.Libdl.dlopen(libsdpx; throw_error=false) !== nothing

"""`SDPX.la_provider_descriptor` for Float64 (default at src/la_backend.jl:12-16,
the MultiFloat extension's at ext/SDPXMultiFloatLinearAlgebraExt.jl:743-765):
the B200 provider advertises the dense-Cholesky route's operations when the
library loads.  `plan_la_backend` reads it only for `provider = :b200`."""
function SDPX.la_provider_descriptor(::Type{Float64}, threads::Int=1)
    _b200_library_ready() || return (available=false, provider=:none, capabilities=(),
                                     capability_model=SDPX.LAProviderCapabilities(),
                                     reason=:missing_library)
    return (available=true, provider=:b200_cuda,
            capabilities=(:chol, :cholesky_factor!, :solve, :trsm, :trsv_lower,
                          :trsv_transpose, :syrk, :mul_owned, :rank_revealing_qr),
            capability_model=_B200_CAPABILITIES)
end

"""Provider payload of a planned `:b200` backend: the device ordinal and the
precision mode (`:fp64` or `:mixed`) the handle is created with."""
struct B200Provider
    device::Int
    precision::Symbol
end

SDPX.la_provider_capability_model(::B200Provider) = _B200_CAPABILITIES

"""Instantiate hook called by the patched `instantiate_la_backend` for
`config.selected === :b200` (beside `instantiate_multifloat_la_backend`,
src/la_backend.jl:508-570)."""
function SDPX.instantiate_b200_la_backend(::Type{Float64}, config::SDPX.LABackendConfiguration,
                                          threads::Int=1)
    config.provider === :b200_cuda || return nothing
    dev = parse(Int, get(ENV, "SDPX_B200_DEVICE", "0"))
    mode = Symbol(get(ENV, "SDPX_B200_PRECISION", "fp64"))
    mode in (:fp64, :mixed) || throw(ArgumentError("SDPX_B200_PRECISION must be fp64 or mixed"))
    return B200Provider(dev, mode)
end

"""Route hook called by the patched `_backend_from_configuration`
(src/kkt_backend.jl:86-100): a `DenseNormalEquations` formulation planned on
the `:b200` provider gets the device backend, with the iterate uploaded once."""
function SDPX.b200_backend_from_configuration(ws, prob::SDPX.SDPProblem{Float64},
                                              provider::B200Provider)
    h = B200Handle(prob; device=provider.device)
    set_precision!(h, provider.precision === :mixed)
    return B200DenseBackend(h)
end

"""Whole-loop hook: the patched `_solve_pipeline!` dense-SDP dispatch
(src/solver/interior_point.jl:3503-3515) calls this instead of
`_solve_sdp_core!` when the plan selected the `:b200` provider, so every
iterate stays in HBM for the whole solve (sdpx_b200_optimize)."""
function SDPX.b200_solve_sdp_core!(prob::SDPX.SDPProblem{Float64}, opts, provider::B200Provider)
    h = B200Handle(prob; device=provider.device)
    tol = min(opts.ϵ_gap, opts.ϵ_primal, opts.ϵ_dual)
    res, (x, Xs, y, Ys) = optimize(h, prob, tol; mixed=provider.precision === :mixed)
    return _to_result(prob, res, x, Xs, y, Ys)
end

# SDPX_B200_STATUS_* (include/sdpx_b200.h), 1-based, in SDPX's status names
const _STATUS = (:Optimal, :IterLimit, :Stalled, :InsufficientPrecision, :NumericalBreakdown,
                 :MaxRestarts, :TimeLimit)

function _unstack(prob, v)
    out, o = Matrix{Float64}[], 0
    for l in 1:prob.dims.L
        k = prob.dims.k[l]
        push!(out, reshape(v[o+1:o+k*k], k, k)); o += k * k
    end
    return out
end

function _to_result(prob, res::B200SolveResult, x, Xs, y, Ys)
    return (status=_STATUS[res.status], iterations=Int(res.iterations),
            x=x, X=_unstack(prob, Xs), y=y, Y=_unstack(prob, Ys),
            pObj=res.p_obj, dObj=res.d_obj, pRes=res.p_res, dRes=res.d_res,
            mixed_iterations=Int(res.mixed_iterations), seconds=res.seconds)
end

# ------------------------------------------- differentiation (rrule) ---
"""Solve on the B200 and return the solution (x, X, y, Y) in original
coordinates; differentiable through the ChainRulesCore `rrule` below."""
function b200_solve(prob::SDPX.SDPProblem{Float64}; tolerance::Float64=1e-9, device::Int=0)
    h = B200Handle(prob; device=device)
    res, (x, Xs, y, Ys) = optimize(h, prob, tolerance)
    r = _to_result(prob, res, x, Xs, y, Ys)
    return (x=r.x, X=r.X, y=r.y, Y=r.Y)
end

"""`rrule` for `b200_solve` (the Julia counterpart of a torch.autograd.Function):
the pullback factors the Newton system once more at the solution and calls the
hand-written adjoint kernel (sdpx_b200_adjoint), one KKT solve with the
cotangents as right-hand side, for the gradients with respect to c, b, C and
every A_i.  The tangent of `prob` is returned as a NamedTuple with fields
`c`, `b`, `C` (per block) and `A` (per variable, per block)."""
function ChainRulesCore.rrule(::typeof(b200_solve), prob::SDPX.SDPProblem{Float64};
                              tolerance::Float64=1e-9, device::Int=0)
    sol = b200_solve(prob; tolerance=tolerance, device=device)
    function b200_solve_pullback(Δ)
        Δ = ChainRulesCore.unthunk(Δ)
        m, n = prob.dims.m, prob.dims.n
        stacked = sum(k -> k * k, prob.dims.k)
        seed(v, len) = v isa ChainRulesCore.AbstractZero ? C_NULL : Vector{Float64}(v)
        seedblocks(v) = v isa ChainRulesCore.AbstractZero ? C_NULL :
                        reduce(vcat, [vec(Matrix{Float64}(b)) for b in v])
        wx, wy = seed(Δ.x, m), seed(Δ.y, n)
        WX, WY = seedblocks(Δ.X), seedblocks(Δ.Y)
        h = B200Handle(prob; device=device)
        Xs = reduce(vcat, vec.(sol.X)); Ys = reduce(vcat, vec.(sol.Y))
        _check(h, ccall((:sdpx_b200_set_iterate, libsdpx), Cint,
                        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                        h.ptr, sol.x, Xs, Ys), "set_iterate")
        pres = Ref{Float64}(0); dres = Ref{Float64}(0); okb = Ref{Cint}(0)
        mu = zeros(prob.dims.L)
        _check(h, ccall((:sdpx_b200_residuals, libsdpx), Cint,
                        (Ptr{Cvoid}, Ptr{Float64}, Cint, Cint, Ref{Float64}, Ref{Float64},
                         Ref{Cint}), h.ptr, mu, 1, 1, pres, dres, okb), "residuals")
        okb[] == 1 || error("solution blocks are not positive definite")
        _check(h, ccall((:sdpx_b200_schur_build, libsdpx), Cint, (Ptr{Cvoid}, Cint), h.ptr, 0),
               "schur_build")
        ok = Ref{Cint}(0); att = Ref{Cint}(0); q = Ref{Float64}(0)
        _check(h, ccall((:sdpx_b200_factorize, libsdpx), Cint,
                        (Ptr{Cvoid}, Ref{Cint}, Ref{Cint}, Ref{Float64}), h.ptr, ok, att, q),
               "factorize")
        ok[] == 1 || error("the Newton system at the solution could not be factored")
        gc, gb, gC = zeros(m), zeros(n), zeros(stacked)
        idx = Int32.(0:m-1)
        gA = zeros(stacked * m)
        _check(h, ccall((:sdpx_b200_adjoint, libsdpx), Cint,
                        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Int32},
                         Ptr{Float64}),
                        h.ptr, wx, wy, WX, WY, gc, n > 0 ? gb : C_NULL, gC, Int32(m), idx, gA),
               "adjoint")
        gA_blocks = [_unstack(prob, view(gA, i*stacked+1:(i+1)*stacked)) for i in 0:m-1]
        dprob = ChainRulesCore.Tangent{typeof(prob)}(; c=gc, b=gb, C=_unstack(prob, gC),
                                                     A=gA_blocks)
        return (ChainRulesCore.NoTangent(), dprob)
    end
    return sol, b200_solve_pullback
end

# ------------------------------------------------------------ certificate ---
struct B200Certificate
    valid::Int32; failures::Int32
    primal_psd_failing_blocks::Int32; dual_psd_failing_blocks::Int32
    primal_objective::Float64; dual_objective::Float64; gap::Float64; gap_relative::Float64
    primal_residual::Float64; dual_residual::Float64
    primal_affine_residual::Float64; dual_affine_residual::Float64
    primal_cone_violation::Float64; dual_cone_violation::Float64
    primal_residual_scaled::Float64; dual_residual_scaled::Float64
    equality_backward_error::Float64; equality_strict_backward_error::Float64
    primal_block_backward_error::Float64; primal_block_strict_backward_error::Float64
    dual_backward_error::Float64; dual_strict_backward_error::Float64
    complementarity::Float64; complementarity_relative::Float64
end

"""`result_certificate` (src/validation.jl:948-1115) recomputed on the B200."""
function certificate(h::B200Handle, result::SDPX.SDPResult{Float64}, opts)
    X = reduce(vcat, vec.(result.X)); Y = reduce(vcat, vec.(result.Y))
    out = Ref{B200Certificate}()
    _check(h, ccall((:sdpx_b200_certificate, libsdpx), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Float64,
                     Int32, Ref{B200Certificate}),
                    h.ptr, result.x, X, Y, opts.ϵ_primal, opts.ϵ_dual, opts.ϵ_gap,
                    opts.termination === :legacy ? 1 : 0, out), "certificate")
    return out[]
end

# ------------------------------------------------------ LP / SOC reduced system ---
mutable struct B200Normal
    ptr::Ptr{Cvoid}
end

"""Device copy of `LPStandardFormSystem` (src/lp_solver.jl:85-100) plus Lorentz cones."""
function B200Normal(B::Matrix{Float64}, n_lp::Integer, cone_dims::Vector{Int32},
                    row_for_variable::Vector{Int32}, coefficient::Vector{Float64},
                    n_weights::Integer; device::Integer=0)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rows0 = row_for_variable .- Int32(1)       # 0-based on the C side
    status = ccall((:sdpx_b200_normal_create, libsdpx), Cint,
                   (Int32, Int32, Ptr{Int32}, Int32, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Int32,
                    Cint, Ref{Ptr{Cvoid}}),
                   n_lp, length(cone_dims), cone_dims, size(B, 2), B, rows0, coefficient,
                   n_weights, device, out)
    status == 0 || error(unsafe_string(ccall((:sdpx_b200_normal_create_error, libsdpx), Cstring, ())))
    h = B200Normal(out[])
    finalizer(x -> (x.ptr == C_NULL || ccall((:sdpx_b200_normal_destroy, libsdpx), Cvoid,
                                              (Ptr{Cvoid},), x.ptr); x.ptr = C_NULL), h)
    return h
end

"""`_native_soc_scaling!` (src/soc_native.jl:1083-1098): (ok, failed_block)."""
function nt_scaling!(h::B200Normal, s::Vector{Float64}, z::Vector{Float64}, ncones::Integer)
    ok = zeros(Int32, ncones)
    status = ccall((:sdpx_b200_normal_nt_scaling, libsdpx), Cint,
                   (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Ptr{Float64},
                    Ptr{Float64}, Ptr{Float64}),
                   h.ptr, s, z, ok, C_NULL, C_NULL, C_NULL, C_NULL)
    status < 0 && error("nt_scaling failed")
    bad = findfirst(==(0), ok)
    return bad === nothing ? (true, 0) : (false, bad)
end

"""`_lp_factor_reduced!` with the ×10 regularization retries (src/lp_solver.jl:4090-4115)."""
function factor_reduced!(h::B200Normal, weights::Vector{Float64}, regularization::Float64)
    attempts = Ref{Int32}(0); used = Ref{Float64}(0)
    status = ccall((:sdpx_b200_normal_factorize, libsdpx), Cint,
                   (Ptr{Cvoid}, Ptr{Float64}, Float64, Int32, Ref{Int32}, Ref{Float64}),
                   h.ptr, weights, regularization, 8, attempts, used)
    status < 0 && error("factorize failed")
    return (status == 0, Int(attempts[]), used[])
end

"""`_lp_solve_factor!` (src/lp_solver.jl:2177-2213): rhs = [rx; ry] → [dx; dy] in place."""
function solve_factor!(h::B200Normal, rhs::Vector{Float64})
    status = ccall((:sdpx_b200_normal_solve, libsdpx), Cint, (Ptr{Cvoid}, Ptr{Float64}), h.ptr, rhs)
    status == 0 || throw(LinearAlgebra.PosDefException(1))
    return rhs
end

# --------------------------------------------- batched small SDPs ---------
# include/sdpx_b200_batch.h: many one-block SDPs in one pooled device
# workspace, one kernel per interior-point phase over all of them.  SDPX has no
# batch solver; this replaces a loop of `SDPX.solve` calls over instances.
struct B200BatchProblem
    count::Int32
    block_order::Ptr{Int32}
    m::Ptr{Int32}
    Av::Ptr{Ptr{Float64}}
    C::Ptr{Ptr{Float64}}
    c::Ptr{Ptr{Float64}}
end

mutable struct B200Batch
    ptr::Ptr{Cvoid}
    count::Int
    dims::Vector{Tuple{Int,Int}}  # (k, m) per instance
end

"""Upload one-block problems (each `prob.dims.L == 1`, `prob.dims.n == 0`,
3 ≤ k ≤ 64, m ≤ 256) into one batch workspace."""
function B200Batch(probs::Vector{<:SDPX.SDPProblem{Float64}}; device::Integer=0)
    n = length(probs)
    ks = Int32[p.dims.k[1] for p in probs]
    ms = Int32[p.dims.m for p in probs]
    Av = [Matrix{Float64}((p.cons::SDPX.DenseCons{Float64}).Av[1]) for p in probs]  # k²×m
    Cm = [Matrix{Float64}(p.C[1]) for p in probs]
    cv = [Vector{Float64}(p.c) for p in probs]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve ks ms Av Cm cv begin
        pA = [pointer(a) for a in Av]; pC = [pointer(a) for a in Cm]; pc = [pointer(a) for a in cv]
        GC.@preserve pA pC pc begin
            bp = B200BatchProblem(Int32(n), pointer(ks), pointer(ms), pointer(pA), pointer(pC),
                                  pointer(pc))
            status = ccall((:sdpx_b200_batch_create, libsdpx), Cint,
                           (Ref{B200BatchProblem}, Cint, Ref{Ptr{Cvoid}}), bp, device, out)
            status == 0 || error(unsafe_string(ccall((:sdpx_b200_batch_create_error, libsdpx),
                                                     Cstring, ())))
        end
    end
    b = B200Batch(out[], n, [(Int(ks[i]), Int(ms[i])) for i in 1:n])
    finalizer(x -> (x.ptr == C_NULL || ccall((:sdpx_b200_batch_destroy, libsdpx), Cvoid,
                                             (Ptr{Cvoid},), x.ptr)), b)
    return b
end

function _bcheck(b::B200Batch, status::Cint, what)
    status == 0 && return nothing
    msg = unsafe_string(ccall((:sdpx_b200_batch_last_error, libsdpx), Cstring, (Ptr{Cvoid},),
                              b.ptr))
    error("sdpx_b200_batch_$(what): $(msg)")
end

"""Times the Schur launch shapes on the device and keeps the fastest
(sdpx_b200_batch_autotune); returns rows (threads, tile, grain, ms)."""
function autotune!(b::B200Batch, o::B200SolveOptions)
    table = zeros(4 * 64)
    cnt = Ref{Int32}(0)
    _bcheck(b, ccall((:sdpx_b200_batch_autotune, libsdpx), Cint,
                     (Ptr{Cvoid}, Ref{B200SolveOptions}, Ptr{Float64}, Int32, Ref{Int32}),
                     b.ptr, o, table, Int32(64), cnt), "autotune")
    return [Tuple(table[4i+1:4i+4]) for i in 0:cnt[]-1]
end

"""Solve every instance of the batch with the fixed start and no
equilibration (the options the batched engine serves); per instance the
status, iterations, objectives and (x, X, Y).  `float64x2` forms and solves
the Newton system in double-double (for gaps such as 1e-12); `bisection`
selects the reference's Cholesky-trial bisection for the affine step bounds
instead of the eigenvalue bound."""
function optimize(b::B200Batch, tolerance::Float64; autotune::Bool=false,
                  float64x2::Bool=false, bisection::Bool=false)
    o = B200SolveOptions()
    ccall((:sdpx_b200_default_options, libsdpx), Cvoid, (Ref{B200SolveOptions},), o)
    o.eps_gap = o.eps_primal = o.eps_dual = tolerance
    o.parameter_policy = Int32(1)
    o.scaling = Int32(1)
    o.precision = float64x2 ? Int32(2) : Int32(0)
    _bcheck(b, ccall((:sdpx_b200_batch_set_step_bounds, libsdpx), Cint, (Ptr{Cvoid}, Int32),
                     b.ptr, bisection ? Int32(0) : Int32(1)), "set_step_bounds")
    autotune && autotune!(b, o)
    res = Vector{B200SolveResult}(undef, b.count)
    _bcheck(b, ccall((:sdpx_b200_batch_optimize, libsdpx), Cint,
                     (Ptr{Cvoid}, Ref{B200SolveOptions}, Ptr{B200SolveResult}), b.ptr, o, res),
            "optimize")
    # every instance's (x, X, Y) in one read-back, concatenated in input order
    mt = sum(d[2] for d in b.dims)
    kt = sum(d[1]^2 for d in b.dims)
    xs, Xs, Ys = zeros(mt), zeros(kt), zeros(kt)
    _bcheck(b, ccall((:sdpx_b200_batch_get_solutions, libsdpx), Cint,
                     (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                     b.ptr, xs, Xs, Ys), "get_solutions")
    out = Vector{Any}(undef, b.count)
    mo = ko = 0
    for i in 1:b.count
        k, m = b.dims[i]
        x = xs[mo+1:mo+m]
        X = reshape(Xs[ko+1:ko+k*k], k, k)
        Y = reshape(Ys[ko+1:ko+k*k], k, k)
        mo += m
        ko += k * k
        r = res[i]
        out[i] = (status=_STATUS[r.status], iterations=Int(r.iterations), x=x,
                  X=X, Y=Y, pObj=r.p_obj, dObj=r.d_obj, pRes=r.p_res, dRes=r.d_res)
    end
    return out
end

"""Certificates of every instance's current solution (after `optimize`) in one
device kernel and one read-back (sdpx_b200_batch_certificate)."""
function certificate(b::B200Batch, tolerance::Float64; legacy::Bool=false)
    out = Vector{B200Certificate}(undef, b.count)
    _bcheck(b, ccall((:sdpx_b200_batch_certificate, libsdpx), Cint,
                     (Ptr{Cvoid}, Float64, Float64, Float64, Int32, Ptr{B200Certificate}),
                     b.ptr, tolerance, tolerance, tolerance, legacy ? Int32(1) : Int32(0), out),
            "certificate")
    return out
end

end # module
