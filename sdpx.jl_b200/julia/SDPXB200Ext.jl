# SDPX package extension binding libsdpx_b200.so (sm_100a) through ccall.
#
# This file is the reference-side glue a maintainer adds as ext/SDPXB200Ext.jl
# (with `[weakdeps] CUDA` / `[extensions] SDPXB200Ext = "CUDA"` in Project.toml).
# It is written against SDPX's seams but is not executed in this repository's
# tests: the build environment has no Julia.  Every ccall below matches a
# declaration in include/sdpx_b200.h or include/sdpx_b200_normal.h.
module SDPXB200Ext

using SDPX
using LinearAlgebra

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

end # module
