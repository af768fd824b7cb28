# PDCSB200.jl -- Julia binding of libpdcs_b200.so (include/pdcs.h) for the
# reference's callers.
#
#   rpdhg_gpu_solve(; ...)                  same keywords, defaults and result
#                                           fields as PDCS_GPU.rpdhg_gpu_solve
#                                           (src/pdcs_gpu/rpdhg_alg_gpu_gen.jl:1219-1268)
#   rpdhg_gpu_solve_input_gpu_data(; ...)   device-resident inputs (:387), raw
#                                           device pointers or CuArrays
#   rpdhg_gpu_solve_batch(problems; ...)    many programs in one call
#   BatchHandle / batch_solve / batch_grad  prepared batch and the solution-map adjoint
#   conic_layer + ChainRulesCore.rrule      x*(c, h, G.nzval, bl, bu) with a pullback
#                                           through pdcs_batch_grad
#   forward_moi!()                          points the reference's MOI wrapper
#                                           (src/pdcs_gpu/MOI_wrapper/MOI_wrapper.jl:610,
#                                           :661) at this binding
#
# The structs below repeat the C structs of include/pdcs.h field by field, in
# order, with the same widths (Julia lays isbits structs out like C).
# Julia is not installed where this library is built, so this file is
# checked there only structurally (tests/test_julia_binding.py compares its
# struct layouts with include/pdcs.h); it has not been run.
module PDCSB200

using LinearAlgebra
using SparseArrays

export rpdhg_gpu_solve, rpdhg_gpu_solve_input_gpu_data, rpdhg_gpu_solve_batch,
       BatchHandle, batch_solve, batch_grad, ConicStructure, conic_layer, forward_moi!

const libpdcs = Ref{String}(normpath(joinpath(@__DIR__, "..", "libpdcs_b200.so")))
set_library!(path::AbstractString) = (libpdcs[] = String(path))

# ---------------------------------------------------------------------------
# C structs (include/pdcs.h)
# ---------------------------------------------------------------------------
struct PdcsProblem
    n::Int64
    m::Int64
    nb::Int64
    nnz::Int64
    G_rowptr::Ptr{Int32}
    G_colind::Ptr{Int32}
    G_val::Ptr{Float64}
    c::Ptr{Float64}
    h::Ptr{Float64}
    bl::Ptr{Float64}
    bu::Ptr{Float64}
    mGzero::Int64
    mGnonnegative::Int64
    socG::Ptr{Int64}
    n_socG::Int64
    rsocG::Ptr{Int64}
    n_rsocG::Int64
    expG::Int64
    dual_expG::Int64
    soc_x::Ptr{Int64}
    n_soc_x::Int64
    rsoc_x::Ptr{Int64}
    n_rsoc_x::Int64
    exp_x::Int64
    dual_exp_x::Int64
    on_device::Int32
    reserved::Int32
end

mutable struct PdcsOptions
    rescaling_method::Int32
    use_preconditioner::Int32
    use_adaptive_restart::Int32
    use_adaptive_step_size_weight::Int32
    use_aggressive::Int32
    use_accelerated::Int32
    use_resolving::Int32
    warm_start::Int32
    primal_sol::Ptr{Float64}
    dual_sol::Ptr{Float64}
    max_outer_iter::Int64
    max_inner_iter::Int64
    abs_tol::Float64
    rel_tol::Float64
    eps_primal_infeasible_low_acc::Float64
    eps_dual_infeasible_low_acc::Float64
    eps_primal_infeasible_high_acc::Float64
    eps_dual_infeasible_high_acc::Float64
    print_freq::Int64
    check_terminate_freq::Int64
    verbose::Int32
    use_kkt_restart::Int32
    time_limit::Float64
    kkt_restart_freq::Int64
    use_duality_gap_restart::Int32
    precision::Int32
    duality_gap_restart_freq::Int64
    attempt_limit::Int64
    stream::Ptr{Cvoid}
    attempts_per_graph::Int32
    force_resolving::Int32
    spmv_lane_nnz::Int32
    differentiable::Int32
    spmv_tiles::Int32
    reserved::Int32
    PdcsOptions() = new()
end

mutable struct PdcsResult
    x::Ptr{Float64}
    y::Ptr{Float64}
    x_device::Ptr{Float64}
    y_device::Ptr{Float64}
    exit_code::Int32
    returned_sequence::Int32
    pObj::Float64
    dObj::Float64
    iter::Int64
    restart_used::Int64
    time::Float64
    setup_time::Float64
    l_inf_rel_primal_res::Float64
    l_inf_rel_dual_res::Float64
    rel_gap::Float64
    l_2_rel_primal_res::Float64
    l_2_rel_dual_res::Float64
    l_inf_abs_primal_res::Float64
    l_inf_abs_dual_res::Float64
    abs_gap::Float64
    kernel_launches::Int64
    graph_launches::Int64
    time_iterations::Float64
    time_exit_checks::Float64
    time_restarts::Float64
    restart_probes::Int64
    spmv_lane_nnz_G::Int32
    spmv_lane_nnz_Gt::Int32
    PdcsResult() = new()
end

mutable struct PdcsBatchInfo
    setup_time::Float64
    solve_time::Float64
    time_iterations::Float64
    kernel_launches::Int64
    graph_launches::Int64
    service_rounds::Int64
    single_fallbacks::Int64
    spmv_tiled::Int32
    tail_rounds::Int32
    PdcsBatchInfo() = new()
end

mutable struct PdcsGradOptions
    rel_tol::Float64
    restart::Int32
    reserved::Int32
    max_iter::Int64
end
PdcsGradOptions() = PdcsGradOptions(1e-10, 100, 0, 5000)

mutable struct PdcsGradInfo
    iterations::Int64
    residual::Float64
    time::Float64
    converged::Int32
    reserved::Int32
    PdcsGradInfo() = new()
end

# status codes and exit codes (include/pdcs.h; def_struct.jl:735-745)
const STATUS_TEXT = Dict(-1 => "invalid argument", -2 => "CUDA error",
    -3 => "m does not match the sum of mGzero, mGnonnegative, socG, rsocG, 3 (expG + dual_expG)",
    -4 => "an SOC block has dimension < 2", -5 => "an RSOC block has dimension < 3",
    -6 => "Not all elements of bl are less than or equal to the corresponding elements in bu",
    -7 => "cone blocks of x exceed n", -8 => "no CUDA device", -9 => "option combination not implemented",
    -10 => "problem exceeds the fixed scratch of pdcs_spmv_csr_noalloc")
const EXIT_STATUS = Dict(0 => :optimal, 1 => :max_iter, 2 => :primal_infeasible_low_acc,
    3 => :primal_infeasible_high_acc, 4 => :dual_infeasible_low_acc, 5 => :dual_infeasible_high_acc,
    6 => :time_limit, 7 => :continue, 8 => :numerical_error_nan, 9 => :numerical_error_inf,
    10 => :attempt_limit)
const RESCALING = Dict(:none => 0, :ruiz => 1, :pock_chambolle => 2, :ruiz_pock_chambolle => 3)

check(rc, what) = rc == 0 || error("$what: status $rc ($(get(STATUS_TEXT, Int(rc), "unknown")))")

# ---------------------------------------------------------------------------
# Options (the keyword arguments of rpdhg_gpu_solve, rpdhg_alg_gpu_gen.jl:1219-1268)
# ---------------------------------------------------------------------------
function make_options(; n, m, rescaling_method::Symbol = :ruiz_pock_chambolle, use_preconditioner::Bool = true,
                      use_adaptive_restart::Bool = true, use_adaptive_step_size_weight::Bool = true,
                      use_aggressive::Bool = true, use_accelerated::Bool = false, use_resolving::Bool = true,
                      primal_sol::Vector{Float64} = zeros(n), dual_sol::Vector{Float64} = zeros(m),
                      warm_start::Bool = false, max_outer_iter::Integer = 10000, max_inner_iter::Integer = 500000,
                      abs_tol::Float64 = 1e-6, rel_tol::Float64 = 1e-6,
                      eps_primal_infeasible_low_acc::Float64 = 1e-12, eps_dual_infeasible_low_acc::Float64 = 1e-12,
                      eps_primal_infeasible_high_acc::Float64 = 1e-16,
                      eps_dual_infeasible_high_acc::Float64 = 1e-16, print_freq::Integer = 2000,
                      check_terminate_freq::Integer = 2000, verbose::Integer = 1, time_limit::Float64 = Inf,
                      method::Symbol = :average, logfile_name::Union{String, Nothing} = nothing,
                      use_kkt_restart::Bool = false, kkt_restart_freq::Integer = 2000,
                      use_duality_gap_restart::Bool = true, duality_gap_restart_freq::Integer = 2000,
                      precision::Symbol = :fp64, attempt_limit::Integer = 0, stream::Ptr{Cvoid} = C_NULL,
                      spmv_lane_nnz::Integer = 0, spmv_tiles::Integer = 0, differentiable::Bool = false)
    method in (:average, :halpern) || error("method only available for :average and :halpern")
    method == :halpern && error("method = :halpern is not wired into the reference GPU module either")
    if warm_start && (length(primal_sol) != n || length(dual_sol) != m)
        error("Warmstart doesn't match the problem size")
    end
    o = Ref(PdcsOptions())
    check(ccall((:pdcs_default_options, libpdcs[]), Cint, (Ref{PdcsOptions},), o), "pdcs_default_options")
    O = o[]
    O.rescaling_method = RESCALING[rescaling_method]
    O.use_preconditioner = use_preconditioner
    O.use_adaptive_restart = use_adaptive_restart
    O.use_adaptive_step_size_weight = use_adaptive_step_size_weight
    O.use_aggressive = use_aggressive
    O.use_accelerated = use_accelerated
    O.use_resolving = use_resolving
    O.warm_start = warm_start
    O.primal_sol = warm_start ? pointer(primal_sol) : C_NULL   # caller keeps them alive (GC.@preserve)
    O.dual_sol = warm_start ? pointer(dual_sol) : C_NULL
    O.max_outer_iter = max_outer_iter
    O.max_inner_iter = max_inner_iter
    O.abs_tol = abs_tol
    O.rel_tol = rel_tol
    O.eps_primal_infeasible_low_acc = eps_primal_infeasible_low_acc
    O.eps_dual_infeasible_low_acc = eps_dual_infeasible_low_acc
    O.eps_primal_infeasible_high_acc = eps_primal_infeasible_high_acc
    O.eps_dual_infeasible_high_acc = eps_dual_infeasible_high_acc
    O.print_freq = print_freq
    O.check_terminate_freq = check_terminate_freq
    O.verbose = verbose
    O.use_kkt_restart = use_kkt_restart
    O.time_limit = isfinite(time_limit) ? time_limit : 0.0
    O.kkt_restart_freq = kkt_restart_freq
    O.use_duality_gap_restart = use_duality_gap_restart
    O.duality_gap_restart_freq = duality_gap_restart_freq
    O.precision = precision == :fp32 ? 1 : 0
    O.attempt_limit = attempt_limit
    O.stream = stream
    O.spmv_lane_nnz = spmv_lane_nnz
    O.spmv_tiles = spmv_tiles
    O.differentiable = differentiable
    # logfile_name: the library prints to stdout (verbose); a caller that wants a
    # file redirects stdout, as the reference's Tee logger does (PDCS_GPU.jl:66-91)
    return O
end

# ---------------------------------------------------------------------------
# Host problems: CSR of G from a SparseMatrixCSC (CSC of G' == CSR of G), 0-based
# ---------------------------------------------------------------------------
struct HostData
    rowptr::Vector{Int32}
    colind::Vector{Int32}
    val::Vector{Float64}
    c::Vector{Float64}
    h::Vector{Float64}
    bl::Vector{Float64}
    bu::Vector{Float64}
    socG::Vector{Int64}
    rsocG::Vector{Int64}
    soc_x::Vector{Int64}
    rsoc_x::Vector{Int64}
end

function host_data(; n, m, nb, c, G::AbstractMatrix, h, socG, rsocG, bl, bu, soc_x, rsoc_x, kw...)
    size(G) == (m, n) || error("G is $(size(G)), expected ($m, $n)")
    Gt = SparseMatrixCSC(sparse(G)')
    return HostData(Int32.(Gt.colptr .- 1), Int32.(Gt.rowval .- 1), Vector{Float64}(Gt.nzval),
                    Vector{Float64}(c), Vector{Float64}(Vector(h)), Vector{Float64}(bl), Vector{Float64}(bu),
                    Int64.(socG), Int64.(rsocG), Int64.(soc_x), Int64.(rsoc_x))
end

ptr_or_null(a::Vector) = isempty(a) ? Ptr{eltype(a)}(C_NULL) : pointer(a)

function problem_struct(d::HostData; n, m, nb, mGzero, mGnonnegative, expG, dual_expG, exp_x = 0,
                        dual_exp_x = 0, kw...)
    return PdcsProblem(n, m, nb, length(d.val), ptr_or_null(d.rowptr), ptr_or_null(d.colind), ptr_or_null(d.val),
                       ptr_or_null(d.c), ptr_or_null(d.h), ptr_or_null(d.bl), ptr_or_null(d.bu),
                       mGzero, mGnonnegative, ptr_or_null(d.socG), length(d.socG), ptr_or_null(d.rsocG),
                       length(d.rsocG), expG, dual_expG, ptr_or_null(d.soc_x), length(d.soc_x),
                       ptr_or_null(d.rsoc_x), length(d.rsoc_x), exp_x, dual_exp_x, 0, 0)
end

const PROBLEM_KEYS = (:n, :m, :nb, :c, :G, :h, :mGzero, :mGnonnegative, :socG, :rsocG, :expG, :dual_expG,
                      :bl, :bu, :soc_x, :rsoc_x, :exp_x, :dual_exp_x, :Dl, :Dr)
split_kw(kw) = (Dict(k => v for (k, v) in kw if k in PROBLEM_KEYS), Dict(k => v for (k, v) in kw if !(k in PROBLEM_KEYS)))

# The reference's Solution, as far as its callers read it (MOI_wrapper.jl:648-658):
# sol.x.recovered_primal.primal_sol.x, sol.y.recovered_dual.dual_sol.y,
# sol.y.slack.primal_sol.x (lambda = c - G'y), sol.info.{exit_status, exit_code, pObj, dObj, iter, time}.
function solution(x, y, lam, R::PdcsResult)
    info = (exit_status = get(EXIT_STATUS, Int(R.exit_code), :unknown), exit_code = Int(R.exit_code),
            pObj = R.pObj, dObj = R.dObj, iter = R.iter, time = R.time, restart_used = R.restart_used,
            setup_time = R.setup_time, l_inf_rel_primal_res = R.l_inf_rel_primal_res,
            l_inf_rel_dual_res = R.l_inf_rel_dual_res, rel_gap = R.rel_gap, abs_gap = R.abs_gap)
    return (x = (recovered_primal = (primal_sol = (x = x,),),),
            y = (recovered_dual = (dual_sol = (y = y,),), slack = (primal_sol = (x = lam,),)),
            info = info, result = R)
end

function rpdhg_gpu_solve(; kw...)
    pk, ok = split_kw(kw)
    n, m = pk[:n], pk[:m]
    d = host_data(; pk...)
    x, y = zeros(n), zeros(m)
    R = Ref(PdcsResult())
    GC.@preserve d x y begin
        prob = Ref(problem_struct(d; pk...))
        O = Ref(make_options(; n = n, m = m, ok...))
        GC.@preserve O begin
            R[].x, R[].y, R[].x_device, R[].y_device = pointer(x), pointer(y), C_NULL, C_NULL
            check(ccall((:pdcs_solve, libpdcs[]), Cint, (Ref{PdcsProblem}, Ref{PdcsOptions}, Ref{PdcsResult}),
                        prob, O, R), "pdcs_solve")
        end
    end
    lam = d.c .- sparse(pk[:G])' * y
    return solution(x, y, lam, R[])
end

# Device-resident inputs (rpdhg_gpu_solve_input_gpu_data, rpdhg_alg_gpu_gen.jl:387): G as 0-based
# int32 CSR device buffers (rowptr, colind, val) and c, h, bl, bu as device pointers; the
# solution is written to the device buffers x_device (n) and y_device (m).  With CUDA.jl,
# pass pointer(cuarray) (a CuPtr) reinterpreted as Ptr: reinterpret(Ptr{Float64}, pointer(a)).
function rpdhg_gpu_solve_input_gpu_data(; n, m, nb, nnz, G_rowptr::Ptr{Int32}, G_colind::Ptr{Int32},
                                        G_val::Ptr{Float64}, c::Ptr{Float64}, h::Ptr{Float64},
                                        bl::Ptr{Float64}, bu::Ptr{Float64}, mGzero, mGnonnegative,
                                        socG, rsocG, expG, dual_expG, soc_x, rsoc_x, exp_x = 0, dual_exp_x = 0,
                                        x_device::Ptr{Float64}, y_device::Ptr{Float64}, kw...)
    s, r, sx, rx = Int64.(socG), Int64.(rsocG), Int64.(soc_x), Int64.(rsoc_x)
    R = Ref(PdcsResult())
    GC.@preserve s r sx rx begin
        prob = Ref(PdcsProblem(n, m, nb, nnz, G_rowptr, G_colind, G_val, c, h, bl, bu, mGzero, mGnonnegative,
                               ptr_or_null(s), length(s), ptr_or_null(r), length(r), expG, dual_expG,
                               ptr_or_null(sx), length(sx), ptr_or_null(rx), length(rx), exp_x, dual_exp_x, 1, 0))
        O = Ref(make_options(; n = n, m = m, kw...))
        R[].x, R[].y, R[].x_device, R[].y_device = C_NULL, C_NULL, x_device, y_device
        check(ccall((:pdcs_solve, libpdcs[]), Cint, (Ref{PdcsProblem}, Ref{PdcsOptions}, Ref{PdcsResult}),
                    prob, O, R), "pdcs_solve")
    end
    return R[]
end

# ---------------------------------------------------------------------------
# Batches: problems is a vector of keyword collections (NamedTuples or Dicts)
# with rpdhg_gpu_solve's problem keywords; options apply to every instance.
# ---------------------------------------------------------------------------
mutable struct BatchHandle
    ptr::Ptr{Cvoid}
    data::Vector{HostData}
    kws::Vector{Dict{Symbol, Any}}
end

function BatchHandle(problems::AbstractVector; kw...)
    kws = [Dict{Symbol, Any}(pairs(p)) for p in problems]
    data = [host_data(; k...) for k in kws]
    probs = [problem_struct(d; k...) for (d, k) in zip(data, kws)]
    O = Ref(make_options(; n = 0, m = 0, kw...))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve data begin
        check(ccall((:pdcs_batch_create, libpdcs[]), Cint, (Int64, Ptr{PdcsProblem}, Ref{PdcsOptions}, Ref{Ptr{Cvoid}}),
                    length(probs), probs, O, out), "pdcs_batch_create")
    end
    h = BatchHandle(out[], data, kws)
    finalizer(close, h)  # the host arrays in `data` stay alive with the handle
    return h
end

function Base.close(h::BatchHandle)
    if h.ptr != C_NULL
        ccall((:pdcs_batch_destroy, libpdcs[]), Cvoid, (Ptr{Cvoid},), h.ptr)
        h.ptr = C_NULL
    end
    return nothing
end

function batch_solve(h::BatchHandle; attempt_limit::Integer = 0)
    K = length(h.data)
    xs = [zeros(k[:n]) for k in h.kws]
    ys = [zeros(k[:m]) for k in h.kws]
    res = [PdcsResult() for _ in 1:K]
    for (r, x, y) in zip(res, xs, ys)
        r.x, r.y, r.x_device, r.y_device = pointer(x), pointer(y), C_NULL, C_NULL
    end
    flat = Vector{PdcsResult}(undef, 0)
    info = Ref(PdcsBatchInfo())
    # the C side writes an array of pdcs_result: lay the structs out contiguously
    buf = Vector{UInt8}(undef, K * sizeof(PdcsResult))
    GC.@preserve xs ys buf res begin
        for k in 1:K
            unsafe_store!(Ptr{PdcsResult}(pointer(buf)) + (k - 1) * sizeof(PdcsResult), res[k])
        end
        check(ccall((:pdcs_batch_solve, libpdcs[]), Cint, (Ptr{Cvoid}, Int64, Ptr{UInt8}, Ref{PdcsBatchInfo}),
                    h.ptr, attempt_limit, buf, info), "pdcs_batch_solve")
        for k in 1:K
            push!(flat, unsafe_load(Ptr{PdcsResult}(pointer(buf)) + (k - 1) * sizeof(PdcsResult)))
        end
    end
    sols = [solution(xs[k], ys[k], h.data[k].c .- sparse(h.kws[k][:G])' * ys[k], flat[k]) for k in 1:K]
    return sols, info[]
end

function rpdhg_gpu_solve_batch(problems::AbstractVector; kw...)
    h = BatchHandle(problems; kw...)
    try
        return batch_solve(h)
    finally
        close(h)
    end
end

# Gradients at the last batch_solve of a handle made with differentiable = true:
# dldx[k] = dL/dx*_k; returns, per instance, (c, h, G, bl, bu) with G the nonzero
# values of the instance's CSR matrix (row-major order of G).
function batch_grad(h::BatchHandle, dldx::AbstractVector; dldy = nothing, rel_tol = 1e-10, restart = 100,
                    max_iter = 5000)
    K = length(h.data)
    gx = [Vector{Float64}(v) for v in dldx]
    gy = dldy === nothing ? nothing : [Vector{Float64}(v) for v in dldy]
    dc = [zeros(k[:n]) for k in h.kws]
    dh = [zeros(k[:m]) for k in h.kws]
    dG = [zeros(length(d.val)) for d in h.data]
    dl = [zeros(k[:nb]) for k in h.kws]
    du = [zeros(k[:nb]) for k in h.kws]
    P(v) = [ptr_or_null(a) for a in v]
    go = Ref(PdcsGradOptions(rel_tol, restart, 0, max_iter))
    infos = [PdcsGradInfo() for _ in 1:K]
    ibuf = Vector{UInt8}(undef, K * sizeof(PdcsGradInfo))
    GC.@preserve gx gy dc dh dG dl du ibuf begin
        check(ccall((:pdcs_batch_grad, libpdcs[]), Cint,
                    (Ptr{Cvoid}, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}},
                     Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Ref{PdcsGradOptions}, Ptr{UInt8}),
                    h.ptr, P(gx), gy === nothing ? Ptr{Ptr{Float64}}(C_NULL) : P(gy), P(dc), P(dh), P(dG), P(dl),
                    P(du), go, ibuf), "pdcs_batch_grad")
        for k in 1:K
            infos[k] = unsafe_load(Ptr{PdcsGradInfo}(pointer(ibuf)) + (k - 1) * sizeof(PdcsGradInfo))
        end
    end
    return [(c = dc[k], h = dh[k], G = dG[k], bl = dl[k], bu = du[k]) for k in 1:K], infos
end

# ---------------------------------------------------------------------------
# ChainRules: a conic layer x* = conic_layer(c, h, Gval, bl, bu, s) where Gval
# holds G's nonzero values in the CSR order of the structure s (sparsity,
# cones, options); the pullback runs pdcs_batch_grad and returns dL/dc, dL/dh,
# dL/dGval, dL/dbl, dL/dbu.
# ---------------------------------------------------------------------------
struct ConicStructure
    n::Int
    m::Int
    nb::Int
    rowptr::Vector{Int32}   # 0-based CSR of G
    colind::Vector{Int32}
    cones::Dict{Symbol, Any}    # mGzero, mGnonnegative, socG, rsocG, expG, dual_expG, soc_x, rsoc_x, exp_x, dual_exp_x
    options::Dict{Symbol, Any}  # rpdhg_gpu_solve's option keywords
end

function ConicStructure(; n, m, nb, G::AbstractMatrix, options = Dict{Symbol, Any}(), cones...)
    Gt = SparseMatrixCSC(sparse(G)')
    return ConicStructure(n, m, nb, Int32.(Gt.colptr .- 1), Int32.(Gt.rowval .- 1), Dict{Symbol, Any}(cones),
                          Dict{Symbol, Any}(options))
end

function _layer_handle(c, h, Gval, bl, bu, s::ConicStructure)
    cn = s.cones
    d = HostData(s.rowptr, s.colind, Vector{Float64}(Gval), Vector{Float64}(c), Vector{Float64}(h),
                 Vector{Float64}(bl), Vector{Float64}(bu), Int64.(get(cn, :socG, Int[])), Int64.(get(cn, :rsocG, Int[])),
                 Int64.(get(cn, :soc_x, Int[])), Int64.(get(cn, :rsoc_x, Int[])))
    kw = Dict{Symbol, Any}(:n => s.n, :m => s.m, :nb => s.nb, :mGzero => get(cn, :mGzero, 0),
                           :mGnonnegative => get(cn, :mGnonnegative, 0), :expG => get(cn, :expG, 0),
                           :dual_expG => get(cn, :dual_expG, 0), :exp_x => get(cn, :exp_x, 0),
                           :dual_exp_x => get(cn, :dual_exp_x, 0),
                           :G => SparseMatrixCSC(sparse(Int.(repeat_rows(s.rowptr)), Int.(s.colind) .+ 1, d.val,
                                                        s.m, s.n)))
    prob = [problem_struct(d; kw...)]
    O = Ref(make_options(; n = s.n, m = s.m, differentiable = true, s.options...))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve d begin
        check(ccall((:pdcs_batch_create, libpdcs[]), Cint, (Int64, Ptr{PdcsProblem}, Ref{PdcsOptions}, Ref{Ptr{Cvoid}}),
                    1, prob, O, out), "pdcs_batch_create")
    end
    hd = BatchHandle(out[], [d], [kw])
    finalizer(close, hd)
    return hd
end

# row index (1-based) of every nonzero of a 0-based CSR
repeat_rows(rowptr) = reduce(vcat, [fill(i, rowptr[i + 1] - rowptr[i]) for i in 1:length(rowptr) - 1]; init = Int[])

function conic_layer(c, h, Gval, bl, bu, s::ConicStructure)
    hd = _layer_handle(c, h, Gval, bl, bu, s)
    try
        sols, _ = batch_solve(hd)
        return sols[1].x.recovered_primal.primal_sol.x
    finally
        close(hd)
    end
end

# ChainRulesCore is optional: the rrule is defined when the package is available.
if Base.find_package("ChainRulesCore") !== nothing
    @eval import ChainRulesCore
    @eval function ChainRulesCore.rrule(::typeof(conic_layer), c, h, Gval, bl, bu, s::ConicStructure)
        hd = _layer_handle(c, h, Gval, bl, bu, s)
        sols, _ = batch_solve(hd)
        x = sols[1].x.recovered_primal.primal_sol.x
        function conic_layer_pullback(xbar)
            g, infos = batch_grad(hd, [collect(ChainRulesCore.unthunk(xbar))])
            close(hd)
            infos[1].converged == 1 || @warn "adjoint solve did not converge" infos[1]
            nt = ChainRulesCore.NoTangent()
            return (nt, g[1].c, g[1].h, g[1].G, g[1].bl, g[1].bu, nt)
        end
        return x, conic_layer_pullback
    end
end

# ---------------------------------------------------------------------------
# MOI: the reference's wrapper calls PDCS_GPU.rpdhg_gpu_solve(; ...) and reads
# the fields that `solution` above provides.  forward_moi!() rebinds that call
# to this library by evaluating, inside PDCS_GPU, a method that forwards every
# keyword; run it after `using PDCS_GPU`.
# ---------------------------------------------------------------------------
function forward_moi!(pdcs_gpu_module::Module)
    Core.eval(pdcs_gpu_module, :(rpdhg_gpu_solve(; kw...) = $(PDCSB200).rpdhg_gpu_solve(; kw...)))
    return nothing
end

end # module
