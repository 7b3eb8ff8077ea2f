# Julia host binding of libbpf.so: the reference's API (module BlockPowerFlow) on top of the
# C ABI in include/bpf.h.  Same function names, keyword arguments, defaults, stats types and
# error behaviour as src/block_gmres.jl, src/block_bicgstab.jl, src/preconditioners_nvidia.jl
# and src/cusolverRF.jl; the arithmetic runs in the library's sm_100a kernels.
#
# Device pointers come from CUDA.jl arrays; the library works on the CUDA.jl task stream.
# CuSparseMatrixCSR{Float64,Cint} is passed as it is (1-based, index_base = 1).
module BlockPowerFlowB200

using LinearAlgebra
using CUDA
using CUDA.CUSPARSE
using SparseArrays

import LinearAlgebra: ldiv!

export block_gmres, block_bicgstab, ilu0, ic0, CUSOLVERRF, BatchPlan, batch_solve!, BlockJacobiPreconditioner
export householder, householder!
export BlockGMRESSolver, block_gmres!, warm_start!, BlockBicgstabSolver, block_bicgstab!
export PowerFlowAssembly, mismatch!, jacobian!
export WarmStartMLP, set_scale!, warm_start, train_step!, deflation_basis, judged_warm_start, learned_solve

const libbpf = joinpath(@__DIR__, "..", "lib", "libbpf.so")

struct CsrDesc
    n::Cint
    nnz::Cint
    rowptr::CuPtr{Cint}
    colind::CuPtr{Cint}
    vals::CuPtr{Cdouble}
    index_base::Cint
    dtype::Cint
end

struct GmresOpts
    memory::Cint
    restart::Cint
    reorthogonalization::Cint
    ldiv::Cint
    atol::Cdouble
    rtol::Cdouble
    itmax::Cint
    timemax::Cdouble
    verbose::Cint
    history::Cint
end

struct BicgstabOpts
    atol::Cdouble
    rtol::Cdouble
    itmax::Cint
    timemax::Cdouble
    verbose::Cint
    history::Cint
end

mutable struct CStats
    niter::Cint
    solved::Cint
    status::Cint
    timer::Cdouble
    n_residuals::Cint
    residuals_capacity::Cint
    residuals::Ptr{Cdouble}
    npass::Cint
end

# BlockGMRESStats (src/block_utils.jl:62-68) and SimpleStats (src/block_bicgstab.jl:15-21)
mutable struct BlockGMRESStats{T}
    niter::Int
    solved::Bool
    residuals::Vector{T}
    timer::Float64
    status::String
end
mutable struct SimpleStats{T}
    niter::Int
    solved::Bool
    residuals::Vector{T}
    timer::Float64
    status::String
end

const _ctx = Ref{Ptr{Cvoid}}(C_NULL)
function ctx()
    if _ctx[] == C_NULL
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:bpf_ctx_create, libbpf), Cint, (Ref{Ptr{Cvoid}}, Ptr{Cvoid}), r,
                    CUDA.stream().handle))
        _ctx[] = r[]
    end
    ccall((:bpf_ctx_set_stream, libbpf), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), _ctx[], CUDA.stream().handle)
    return _ctx[]
end

function check(st::Cint)
    st == 0 && return nothing
    msg = _ctx[] == C_NULL ? "libbpf status $st" :
          unsafe_string(ccall((:bpf_last_error, libbpf), Cstring, (Ptr{Cvoid},), _ctx[]))
    st == 2 && throw(DimensionMismatch(msg))
    st == 5 && throw(SingularException(0))
    error(msg)
end

desc(A::CuSparseMatrixCSR{Float64,Cint}) =
    CsrDesc(size(A, 1), nnz(A), pointer(A.rowPtr), pointer(A.colVal), pointer(A.nzVal), 1, 0)

status_string(code) = unsafe_string(ccall((:bpf_solve_status_string, libbpf), Cstring, (Cint,), code))

# ---- preconditioners (src/preconditioners_nvidia.jl) -----------------------------------
mutable struct NVIDIA_ILU0
    h::Ptr{Cvoid}
    n::Int
end
mutable struct NVIDIA_IC0
    h::Ptr{Cvoid}
    n::Int
end
const DevicePrec = Union{NVIDIA_ILU0,NVIDIA_IC0}

const PREC_ORDER = Dict(:natural => 4, :AMD => 0, :MDQ => 1, :METIS => 2, :RCM => 3)

function _prec(fn::Symbol, A, nrhs, factor_type, ordering)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    d = Ref(desc(A))
    fd = factor_type === Float32 ? 1 : 0
    if ordering === :natural
        check(ccall((fn, libbpf), Cint, (Ptr{Cvoid}, Ref{CsrDesc}, Cint, Cint, Ref{Ptr{Cvoid}}),
                    ctx(), d, nrhs, fd, r))
    else   # an addition: the reference factors A in its natural order
        check(ccall((Symbol(fn, :_ordered), libbpf), Cint,
                    (Ptr{Cvoid}, Ref{CsrDesc}, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                    ctx(), d, nrhs, fd, PREC_ORDER[ordering], r))
    end
    return r[]
end

function ilu0(A::CuSparseMatrixCSR{Float64,Cint}, nrhs::Int; factor_type=Float64, ordering=:natural)
    P = NVIDIA_ILU0(_prec(:bpf_ilu0_create, A, nrhs, factor_type, ordering), size(A, 1))
    finalizer(p -> ccall((:bpf_prec_destroy, libbpf), Cint, (Ptr{Cvoid},), p.h), P)
    return P
end

function ic0(A::CuSparseMatrixCSR{Float64,Cint}, nrhs::Int; factor_type=Float64, ordering=:natural)
    P = NVIDIA_IC0(_prec(:bpf_ic0_create, A, nrhs, factor_type, ordering), size(A, 1))
    finalizer(p -> ccall((:bpf_prec_destroy, libbpf), Cint, (Ptr{Cvoid},), p.h), P)
    return P
end

# CSC input, which the reference's ilu0 / ic0 accept (src/preconditioners_nvidia.jl:6,42): there
# the factors are those of A^T and are applied transposed.  The incomplete factorization whose
# product matches A on A's pattern is unique, so that is the same preconditioner as the CSR
# form's; the matrix is converted to CSR once (the library keeps no pointer to it).
ilu0(A::CuSparseMatrixCSC{Float64,Cint}, nrhs::Int; kwargs...) = ilu0(CuSparseMatrixCSR(A), nrhs; kwargs...)
ic0(A::CuSparseMatrixCSC{Float64,Cint}, nrhs::Int; kwargs...) = ic0(CuSparseMatrixCSR(A), nrhs; kwargs...)

function ldiv!(y::CuVecOrMat{Float64}, P::DevicePrec, x::CuVecOrMat{Float64})
    p = size(x, 2)
    check(ccall((:bpf_prec_apply, libbpf), Cint,
                (Ptr{Cvoid}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint),
                P.h, p, pointer(x), stride(x, 2), pointer(y), stride(y, 2)))
    return y
end

# ---- block-Jacobi (ExaPF's LS.BlockJacobiPreconditioner as test/block_gmres.jl:5 uses it) ------
mutable struct BlockJacobiPreconditioner
    h::Ptr{Cvoid}
    n::Int
end

function BlockJacobiPreconditioner(A::CuSparseMatrixCSR{Float64,Cint}, nblocks::Int; ordering=:natural)
    n = size(A, 1)
    bs = min(32, cld(n, max(nblocks, 1)))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:bpf_block_jacobi_create, libbpf), Cint,
                (Ptr{Cvoid}, Ref{CsrDesc}, Cint, Cint, Ref{Ptr{Cvoid}}),
                ctx(), Ref(desc(A)), bs, PREC_ORDER[ordering], r))
    P = BlockJacobiPreconditioner(r[], n)
    finalizer(p -> ccall((:bpf_prec_destroy, libbpf), Cint, (Ptr{Cvoid},), p.h), P)
    return P
end

# ExaPF's LS.update(BJ, A, device): the block inverses from A's current values
update(P::BlockJacobiPreconditioner, A::CuSparseMatrixCSR{Float64,Cint}) =
    check(ccall((:bpf_prec_refactor, libbpf), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}), P.h, pointer(A.nzVal)))

# mul!(y, P, x): y = P x
function LinearAlgebra.mul!(y::CuVecOrMat{Float64}, P::BlockJacobiPreconditioner, x::CuVecOrMat{Float64})
    check(ccall((:bpf_prec_apply, libbpf), Cint,
                (Ptr{Cvoid}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint),
                P.h, size(x, 2), pointer(x), stride(x, 2), pointer(y), stride(y, 2)))
    return y
end

# ---- block-GMRES (src/block_gmres.jl:127-154) -----------------------------------------
_handle(::typeof(I)) = C_NULL
_handle(P::DevicePrec) = P.h
_handle(P::BlockJacobiPreconditioner) = P.h

function block_gmres(A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64},
                     X0::Union{Nothing,CuMatrix{Float64}}=nothing; memory::Int=20, M=I, N=I,
                     ldiv::Bool=false, restart::Bool=false, reorthogonalization::Bool=false,
                     atol::Float64=√eps(Float64), rtol::Float64=√eps(Float64), itmax::Int=0,
                     timemax::Float64=Inf, verbose::Int=0, history::Bool=false,
                     deflation::Union{Nothing,CuMatrix{Float64}}=nothing)
    n, p = size(B)
    size(A, 1) == size(A, 2) || error("System must be square")
    size(A, 1) == n || error("Inconsistent problem size")
    X = CuMatrix{Float64}(undef, n, p)
    cap = (itmax == 0 ? 2 * div(n, p) : itmax) + 2
    res = zeros(Float64, cap)
    opts = Ref(GmresOpts(memory, restart, reorthogonalization, ldiv, atol, rtol, itmax,
                         isfinite(timemax) ? timemax : 0.0, verbose, history))
    st = Ref(CStats(0, 0, 0, 0.0, 0, cap, pointer(res), 0))
    x0p = X0 === nothing ? CU_NULL : pointer(X0)
    GC.@preserve res begin
        if deflation === nothing
            check(ccall((:bpf_block_gmres, libbpf), Cint,
                        (Ptr{Cvoid}, Ref{CsrDesc}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint,
                         CuPtr{Cdouble}, Cint, Ptr{Cvoid}, Ptr{Cvoid}, Ref{GmresOpts}, Ref{CStats}),
                        ctx(), Ref(desc(A)), p, pointer(B), stride(B, 2), pointer(X), stride(X, 2),
                        x0p, n, _handle(M), _handle(N), opts, st))
        else   # an addition: GCRO deflation with an n x rank basis (rank <= p)
            size(deflation, 1) == n || error("Inconsistent deflation basis size")
            check(ccall((:bpf_block_gmres_deflated, libbpf), Cint,
                        (Ptr{Cvoid}, Ref{CsrDesc}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint,
                         CuPtr{Cdouble}, Cint, Ptr{Cvoid}, Ptr{Cvoid}, Ref{GmresOpts},
                         CuPtr{Cdouble}, Cint, Cint, Ref{CStats}),
                        ctx(), Ref(desc(A)), p, pointer(B), stride(B, 2), pointer(X), stride(X, 2),
                        x0p, n, _handle(M), _handle(N), opts, pointer(deflation),
                        stride(deflation, 2), size(deflation, 2), st))
        end
    end
    s = st[]
    stats = BlockGMRESStats{Float64}(s.niter, s.solved != 0,
                                     history ? res[1:min(s.n_residuals, cap)] : Float64[],
                                     s.timer, status_string(s.status))
    return X, stats
end

# ---- in-place forms (src/block_gmres.jl:21-168,397-411; src/block_bicgstab.jl:23-55,187-299) -----
# The solver objects hold the solution block, the statistics and (GMRES) the basis size and a
# pending warm start; the Krylov basis and the small blocks live in the library's context.
mutable struct BlockGMRESSolver
    m::Int
    n::Int
    p::Int
    memory::Int
    X::CuMatrix{Float64}
    ΔX::Union{Nothing,CuMatrix{Float64}}
    warm_start::Bool
    stats::BlockGMRESStats{Float64}
end

BlockGMRESSolver(m::Int, n::Int, p::Int, memory::Int) =
    BlockGMRESSolver(m, n, p, min(div(n, p), memory), CuMatrix{Float64}(undef, n, p), nothing, false,
                     BlockGMRESStats{Float64}(0, false, Float64[], 0.0, "unknown"))
BlockGMRESSolver(A, B; memory::Int=5) = BlockGMRESSolver(size(A, 1), size(A, 2), size(B, 2), memory)

function warm_start!(solver::BlockGMRESSolver, X0::CuMatrix{Float64})
    n, p = size(solver.X)
    size(X0) == (n, p) || error("X0 should have size ($n, $p)")
    solver.ΔX = copy(X0)
    solver.warm_start = true
    return solver
end

function block_gmres!(solver::BlockGMRESSolver, A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64},
                      X0::CuMatrix{Float64}; kwargs...)
    warm_start!(solver, X0)
    return block_gmres!(solver, A, B; kwargs...)
end

function block_gmres!(solver::BlockGMRESSolver, A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64};
                      M=I, N=I, ldiv::Bool=false, restart::Bool=false, reorthogonalization::Bool=false,
                      atol::Float64=√eps(Float64), rtol::Float64=√eps(Float64), itmax::Int=0,
                      timemax::Float64=Inf, verbose::Int=0, history::Bool=false)
    size(B) == size(solver.X) || error("Inconsistent problem size")
    X, stats = block_gmres(A, B, solver.warm_start ? solver.ΔX : nothing; memory=solver.memory, M, N, ldiv,
                           restart, reorthogonalization, atol, rtol, itmax, timemax, verbose, history)
    copyto!(solver.X, X)
    solver.stats = stats
    solver.warm_start = false
    solver.ΔX = nothing
    return solver
end

mutable struct BlockBicgstabSolver
    X::CuMatrix{Float64}
    stats::SimpleStats{Float64}
end

BlockBicgstabSolver(A, B) = BlockBicgstabSolver(CuMatrix{Float64}(undef, size(A, 1), size(B, 2)),
                                                SimpleStats{Float64}(0, false, Float64[], 0.0, "unknown"))

function block_bicgstab!(solver::BlockBicgstabSolver, A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64};
                         kwargs...)
    size(B) == size(solver.X) || error("Inconsistent problem size")
    X, stats = block_bicgstab(A, B; kwargs...)
    copyto!(solver.X, X)
    solver.stats = stats
    return (solver.X, solver.stats)
end

# ---- batched block-GMRES (an addition: many systems in one graph launch) ----------------
struct BatchOpts
    atol::Cdouble
    rtol::Cdouble
    itmax::Cint
    memory::Cint
    factor_dtype::Cint
    ordering::Cint
    slice::Cint
    ctas_per_sm::Cint
end

mutable struct BatchPlan
    h::Ptr{Cvoid}
    mats::Vector{CuSparseMatrixCSR{Float64,Cint}}   # kept alive: their values are re-read per solve
    nrhs::Vector{Int}
end

# slices: optional widest column slice per system (0: `slice`), as the autotuner's refinement
# narrows the systems on the critical path (bpf_batch_plan_sliced)
function BatchPlan(As::Vector{CuSparseMatrixCSR{Float64,Cint}}, nrhs::Vector{Int}; atol=0.0, rtol=1e-8,
                   itmax=0, memory=0, factor_type=Float32, ordering=:AMD, slice=0, ctas_per_sm=0,
                   slices::Union{Nothing,Vector{Int}}=nothing)
    length(As) == length(nrhs) || throw(DimensionMismatch("one nrhs per system expected"))
    slices === nothing || length(slices) == length(As) ||
        throw(DimensionMismatch("one slice width per system expected"))
    descs = [desc(A) for A in As]
    opts = Ref(BatchOpts(atol, rtol, itmax, memory, factor_type === Float32 ? 1 : 0,
                         PREC_ORDER[ordering], slice, ctas_per_sm))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    if slices === nothing
        check(ccall((:bpf_batch_plan, libbpf), Cint,
                    (Ptr{Cvoid}, Cint, Ptr{CsrDesc}, Ptr{Cint}, Ref{BatchOpts}, Ref{Ptr{Cvoid}}),
                    ctx(), length(As), descs, Cint.(nrhs), opts, r))
    else
        check(ccall((:bpf_batch_plan_sliced, libbpf), Cint,
                    (Ptr{Cvoid}, Cint, Ptr{CsrDesc}, Ptr{Cint}, Ptr{Cint}, Ref{BatchOpts}, Ref{Ptr{Cvoid}}),
                    ctx(), length(As), descs, Cint.(nrhs), Cint.(slices), opts, r))
    end
    P = BatchPlan(r[], As, nrhs)
    finalizer(p -> ccall((:bpf_batch_destroy, libbpf), Cint, (Ptr{Cvoid},), p.h), P)
    return P
end

# Xs[s] = As[s] \ Bs[s] for every system; returns per-system (niter, solved, status).
function batch_solve!(Xs::Vector{CuMatrix{Float64}}, P::BatchPlan, Bs::Vector{CuMatrix{Float64}})
    ns = length(P.nrhs)
    length(Bs) == ns == length(Xs) || throw(DimensionMismatch("one block per system expected"))
    buf = Vector{UInt8}(undef, ns * sizeof(CStats))
    check(ccall((:bpf_batch_solve, libbpf), Cint,
                (Ptr{Cvoid}, Ptr{CuPtr{Cdouble}}, Ptr{Cint}, Ptr{CuPtr{Cdouble}}, Ptr{Cint}, Ptr{UInt8}),
                P.h, [pointer(B) for B in Bs], Cint[stride(B, 2) for B in Bs],
                [pointer(X) for X in Xs], Cint[stride(X, 2) for X in Xs], buf))
    stats = [unsafe_load(Ptr{CStats}(pointer(buf)) + (s - 1) * sizeof(CStats)) for s in 1:ns]
    return [(niter=Int(c.niter), solved=c.solved != 0, status=status_string(c.status)) for c in stats]
end

# ---- power-flow assembly (an addition: the Newton loop's F, Gx, Gu on the device) -------
# Unknowns x = [theta(non-slack); |V|(PQ)], equations [P(non-slack); Q(PQ)], controls |V| of the
# slack then the PV buses, all in bus order; bus_type: 1 PQ, 2 PV, 3 slack (exactly one).
mutable struct PowerFlowAssembly
    h::Ptr{Cvoid}
    Gx::CuSparseMatrixCSR{Float64,Cint}
    n::Int
    nctrl::Int
end

function PowerFlowAssembly(Ybus::SparseMatrixCSC{ComplexF64}, bus_type::Vector{<:Integer},
                           vm::Vector{Float64}, va::Vector{Float64}, Sspec::Vector{ComplexF64},
                           Gx::CuSparseMatrixCSR{Float64,Cint})
    nb = size(Ybus, 1)
    Yt = SparseMatrixCSC(transpose(Ybus))          # CSC of the transpose = CSR of Ybus
    rowptr = Cint.(Yt.colptr .- 1)
    colind = Cint.(Yt.rowval .- 1)
    vals = reinterpret(Float64, Yt.nzval) |> collect   # (re, im) interleaved
    s = reinterpret(Float64, Sspec) |> collect
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:bpf_pf_create, libbpf), Cint,
                (Ptr{Cvoid}, Cint, Ptr{Cint}, Ptr{Cint}, Ptr{Cdouble}, Ptr{Cint}, Ptr{Cdouble},
                 Ptr{Cdouble}, Ptr{Cdouble}, Ref{CsrDesc}, Ref{Ptr{Cvoid}}),
                ctx(), nb, rowptr, colind, vals, Cint.(bus_type), vm, va, s, Ref(desc(Gx)), r))
    n, nc = Ref{Cint}(0), Ref{Cint}(0)
    check(ccall((:bpf_pf_info, libbpf), Cint, (Ptr{Cvoid}, Ref{Cint}, Ref{Cint}, Ptr{Cint}),
                r[], n, nc, C_NULL))
    PF = PowerFlowAssembly(r[], Gx, n[], nc[])
    finalizer(p -> ccall((:bpf_pf_destroy, libbpf), Cint, (Ptr{Cvoid},), p.h), PF)
    return PF
end

# F = F(x + alpha dx) (dx nothing -> at x); xout (optional, may be x) receives that point.
function mismatch!(F::CuVector{Float64}, PF::PowerFlowAssembly, x::CuVector{Float64},
                   dx::Union{Nothing,CuVector{Float64}}=nothing, alpha::Float64=0.0,
                   xout::Union{Nothing,CuVector{Float64}}=nothing)
    length(x) == length(F) == PF.n || throw(DimensionMismatch("x and F need $(PF.n) entries"))
    nrm = Ref{Cdouble}(0.0)
    check(ccall((:bpf_pf_mismatch, libbpf), Cint,
                (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cdouble, CuPtr{Cdouble}, CuPtr{Cdouble}, Ref{Cdouble}),
                PF.h, pointer(x), dx === nothing ? CU_NULL : pointer(dx), alpha,
                xout === nothing ? CU_NULL : pointer(xout), pointer(F), nrm))
    return nrm[]
end

# Gx values at x into PF.Gx (refactor it next); Gu (n x nctrl), if given, = dF/du.
function jacobian!(PF::PowerFlowAssembly, x::CuVector{Float64}, Gu::Union{Nothing,CuMatrix{Float64}}=nothing)
    Gu === nothing || size(Gu) == (PF.n, PF.nctrl) || throw(DimensionMismatch("Gu must be $(PF.n) x $(PF.nctrl)"))
    check(ccall((:bpf_pf_jacobian, libbpf), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, CuPtr{Cdouble}, CuPtr{Cdouble}, Cint),
                PF.h, pointer(x), pointer(nonzeros(PF.Gx)), Gu === nothing ? CU_NULL : pointer(Gu),
                Gu === nothing ? 0 : stride(Gu, 2)))
    return PF.Gx
end

# ---- learned warm start and deflation basis (an addition) ----------------------------------
# A 3-layer MLP (n -> hidden -> hidden -> n, BF16 weights, tensor-core products, Adam) trained on
# the solver's own (b, x) pairs; block-GMRES runs from its judged warm start with its deflation
# basis, to the requested residual whatever the network predicts.
mutable struct WarmStartMLP
    h::Ptr{Cvoid}
    n::Int
end

function WarmStartMLP(n::Int; hidden::Int=512, seed::Integer=0)
    hidden % 128 == 0 || throw(ArgumentError("hidden must be a multiple of 128"))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:bpf_mlp_create, libbpf), Cint, (Ptr{Cvoid}, Cint, Cint, Culonglong, Ref{Ptr{Cvoid}}),
                ctx(), n, hidden, seed, r))
    M = WarmStartMLP(r[], n)
    finalizer(m -> ccall((:bpf_mlp_destroy, libbpf), Cint, (Ptr{Cvoid},), m.h), M)
    return M
end

# the output scale: the training set's typical ||x|| / ||b||
set_scale!(M::WarmStartMLP, s::Real) =
    check(ccall((:bpf_mlp_set_scale, libbpf), Cint, (Ptr{Cvoid}, Cdouble), M.h, s))

function warm_start(M::WarmStartMLP, B::CuMatrix{Float64})
    size(B, 1) == M.n || throw(DimensionMismatch("B has $(size(B, 1)) rows, the network $(M.n)"))
    X = CuMatrix{Float64}(undef, size(B)...)
    check(ccall((:bpf_mlp_forward, libbpf), Cint,
                (Ptr{Cvoid}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint),
                M.h, size(B, 2), pointer(B), stride(B, 2), pointer(X), stride(X, 2)))
    return X
end

# one Adam step on the pairs (B, X), at most 128 columns; returns the batch loss
function train_step!(M::WarmStartMLP, B::CuMatrix{Float64}, X::CuMatrix{Float64}; lr::Float64=2e-4)
    size(B) == size(X) || throw(DimensionMismatch("B and X differ in size"))
    loss = Ref{Cdouble}(0.0)
    check(ccall((:bpf_mlp_train_step, libbpf), Cint,
                (Ptr{Cvoid}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint, Cdouble, Ref{Cdouble}),
                M.h, size(B, 2), pointer(B), stride(B, 2), pointer(X), stride(X, 2), lr, loss))
    return loss[]
end

# orthonormal n x rank basis of the network's outputs on Gaussian probes
function deflation_basis(M::WarmStartMLP, rank::Int; seed::Integer=0)
    Z = CuMatrix{Float64}(undef, M.n, rank)
    check(ccall((:bpf_mlp_basis, libbpf), Cint, (Ptr{Cvoid}, Cint, Culonglong, CuPtr{Cdouble}, Cint),
                M.h, rank, seed, pointer(Z), stride(Z, 2)))
    return Z
end

# The network's warm start if it beats the zero start, else nothing.  Without N: the residual,
# ||B - A X0|| < ||B||.  With the right preconditioner N: the estimated error,
# ||N \ (B - A X0)|| < ||N \ B|| (the network's misses are short-wavelength components that A
# amplifies in the residual and the preconditioner removes).
function judged_warm_start(M::WarmStartMLP, A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64}, N=nothing)
    X0 = warm_start(M, B)
    R = copy(B)
    check(ccall((:bpf_spmm, libbpf), Cint,
                (Ptr{Cvoid}, Ref{CsrDesc}, Cint, Cdouble, CuPtr{Cdouble}, Cint, Cdouble, CuPtr{Cdouble}, Cint),
                ctx(), Ref(desc(A)), size(X0, 2), -1.0, pointer(X0), stride(X0, 2), 1.0, pointer(R), stride(R, 2)))
    N === nothing && return norm(R) < norm(B) ? X0 : nothing
    E = similar(B)
    ldiv!(E, N, R)
    e0 = norm(E)
    ldiv!(E, N, B)
    return e0 < norm(E) ? X0 : nothing
end

# right-preconditioned block-GMRES from the judged warm start, with the deflation basis Z if given;
# tolerance rtol ||B||_F whatever the start; if it does not reach it within itmax, the plain solve
# from the zero start runs instead (the network can cost iterations, never accuracy)
function learned_solve(A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64}, N, M::WarmStartMLP;
                       Z::Union{Nothing,CuMatrix{Float64}}=nothing, rtol::Float64=1e-8, itmax::Int=300)
    X0 = judged_warm_start(M, A, B, N)
    X, st = block_gmres(A, B, X0; N=N, ldiv=true, restart=false, memory=itmax, atol=rtol * norm(B),
                        rtol=0.0, itmax=itmax, deflation=Z)
    (st.solved || (X0 === nothing && Z === nothing)) && return X, st
    return block_gmres(A, B; N=N, ldiv=true, restart=false, memory=itmax, atol=rtol * norm(B),
                       rtol=0.0, itmax=itmax)
end

# ---- householder (src/block_utils.jl:38-53) ----------------------------------------------
# Reduced QR of an n x k device block with LAPACK's conventions: R (k x k) has geqrf's signs,
# tau (k) the reflectors' scalars, and Q is overwritten by orgqr's orthonormal factor, or with
# compact = true by geqrf's compact form (R on and above the diagonal, the reflector vectors below).
function householder!(Q::CuMatrix{Float64}, R::CuMatrix{Float64},
                      tau::CuVector{Float64}=CuVector{Float64}(undef, size(Q, 2)); compact::Bool=false)
    n, k = size(Q)
    n >= k || throw(DimensionMismatch("householder needs n >= k"))
    size(R) == (k, k) || throw(DimensionMismatch("R must be $k x $k"))
    length(tau) >= k || throw(DimensionMismatch("tau must hold $k values"))
    fill!(R, 0.0)
    check(ccall((:bpf_householder_lapack, libbpf), Cint,
                (Ptr{Cvoid}, Cint, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint),
                ctx(), n, k, pointer(Q), stride(Q, 2), pointer(R), stride(R, 2), pointer(tau), Cint(compact)))
    return Q, R
end

householder(A::CuMatrix{Float64}; compact::Bool=false) =
    householder!(copy(A), CuMatrix{Float64}(undef, size(A, 2), size(A, 2)); compact)

# ---- block-BiCGSTAB (src/block_bicgstab.jl:182-299) -----------------------------------
function block_bicgstab(A::CuSparseMatrixCSR{Float64,Cint}, B::CuMatrix{Float64};
                        C::Union{Nothing,CuMatrix{Float64}}=nothing, N=I,
                        atol::Float64=√eps(Float64), rtol::Float64=√eps(Float64), itmax::Int=0,
                        timemax::Float64=Inf, verbose::Int=0, history::Bool=false)
    n, p = size(B)
    size(A, 1) == size(A, 2) || error("System must be square")
    size(A, 1) == n || error("Inconsistent problem size")
    X = CuMatrix{Float64}(undef, n, p)
    cap = (itmax == 0 ? 2n : itmax) + 2
    res = zeros(Float64, cap)
    opts = Ref(BicgstabOpts(atol, rtol, itmax, isfinite(timemax) ? timemax : 0.0, verbose, history))
    st = Ref(CStats(0, 0, 0, 0.0, 0, cap, pointer(res), 0))
    cp = C === nothing ? CU_NULL : pointer(C)
    GC.@preserve res begin
        check(ccall((:bpf_block_bicgstab, libbpf), Cint,
                    (Ptr{Cvoid}, Ref{CsrDesc}, Cint, CuPtr{Cdouble}, Cint, CuPtr{Cdouble}, Cint,
                     CuPtr{Cdouble}, Cint, Ptr{Cvoid}, Ref{BicgstabOpts}, Ref{CStats}),
                    ctx(), Ref(desc(A)), p, pointer(B), stride(B, 2), pointer(X), stride(X, 2),
                    cp, n, _handle(N), opts, st))
    end
    s = st[]
    return X, SimpleStats{Float64}(s.niter, s.solved != 0,
                                   history ? res[1:min(s.n_residuals, cap)] : Float64[],
                                   s.timer, status_string(s.status))
end

# ---- CUSOLVERRF (src/cusolverRF.jl) ----------------------------------------------------
module CUSOLVERRF
using CUDA, CUDA.CUSPARSE, LinearAlgebra
import ..BlockPowerFlowB200: libbpf, ctx, check, desc, CsrDesc

const ORDER = Dict(:AMD => 0, :MDQ => 1, :METIS => 2, :RCM => 3)

abstract type CusolverFactorization{T} <: LinearAlgebra.Factorization{T} end
mutable struct CusolverRfLU{T} <: CusolverFactorization{T}
    h::Ptr{Cvoid}
    n::Int
end
mutable struct CusolverRfLUBatch{T} <: CusolverFactorization{T}
    h::Ptr{Cvoid}
    batchsize::Int
    n::Int
end

function _analyze(A, ordering, tol, fast_mode, batch)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:bpf_rf_analyze, libbpf), Cint,
                (Ptr{Cvoid}, Ref{CsrDesc}, Cint, Cdouble, Cint, Cint, Ref{Ptr{Cvoid}}),
                ctx(), Ref(desc(A)), ORDER[ordering], tol, fast_mode, batch, r))
    return r[]
end

function CusolverRfLU(A::CuSparseMatrixCSR{T}; nrhs=1, ordering=:AMD, tol=1e-8, fast_mode=true) where T
    @assert size(A, 1) == size(A, 2)
    return CusolverRfLU{T}(_analyze(A, ordering, tol, fast_mode, 1), size(A, 1))
end

function CusolverRfLUBatch(A::CuSparseMatrixCSR{T}, batchsize::Int; ordering=:AMD, tol=1e-8,
                           fast_mode=false) where T
    @assert size(A, 1) == size(A, 2)
    batchsize == 1 && error("Please specify a number of batch greater than 1 for `CuSolverRfLUBatch`")
    return CusolverRfLUBatch{T}(_analyze(A, ordering, tol, fast_mode, batchsize), batchsize, size(A, 1))
end

update!(rflu::CusolverFactorization, A::CuSparseMatrixCSR) =
    check(ccall((:bpf_rf_refactor, libbpf), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}), rflu.h, pointer(A.nzVal)))

rf_batch_refactor!(rflu::CusolverRfLUBatch, Anzval::CuMatrix{Float64}) =
    check(ccall((:bpf_rf_refactor_batch, libbpf), Cint, (Ptr{Cvoid}, CuPtr{Cdouble}, Cint),
                rflu.h, pointer(Anzval), stride(Anzval, 2)))

function LinearAlgebra.ldiv!(rflu::CusolverFactorization, X::CuVecOrMat{Float64})
    check(ccall((:bpf_rf_solve, libbpf), Cint, (Ptr{Cvoid}, Cint, CuPtr{Cdouble}, Cint),
                rflu.h, size(X, 2), pointer(X), stride(X, 2)))
    return X
end
function LinearAlgebra.ldiv!(x::CuVecOrMat{Float64}, rflu::CusolverFactorization, b::CuVecOrMat{Float64})
    copyto!(x, b)
    return ldiv!(rflu, x)
end
function solve!(x::Vector{<:CuVector{Float64}}, rflu::CusolverRfLUBatch, b::Vector{<:CuVector{Float64}})
    X = reduce(hcat, b)
    ldiv!(rflu, X)
    for i in eachindex(x)
        copyto!(x[i], view(X, :, i))
    end
end

LinearAlgebra.lu(A::CuSparseMatrixCSR; options...) = CusolverRfLU(A; options...)
LinearAlgebra.lu!(rflu::CusolverFactorization, A::CuSparseMatrixCSR) = update!(rflu, A)
cudestroy!(rflu::CusolverFactorization) =
    (rflu.h != C_NULL && ccall((:bpf_rf_destroy, libbpf), Cint, (Ptr{Cvoid},), rflu.h); rflu.h = C_NULL)
end # module CUSOLVERRF

end # module
