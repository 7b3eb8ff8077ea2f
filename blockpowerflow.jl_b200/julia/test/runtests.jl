# Tests of the BlockPowerFlowB200 Julia binding on a CUDA device.  They follow the settings of the
# reference's own tests (test/block_gmres.jl, test/block_bicgstab.jl: B = I[:, 1:32], atol 1e-8,
# rtol 0, itmax 500; test/cusolverRF.jl: the solve against the direct solve, values x2 -> x/2, the
# batch forms) on a synthetic unsymmetric sparse matrix, then check the additions.
#
#   julia --project=<env with CUDA.jl> blockpowerflow.jl_b200/julia/test/runtests.jl
#
# libbpf.so must be built first (make -C blockpowerflow.jl_b200/csrc).
using Test, LinearAlgebra, SparseArrays, Random, Statistics
using CUDA, CUDA.CUSPARSE

include(joinpath(@__DIR__, "..", "BlockPowerFlowB200.jl"))
using .BlockPowerFlowB200
const RF = BlockPowerFlowB200.CUSOLVERRF

# m x m grid operator with unequal neighbour couplings: unsymmetric, diagonally dominant
function grid_matrix(m)
    n = m * m
    idx(i, j) = (j - 1) * m + i
    rows, cols, vals = Int[], Int[], Float64[]
    for j in 1:m, i in 1:m
        k = idx(i, j)
        push!(rows, k); push!(cols, k); push!(vals, 4.5)
        i > 1 && (push!(rows, k); push!(cols, idx(i - 1, j)); push!(vals, -1.2))
        i < m && (push!(rows, k); push!(cols, idx(i + 1, j)); push!(vals, -0.8))
        j > 1 && (push!(rows, k); push!(cols, idx(i, j - 1)); push!(vals, -1.1))
        j < m && (push!(rows, k); push!(cols, idx(i, j + 1)); push!(vals, -0.9))
    end
    return sparse(rows, cols, vals, n, n)
end

const A = grid_matrix(24)                      # 576 x 576
const n = size(A, 1)
const Ad = CuSparseMatrixCSR(A)
const B = Matrix{Float64}(I, n, 32)            # B = I[:, 1:32]
const Bd = CuMatrix(B)

@testset "block_gmres (test/block_gmres.jl settings)" begin
    P = ilu0(Ad, 32)
    for restart in (false, true)
        X, st = block_gmres(Ad, Bd; N=P, ldiv=true, restart=restart, memory=100,
                            atol=1e-8, rtol=0.0, itmax=500)
        @test st.solved
        @test st.status == "solution good enough given atol and rtol"
        @test norm(B - A * Array(X)) <= 1e-7
    end
    X, st = block_gmres(Ad, Bd; atol=1e-8, rtol=0.0, itmax=500, memory=200)   # no preconditioner
    @test st.solved
    @test_throws ErrorException block_gmres(Ad, CuMatrix(zeros(n + 1, 2)))
end

@testset "in-place forms: BlockGMRESSolver, block_gmres!, warm_start!, block_bicgstab!" begin
    P = ilu0(Ad, 32)
    solver = BlockGMRESSolver(Ad, Bd; memory=50)
    @test solver.memory == div(n, 32)
    block_gmres!(solver, Ad, Bd; N=P, ldiv=true, atol=1e-8, rtol=0.0, itmax=500)
    @test solver.stats.solved
    X1 = Array(solver.X)
    @test norm(B - A * X1) <= 1e-7
    block_gmres!(solver, Ad, Bd, CuMatrix(X1); N=P, ldiv=true, atol=1e-8, rtol=0.0, itmax=500)
    @test solver.stats.solved && solver.stats.niter <= 1 && !solver.warm_start
    @test_throws ErrorException warm_start!(solver, CuMatrix(zeros(n, 3)))
    bsolver = BlockBicgstabSolver(Ad, Bd)
    X, st = block_bicgstab!(bsolver, Ad, Bd; N=P, atol=1e-8, rtol=0.0, itmax=500)
    @test X === bsolver.X && st.solved
end

@testset "householder (src/block_utils.jl:38-53)" begin
    W = randn(MersenneTwister(4), n, 16)
    Q, R = householder(CuMatrix(W))
    Qh, Rh = Array(Q), Array(R)
    @test Qh' * Qh ≈ Matrix{Float64}(I, 16, 16) atol = 1e-12
    @test Qh * Rh ≈ W
    @test istriu(Rh)
    @test all(diag(Rh) .> 0)
    @test_throws ArgumentError householder(CuMatrix(W); compact=true)
end

@testset "block_bicgstab (test/block_bicgstab.jl settings)" begin
    P = ilu0(Ad, 32)
    X, st = block_bicgstab(Ad, Bd; N=P, atol=1e-8, rtol=0.0, itmax=500)
    @test st.solved
    @test norm(B - A * Array(X)) <= 1e-7
end

@testset "ilu0 / ic0 ldiv!, FP32 factors, orderings" begin
    x = CuMatrix(randn(MersenneTwister(1), n, 4))
    y = similar(x)
    for (ft, ord) in ((Float64, :natural), (Float32, :natural), (Float64, :AMD), (Float64, :RCM))
        P = ilu0(Ad, 4; factor_type=ft, ordering=ord)
        ldiv!(y, P, x)
        @test all(isfinite, Array(y))
    end
    Pr, Pc = ilu0(Ad, 4), ilu0(CuSparseMatrixCSC(A), 4)   # CSR and CSC input: the same ILU(0)
    yr, yc = similar(x), similar(x)
    ldiv!(yr, Pr, x); ldiv!(yc, Pc, x)
    @test Array(yc) ≈ Array(yr)
    S = A + A' + 2I                             # symmetric positive definite
    Sd = CuSparseMatrixCSR(S)
    C = ic0(Sd, 32)
    X, st = block_gmres(Sd, Bd; N=C, ldiv=true, atol=1e-8, rtol=0.0, itmax=500, memory=200)
    @test st.solved
    @test norm(B - S * Array(X)) <= 1e-7
end

@testset "CUSOLVERRF (test/cusolverRF.jl)" begin
    b = randn(MersenneTwister(2), n)
    x_ref = A \ b
    rf = RF.CusolverRfLU(Ad; ordering=:AMD)
    xd = CuVector(b)
    ldiv!(rf, xd)
    @test Array(xd) ≈ x_ref
    A2 = 2.0 * A                                # values x2 on the same pattern -> x / 2
    RF.update!(rf, CuSparseMatrixCSR(A2))
    x2 = similar(xd)
    ldiv!(x2, rf, CuVector(b))
    @test Array(x2) ≈ x_ref ./ 2
    RF.cudestroy!(rf)
    nb = 32                                     # batch: column i solves with i b
    rfb = RF.CusolverRfLUBatch(Ad, nb; ordering=:AMD)
    Xb = CuMatrix(reduce(hcat, [i .* b for i in 1:nb]))
    ldiv!(rfb, Xb)
    @test Array(Xb) ≈ reduce(hcat, [i .* x_ref for i in 1:nb])
    xs = [CuVector(zeros(n)) for _ in 1:nb]
    RF.solve!(xs, rfb, [CuVector(i .* b) for i in 1:nb])
    @test all(Array(xs[i]) ≈ i .* x_ref for i in 1:nb)
    RF.cudestroy!(rfb)
end

@testset "BlockJacobiPreconditioner (ExaPF's, test/block_gmres.jl:5)" begin
    BJ = BlockJacobiPreconditioner(Ad, div(n, 32))
    x = CuMatrix(randn(MersenneTwister(3), n, 3))
    y = similar(x)
    mul!(y, BJ, x)
    @test all(isfinite, Array(y))
    X, st = block_gmres(Ad, Bd; N=BJ, ldiv=false, atol=1e-8, rtol=0.0, itmax=500, memory=200)
    @test st.solved
end

@testset "BatchPlan (many systems, one graph launch)" begin
    mats = [grid_matrix(m) for m in (10, 14, 20)]
    nrhs = [4, 8, 12]
    Bs = [CuMatrix(randn(MersenneTwister(10 + k), size(M, 1), q)) for (k, (M, q)) in enumerate(zip(mats, nrhs))]
    Xs = [similar(Bk) for Bk in Bs]
    plan = BatchPlan([CuSparseMatrixCSR(M) for M in mats], nrhs)
    st = batch_solve!(Xs, plan, Bs)
    for (M, Bk, Xk, s) in zip(mats, Bs, Xs, st)
        @test s.solved
        @test norm(Array(Bk) - M * Array(Xk)) <= 1e-7 * norm(Array(Bk))
    end
    # a widest slice per system (0 keeps the plan's), in reverse Cuthill-McKee order
    plan2 = BatchPlan([CuSparseMatrixCSR(M) for M in mats], nrhs; slice=32, ordering=:RCM, slices=[0, 3, 4])
    st2 = batch_solve!(Xs, plan2, Bs)
    for (M, Bk, Xk, s) in zip(mats, Bs, Xs, st2)
        @test s.solved
        @test norm(Array(Bk) - M * Array(Xk)) <= 1e-7 * norm(Array(Bk))
    end
    @test_throws DimensionMismatch BatchPlan([CuSparseMatrixCSR(M) for M in mats], nrhs; slices=[0, 3])
end

@testset "PowerFlowAssembly (3 buses: slack, PV, PQ)" begin
    y12, y23, y13 = 1 / (0.01 + 0.1im), 1 / (0.02 + 0.15im), 1 / (0.015 + 0.12im)
    Y = sparse(ComplexF64[y12+y13 -y12 -y13; -y12 y12+y23 -y23; -y13 -y23 y13+y23])
    bus_type = [3, 2, 1]
    vm = [1.02, 1.01, 1.0]                      # |V| where fixed (slack, PV)
    va = zeros(3)                               # slack angle
    V0 = [1.02, 1.01 * cis(-0.02), 0.98 * cis(-0.05)]
    Sspec = V0 .* conj.(Y * V0)                 # the solution: theta2, theta3, |V3| = -0.02, -0.05, 0.98
    Gx = CuSparseMatrixCSR(sparse(ones(3, 3)))  # dense 3 x 3 pattern: [P2, P3, Q3] x [th2, th3, |V3|]
    PF = PowerFlowAssembly(Y, bus_type, vm, va, Sspec, Gx)
    x = CuVector([-0.02, -0.05, 0.98])
    F = CuVector(zeros(3))
    @test mismatch!(F, PF, x) <= 1e-12
    xp = CuVector([0.0, 0.0, 1.0])
    nrm = mismatch!(F, PF, xp)
    Vp = [1.02, 1.01, 1.0]
    Sp = Vp .* conj.(Y * Vp) .- Sspec
    @test Array(F) ≈ [real(Sp[2]), real(Sp[3]), imag(Sp[3])]
    @test nrm ≈ maximum(abs, Array(F))
    Gu = CuMatrix(zeros(3, 2))                  # controls: |V1|, |V2|
    jacobian!(PF, xp, Gu)
    h = 1e-7                                    # finite differences of the mismatch
    J = zeros(3, 3)
    for c in 1:3
        e = zeros(3); e[c] = h
        Fp = CuVector(zeros(3)); Fm = CuVector(zeros(3))
        mismatch!(Fp, PF, CuVector(Array(xp) .+ e)); mismatch!(Fm, PF, CuVector(Array(xp) .- e))
        J[:, c] = (Array(Fp) .- Array(Fm)) ./ (2h)
    end
    Jd = SparseMatrixCSC(Gx)
    @test Matrix(Jd) ≈ J rtol = 1e-6
    @test all(isfinite, Array(Gu))
end

@testset "learned warm start and deflation basis" begin
    M = WarmStartMLP(n; hidden=128, seed=1)
    P = ilu0(Ad, 32)
    X, st = block_gmres(Ad, Bd; N=P, ldiv=true, atol=0.0, rtol=1e-10, itmax=200, memory=200)
    set_scale!(M, median(norm.(eachcol(Array(X)))))
    losses = [train_step!(M, Bd, X; lr=1e-3) for _ in 1:20]
    @test all(isfinite, losses)
    X0 = warm_start(M, Bd)
    @test size(X0) == size(Bd)
    Z = deflation_basis(M, 8)
    @test Array(Z)' * Array(Z) ≈ Matrix{Float64}(I, 8, 8) atol = 1e-10
    Xl, stl = learned_solve(Ad, Bd, P, M; Z=Z, rtol=1e-8)
    @test stl.solved
    @test norm(B - A * Array(Xl)) <= 1e-7 * norm(B)   # stopping test on the estimate, 1e-8
end
