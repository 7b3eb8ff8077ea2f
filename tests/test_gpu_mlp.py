"""The learned warm start's building block: the tcgen05 BF16 GEMM (TMEM accumulator), through
the C ABI, against torch's FP32 product of the same BF16 operands.

Tolerance: the BF16 products are exact in FP32; only the FP32 summation order differs, so the
results agree to ~K x 2^-24 relative; 1e-4 relative to the output scale is used.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _gemm(bpf, A, B, D=None, accumulate=False, splits=0):
    import torch

    M, K = A.shape
    N = B.shape[0]
    if D is None:
        D = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    lib = bpf._lib.load()
    ctx = bpf._lib.context(0)
    bpf._lib.check(lib.bpf_tc_gemm_bf16(ctx, M, N, K, A.data_ptr(), A.stride(0), B.data_ptr(),
                                        B.stride(0), D.data_ptr(), D.stride(0), int(accumulate),
                                        splits), ctx)
    torch.cuda.synchronize()
    return D


@pytest.mark.parametrize("M,N,K,splits", [(128, 128, 64, 1), (256, 384, 512, 1), (300, 200, 640, 1),
                                          (128, 128, 4096, 8), (512, 128, 8192, 0), (130, 8, 128, 0)])
def test_tc_gemm_matches_fp32_product(bpf, M, N, K, splits):
    import torch

    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    D = _gemm(bpf, A, B, splits=splits)
    ref = A.float() @ B.float().t()
    err = (D - ref).abs().max().item() / ref.abs().max().item()
    assert err <= 1e-4, err


def test_tc_gemm_accumulates(bpf):
    import torch

    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn((256, 256), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((128, 256), generator=g, device="cuda").to(torch.bfloat16)
    D0 = torch.randn((256, 128), generator=g, device="cuda")
    D = _gemm(bpf, A, B, D=D0.clone(), accumulate=True)
    ref = D0 + A.float() @ B.float().t()
    assert (D - ref).abs().max().item() <= 1e-4 * ref.abs().max().item()


def test_tc_gemm_rejects_unaligned_k(bpf):
    import torch

    A = torch.zeros((128, 96), dtype=torch.bfloat16, device="cuda")
    B = torch.zeros((128, 96), dtype=torch.bfloat16, device="cuda")
    D = torch.zeros((128, 128), dtype=torch.float32, device="cuda")
    lib = bpf._lib.load()
    ctx = bpf._lib.context(0)
    st = lib.bpf_tc_gemm_bf16(ctx, 128, 128, 96, A.data_ptr(), 96, B.data_ptr(), 96, D.data_ptr(), 128, 0, 1)
    assert st == bpf._lib.BPF_ERR_INVALID_VALUE


# ---- the network: gradients and forward against the CPU oracle ------------------------------
def _params(mlp):
    from blockpowerflow_b200.learned import PARAMS

    out = {}
    for k in PARAMS:
        v = mlp.param(k).cpu().numpy()
        out[k] = v.reshape(-1) if k.startswith("b") else v
    return out


def test_mlp_gradients_and_forward_match_oracle(bpf):
    import torch

    import mlp_oracle as MO
    from blockpowerflow_b200.learned import PARAMS, WarmStartMLP

    n, p, H, s = 530, 8, 256, 0.05
    mlp = WarmStartMLP(n, hidden=H, seed=1)
    mlp.set_scale(s)
    rng = np.random.default_rng(4)
    # perturb the (zero) biases so that every term of the gradient is exercised
    for k, shape in (("b1", (1, H)), ("b2", (1, H))):
        mlp.set_param(k, torch.as_tensor(0.1 * rng.standard_normal(shape), dtype=torch.float32))
    b3 = np.zeros((1, 640))
    b3[0, :n] = 0.05 * rng.standard_normal(n)
    mlp.set_param("b3", torch.as_tensor(b3, dtype=torch.float32))
    B = rng.standard_normal((n, p))
    X = s * np.linalg.norm(B, axis=0) * rng.standard_normal((n, p)) / np.sqrt(n)
    Bd = bpf.colmajor(torch.as_tensor(B, device="cuda"))
    Xd = bpf.colmajor(torch.as_tensor(X, device="cuda"))
    loss = mlp.gradients(Bd, Xd)
    params = _params(mlp)
    loss_o, g_o = MO.forward_backward(params, B, X, s)
    assert abs(loss - loss_o) <= 1e-5 * abs(loss_o)
    for k in PARAMS:
        g = mlp.param(k, grad=True).cpu().numpy().reshape(g_o[k].shape)
        err = np.linalg.norm(g - g_o[k]) / np.linalg.norm(g_o[k])
        assert err <= 1e-3, (k, err)
    X0 = mlp.forward(Bd).cpu().numpy()
    X0o = MO.forward(params, B, s)
    assert np.linalg.norm(X0 - X0o) / np.linalg.norm(X0o) <= 1e-3


def test_mlp_training_reduces_the_loss(bpf):
    from blockpowerflow_b200 import learned

    gr = bpf.grid.make_grid(300, 68, seed=0)
    J = bpf.grid.jacobian(gr)
    N = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(J), 32)
    pairs, scale = learned.solver_pairs(gr, J, N, blocks=6, p=32, seed=0)
    assert len(pairs) == 6 and scale > 0
    mlp = learned.WarmStartMLP(J.shape[0], hidden=256, seed=0)
    mlp.set_scale(scale)
    hist = learned.train(mlp, pairs, epochs=30, lr=2e-3, batch=32)
    assert hist[-1] < 0.5 * hist[0], hist


def test_learned_warm_start_gain_and_judge(bpf):
    """What the trained network gains over the method without it, on the 300-bus grid (530
    unknowns, trained on 2,048 solver-generated solves at perturbed operating points): its warm
    start is far closer to the solution than the zero start (relative error < 0.5 where the zero
    start has 1), yet its residual is not smaller (A amplifies the error components the network
    misses), so with Gaussian right-hand sides it saves no iteration; the judge (the residual test
    of learned.judged_warm_start) keeps the solve from ever needing more iterations than plain
    ILU(0) block-GMRES.  Both solves reach 1e-8 of ||B||."""
    import torch

    from blockpowerflow_b200 import learned

    gr = bpf.grid.make_grid(300, 68, seed=0)
    J = bpf.grid.jacobian(gr)
    A = bpf.CuSparseMatrixCSR.from_scipy(J)
    N = bpf.ilu0(A, 64)
    pairs, scale = learned.solver_pairs(gr, J, N, blocks=32, p=64, seed=0)
    mlp = learned.WarmStartMLP(J.shape[0], hidden=512, seed=0)
    mlp.set_scale(scale)
    learned.train(mlp, pairs, epochs=30, lr=1e-3, batch=64)
    A.nzVal.copy_(torch.as_tensor(J.data, device="cuda"))
    N.refactor(A.nzVal)
    B = bpf.grid.gaussian_rhs(J.shape[0], 64, 99)
    Bd = torch.as_tensor(B, device="cuda")
    Xs = np.linalg.solve(J.toarray(), B)
    X0 = mlp.forward(Bd).cpu().numpy()
    assert np.linalg.norm(X0 - Xs) / np.linalg.norm(Xs) < 0.5
    nb = np.linalg.norm(B)
    Xp, sp_ = bpf.block_gmres(A, Bd, N=N, ldiv=True, restart=False, memory=100, atol=1e-8 * nb,
                              rtol=0.0, itmax=100)
    Z = mlp.basis(16)
    Zh = Z.cpu().numpy()
    assert np.abs(Zh.T @ Zh - np.eye(16)).max() <= 1e-10
    Xl, sl = learned.solve(A, Bd, N, mlp, Z, rtol=1e-8, itmax=100, judge="residual")
    assert sp_.solved and sl.solved
    assert np.linalg.norm(B - J @ Xl.cpu().numpy()) <= 1e-8 * nb * 1.01
    assert sl.niter <= sp_.niter, (sl.niter, sp_.niter)


def test_learned_start_gains_on_held_out_operating_points(bpf):
    """What the trained network gains over plain ILU(0) block-GMRES, on the solves the Newton
    caller makes: sensitivities Gx^{-1} Gu[:, S] along a sequence of operating points of a
    2,000-bus grid (3,798 unknowns; states perturbed by N(0, 0.001); 64 of the grid's 201 controls
    per block).  The network is trained on 2,560 solver-generated solves at 40 points; at three
    held-out points the learned solve (its judged warm start and its rank-32 deflation basis)
    takes strictly fewer iterations than the plain solve, and both reach 1e-8 of ||B||."""
    import torch

    from blockpowerflow_b200 import learned
    from blockpowerflow_b200 import newton as NT

    prob = NT.make_problem(bpf.grid.make_grid(2000, seed=0))
    A = bpf.CuSparseMatrixCSR.from_scipy(prob.pattern)
    N = bpf.ilu0(A, 64)
    fam = learned.SensitivityFamily(prob, A, 64, sigma=0.001, seed=0)
    pairs, scale = learned.family_pairs(fam, N, range(40))
    assert len(pairs) == 40
    mlp = learned.WarmStartMLP(A.n, hidden=512, seed=0)
    mlp.set_scale(scale)
    hist = learned.train(mlp, pairs, epochs=100, lr=3e-4, batch=64)
    assert hist[-1] < 0.2 * hist[0], hist
    Z = mlp.basis(32)
    for t in (900, 901, 902):
        B = fam.point(t)
        N.refactor(A.nzVal)
        nb = float(torch.linalg.norm(B))
        Xp, sp_ = bpf.block_gmres(A, B, N=N, ldiv=True, restart=False, memory=300, atol=1e-8 * nb, rtol=0.0,
                                  itmax=300)
        Xl, sl = learned.solve(A, B, N, mlp, Z, rtol=1e-8, itmax=300)
        assert sp_.solved and sl.solved
        R = B - bpf.mul(A, Xl)
        assert float(torch.linalg.norm(R)) <= 1e-8 * nb * 1.01
        assert sl.niter < sp_.niter, (t, sl.niter, sp_.niter)


# ---- deflated block-GMRES ---------------------------------------------------------------------
def _slow_modes(A, r):
    """Real basis of the r eigenvectors of A M^{-1} (ILU(0), right) of smallest modulus, mapped
    to x-space by M^{-1} (dense; small systems only)."""
    import oracle as O

    n = A.shape[0]
    F = O.ilu0(A)
    Minv = O.prec_apply(1, F, np.eye(n))
    lam, V = np.linalg.eig(A @ Minv)
    idx = np.argsort(np.abs(lam))[:r]
    Yr = np.linalg.qr(np.hstack([V[:, idx].real, V[:, idx].imag]))[0][:, :r]
    return O.prec_apply(1, F, Yr)


def test_deflated_gmres_with_slow_modes_converges_faster(case300, bpf):
    import torch

    A = case300[0]
    n, p = A.shape[0], 16
    B = bpf.grid.gaussian_rhs(n, p, 3)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    N = bpf.ilu0(Ad, p)
    Bd = torch.as_tensor(B, device="cuda")
    kw = dict(N=N, ldiv=True, restart=False, memory=100, atol=0.0, rtol=1e-10, itmax=100)
    X, st = bpf.block_gmres(Ad, Bd, **kw)
    Z = torch.as_tensor(_slow_modes(A, 16), device="cuda")
    Xd, sd = bpf.block_gmres(Ad, Bd, deflation=Z, **kw)
    assert st.solved and sd.solved
    rel = np.linalg.norm(B - A @ Xd.cpu().numpy()) / np.linalg.norm(B)
    assert rel <= 1e-10 * 10
    assert sd.niter < st.niter, (sd.niter, st.niter)
    Xn = X.cpu().numpy()
    assert np.linalg.norm(Xd.cpu().numpy() - Xn) / np.linalg.norm(Xn) <= 1e-6


@pytest.mark.parametrize("restart", [False, True])
def test_deflated_gmres_with_any_basis_reaches_the_tolerance(case300, bpf, restart):
    import torch

    A = case300[0]
    n, p = A.shape[0], 16
    B = bpf.grid.gaussian_rhs(n, p, 5)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    N = bpf.ilu0(Ad, p)
    Z = torch.as_tensor(np.random.default_rng(0).standard_normal((n, 8)), device="cuda")
    X0 = torch.as_tensor(np.random.default_rng(1).standard_normal((n, p)), device="cuda")
    X, st = bpf.block_gmres(Ad, torch.as_tensor(B, device="cuda"), X0, N=N, ldiv=True, restart=restart,
                            memory=30, atol=1e-9 * np.linalg.norm(B), rtol=0.0, itmax=300, deflation=Z)
    assert st.solved
    assert np.linalg.norm(B - A @ X.cpu().numpy()) <= 1e-9 * np.linalg.norm(B) * 1.01
