"""block_bicgstab on the GPU through the C ABI vs the CPU oracle (src/block_bicgstab.jl).

The oracle is the CPU twin (LU of K); the device uses Householder QR of K like the reference's
GPU variant.  Iteration counts agree within 1 and the first residual norms to 1e-4 relative
(BiCGSTAB's recurrences amplify the different rounding of the LU and QR solves of K).
"""
import numpy as np
import pytest

import oracle as O
from conftest import spd_from

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _t(x):
    import torch

    return torch.as_tensor(np.asarray(x), device="cuda")


def test_bicgstab_synthetic_300bus_ilu0(bpf):
    A = bpf.grid.preset_jacobian("case300", 0)
    B = bpf.grid.gaussian_rhs(A.shape[0], 16, 1)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    X, st = bpf.block_bicgstab(Ad, _t(B), N=bpf.ilu0(Ad, 16), atol=0.0, rtol=1e-8, history=True)
    Xo, so = O.block_bicgstab(A, B, N=(1, O.ilu0(A)), atol=0.0, rtol=1e-8, history=True)
    assert st.solved and so.solved
    assert abs(st.niter - so.niter) <= 1
    k = min(len(st.residuals), len(so.residuals), 8)
    np.testing.assert_allclose(st.residuals[:k], so.residuals[:k], rtol=1e-4)
    X = X.cpu().numpy()
    assert np.linalg.norm(B - A @ X) <= 1e-8 * np.linalg.norm(B) * 1.0001


def test_bicgstab_spd_ic0_and_identity(case300, bpf):
    A, _ = case300
    S = spd_from(A)
    B = np.random.default_rng(2).standard_normal((S.shape[0], 4))
    Sd = bpf.CuSparseMatrixCSR.from_scipy(S)
    X, st = bpf.block_bicgstab(Sd, _t(B), N=bpf.ic0(Sd, 4), atol=0.0, rtol=1e-10, itmax=500,
                               history=True)
    Xo, so = O.block_bicgstab(S, B, N=(2, O.ic0(S)), atol=0.0, rtol=1e-10, itmax=500, history=True)
    assert st.solved and abs(st.niter - so.niter) <= 1
    np.testing.assert_allclose(X.cpu().numpy(), Xo, rtol=0, atol=1e-8 * np.abs(Xo).max())
    X, st = bpf.block_bicgstab(Sd, _t(B), atol=0.0, rtol=1e-10, itmax=500)
    assert st.solved
    assert np.linalg.norm(B - S @ X.cpu().numpy()) <= 1e-10 * np.linalg.norm(B) * 1.0001


def test_bicgstab_explicit_shadow_and_itmax(case300, bpf):
    A, _ = case300
    S = spd_from(A)
    rng = np.random.default_rng(4)
    B = rng.standard_normal((S.shape[0], 3))
    Cs = rng.standard_normal((S.shape[0], 3))
    Sd = bpf.CuSparseMatrixCSR.from_scipy(S)
    X, st = bpf.block_bicgstab(Sd, _t(B), C=_t(Cs), N=bpf.ic0(Sd, 3), atol=0.0, rtol=1e-10,
                               itmax=500, history=True)
    Xo, so = O.block_bicgstab(S, B, C_shadow=Cs, N=(2, O.ic0(S)), atol=0.0, rtol=1e-10, itmax=500,
                              history=True)
    assert st.solved and abs(st.niter - so.niter) <= 1
    X, st = bpf.block_bicgstab(Sd, _t(B), itmax=2, atol=0.0, rtol=1e-15)
    assert st.niter == 2 and not st.solved
    assert st.status == "maximum number of iterations exceeded"
