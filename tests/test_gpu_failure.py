"""Failure detection on the device without a GPU fault: a bounded wait that runs out.

The cooperative kernels (triangular solves, factorizations) meet at grid barriers whose waits are
bounded.  Here one block of a cooperative launch never arrives at the barrier (a flag that nothing
sets); the others give up after the context's wait limit, the call returns BPF_ERR_TIMEOUT, and the
same context then runs a preconditioner apply that still matches the oracle.  Nothing faults,
traps or hangs: every wait ends by itself after ~4,096 polls.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def test_grid_barrier_times_out_and_the_context_stays_usable(bpf, case300):
    import torch

    from blockpowerflow_b200 import _lib

    lib = _lib.load()
    ctx = _lib.context()
    arrived = C.c_int(-1)
    # every block arrives: the barrier passes
    assert lib.bpf_selftest_grid_barrier(ctx, 8, -1, C.byref(arrived)) == _lib.BPF_SUCCESS
    assert arrived.value == 8
    # block 3 never arrives: the other 7 give up after the (shortened) wait limit
    assert lib.bpf_ctx_set_wait_limit(ctx, 4096) == _lib.BPF_SUCCESS
    try:
        st = lib.bpf_selftest_grid_barrier(ctx, 8, 3, C.byref(arrived))
        assert st == _lib.BPF_ERR_TIMEOUT, st
        assert "timed out" in _lib.last_error(ctx)
        assert arrived.value == 0
    finally:
        assert lib.bpf_ctx_set_wait_limit(ctx, 0) == _lib.BPF_SUCCESS
    # the status word was cleared: the same context runs the cooperative ILU(0) apply correctly
    assert lib.bpf_selftest_grid_barrier(ctx, 8, -1, C.byref(arrived)) == _lib.BPF_SUCCESS
    A, _ = case300
    X = np.random.default_rng(5).standard_normal((A.shape[0], 4))
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    P = bpf.ilu0(Ad, 4)
    Y = torch.empty((4, A.shape[0]), dtype=torch.float64, device="cuda").t()
    bpf.ldiv_(Y, P, torch.as_tensor(X, device="cuda"))
    Yo = O.prec_apply(1, O.ilu0(A), X)
    assert np.linalg.norm(Y.cpu().numpy() - Yo) <= 1e-12 * np.linalg.norm(Yo)


def test_selftest_arguments_are_checked(bpf):
    from blockpowerflow_b200 import _lib

    lib = _lib.load()
    ctx = _lib.context()
    assert lib.bpf_selftest_grid_barrier(ctx, 1, -1, None) == _lib.BPF_ERR_INVALID_VALUE
    assert lib.bpf_selftest_grid_barrier(ctx, 4, 4, None) == _lib.BPF_ERR_INVALID_VALUE
    assert lib.bpf_ctx_set_wait_limit(ctx, -1) == _lib.BPF_ERR_INVALID_VALUE
