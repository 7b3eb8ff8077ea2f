"""Generate the golden fixtures of the parity tests from the reference's own data files.

Run once in a container that has the reference checkout (read-only) at REF_ROOT:

    python tests/golden/make_golden.py /path/to/BlockPowerFlow.jl

Outputs (committed, a few hundred KB):
  case300.npz      data/case300.txt (530 x 530 Jacobian used by test/*.jl) as CSR, a seeded
                   b = rand(530) (test/cusolverRF.jl:7 draws an unseeded rand(n)), the direct
                   solution J \\ b (scipy SuperLU; the reference uses UMFPACK, :12) and the
                   identity block B = I[:, 1:32] of test/block_gmres.jl:8-11 with its direct
                   solution.
  dump_case300.npz benchmarks/dump/Gx_case300.mtx and Gu_case300.mtx (the benchmark's
                   Jacobian and dense sensitivity right-hand sides, benchmarks_nvidia.jl:29-39)
                   with the direct solution of Gx X = Gu.
  dump_case118.npz the same for case118 (a second real grid).
  gx_case9241pegase.npz  benchmarks/dump/Gx_case9241pegase.mtx alone (17,036 x 17,036, 129k
                   nonzeros: the Jacobian benchmarks_nvidia.jl solves by default, :22); the tests
                   draw their own right-hand sides and direct solutions.
"""
import os
import sys

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl
from scipy.io import mmread

HERE = os.path.dirname(os.path.abspath(__file__))


def csr_arrays(A):
    A = sp.csr_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    return dict(indptr=A.indptr.astype(np.int32), indices=A.indices.astype(np.int32),
                data=A.data.astype(np.float64), shape=np.array(A.shape))


def main(ref_root):
    J = sp.csr_matrix(mmread(os.path.join(ref_root, "data", "case300.txt")))
    n = J.shape[0]
    rng = np.random.default_rng(20231001)
    b = rng.random(n)
    lu = spl.splu(J.tocsc())
    x = lu.solve(b)
    B32 = np.zeros((n, 32))
    B32[np.arange(32), np.arange(32)] = 1.0
    X32 = lu.solve(B32)
    np.savez_compressed(os.path.join(HERE, "case300.npz"), **csr_arrays(J), b=b, x=x, B32=B32,
                        X32=X32)
    for case in ("case300", "case118"):
        Gx = sp.csr_matrix(mmread(os.path.join(ref_root, "benchmarks", "dump", f"Gx_{case}.mtx")))
        Gu = np.asarray(mmread(os.path.join(ref_root, "benchmarks", "dump", f"Gu_{case}.mtx")).todense())
        Xd = spl.splu(Gx.tocsc()).solve(Gu)
        np.savez_compressed(os.path.join(HERE, f"dump_{case}.npz"), **csr_arrays(Gx), Gu=Gu, X=Xd)
    Gx = sp.csr_matrix(mmread(os.path.join(ref_root, "benchmarks", "dump", "Gx_case9241pegase.mtx")))
    np.savez_compressed(os.path.join(HERE, "gx_case9241pegase.npz"), **csr_arrays(Gx))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
