"""Learned warm start and deflation basis for block-GMRES (the solve path's learned part).

A 3-layer MLP (n -> hidden -> hidden -> n, LeakyReLU, BF16 tensor-core products with FP32
masters, Adam; csrc/mlp.cu) is trained on (b, x) pairs that the solver itself produces on
perturbed operating points of one grid.  It supplies

  * a warm start X0 = s ||b|| f(b / ||b||) for every right-hand side, and
  * a rank-r deflation basis: the orthonormalized outputs of the network on Gaussian probes,
    which block_gmres(..., deflation=Z) uses in the GCRO form.

Plain ILU(0) block-GMRES is the fallback and the judge: the solver always iterates to the
requested residual from whatever the network gives it, so the network can cost iterations but
never accuracy.  No counterpart in the reference (src/ has no learned component).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .sparse import CuSparseMatrixCSR, colmajor, empty_colmajor, ld

PARAMS = ("W1", "b1", "W2", "b2", "W3", "b3")


class WarmStartMLP:
    def __init__(self, n: int, hidden: int = 512, seed: int = 0, device=None):
        self.n, self.hidden = int(n), int(hidden)
        self._ctx = _lib.context(device)
        h = C.c_void_p()
        _lib.check(_lib.load().bpf_mlp_create(self._ctx, self.n, self.hidden, int(seed), C.byref(h)),
                   self._ctx)
        self._h = h
        self.scale = 1.0

    def set_scale(self, scale: float) -> None:
        self.scale = float(scale)
        _lib.check(_lib.load().bpf_mlp_set_scale(self._h, self.scale), self._ctx)

    def forward(self, B):
        """Warm starts (n x p, column-major) for the columns of B."""
        Bc = colmajor(B)
        X = empty_colmajor(self.n, Bc.shape[1], Bc.device)
        _lib.check(_lib.load().bpf_mlp_forward(self._h, Bc.shape[1], Bc.data_ptr(), ld(Bc), X.data_ptr(),
                                               ld(X)), self._ctx)
        return X

    def gradients(self, B, X) -> float:
        Bc, Xc = colmajor(B), colmajor(X)
        loss = C.c_double()
        _lib.check(_lib.load().bpf_mlp_gradients(self._h, Bc.shape[1], Bc.data_ptr(), ld(Bc), Xc.data_ptr(),
                                                 ld(Xc), C.byref(loss)), self._ctx)
        return loss.value

    def train_step(self, B, X, lr: float) -> float:
        Bc, Xc = colmajor(B), colmajor(X)
        loss = C.c_double()
        _lib.check(_lib.load().bpf_mlp_train_step(self._h, Bc.shape[1], Bc.data_ptr(), ld(Bc), Xc.data_ptr(),
                                                  ld(Xc), float(lr), C.byref(loss)), self._ctx)
        return loss.value

    def _shape(self, which: int):
        r, c = C.c_longlong(), C.c_longlong()
        _lib.check(_lib.load().bpf_mlp_params(self._h, which, None, None, C.byref(r), C.byref(c)), self._ctx)
        return r.value, c.value

    def param(self, name: str, grad: bool = False):
        """A copy (torch FP32, rows x cols) of parameter `name` or of its gradient."""
        import torch

        which = PARAMS.index(name)
        rows, cols = self._shape(which)
        out = torch.empty((rows, cols), dtype=torch.float32, device="cuda")
        _lib.check(_lib.load().bpf_mlp_param_copy(self._h, which, int(grad), out.data_ptr(), 0), self._ctx)
        import torch.cuda

        torch.cuda.synchronize()
        return out

    def set_param(self, name: str, value) -> None:
        import torch

        which = PARAMS.index(name)
        rows, cols = self._shape(which)
        v = value.to(device="cuda", dtype=torch.float32).contiguous()
        if v.numel() != rows * cols:
            raise ValueError(f"{name}: expected {rows} x {cols} values")
        _lib.check(_lib.load().bpf_mlp_param_copy(self._h, which, 0, v.data_ptr(), 1), self._ctx)
        torch.cuda.synchronize()

    def basis(self, rank: int = 32, seed: int = 0):
        """Orthonormal n x rank basis of the network's outputs on Gaussian probes."""
        Z = empty_colmajor(self.n, rank)
        _lib.check(_lib.load().bpf_mlp_basis(self._h, int(rank), int(seed), Z.data_ptr(), ld(Z)), self._ctx)
        return Z

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().bpf_mlp_destroy(h)
            except Exception:
                pass


def solver_pairs(grid, pattern, N, blocks: int, p: int, *, sigma: float = 0.01, seed: int = 0,
                 rtol: float = 1e-10, itmax: int = 300, device="cuda"):
    """Training data produced by the solver itself: for t < blocks, the Jacobian at an operating
    point perturbed by N(0, sigma) (fixed pattern), p Gaussian right-hand sides and their block-
    GMRES solutions (preconditioner N refactored per point).  Returns [(B_t, X_t)] (device,
    column-major) and the median ||x|| / ||b|| of the set."""
    import torch

    from . import grid as g
    from .krylov import block_gmres

    A = CuSparseMatrixCSR.from_scipy(pattern, device=device)
    pairs, ratios = [], []
    for t in range(blocks):
        vals = g.perturbed_values(grid, pattern, t, sigma=sigma, seed=seed)
        A.nzVal.copy_(torch.as_tensor(vals, device=device))
        N.refactor(A.nzVal)
        Bh = g.gaussian_rhs(pattern.shape[0], p, seed=10_000 * (seed + 1) + t)
        B = colmajor(torch.as_tensor(Bh, device=device))
        X, st = block_gmres(A, B, N=N, ldiv=True, restart=False, memory=itmax, atol=0.0, rtol=rtol,
                            itmax=itmax)
        if not st.solved:
            continue
        pairs.append((B, X))
        ratios.append((torch.linalg.norm(X, dim=0) / torch.linalg.norm(B, dim=0)).cpu().numpy())
    scale = float(np.median(np.concatenate(ratios))) if ratios else 1.0
    return pairs, scale


def train(mlp: WarmStartMLP, pairs, *, epochs: int = 10, lr: float = 2e-4, batch: int = 64, seed: int = 0):
    """Adam over the solver-generated pairs in batches of `batch` columns; returns the per-epoch
    mean losses."""
    rng = np.random.default_rng(seed)
    hist = []
    for _ in range(epochs):
        losses = []
        for t in rng.permutation(len(pairs)):
            B, X = pairs[t]
            for j0 in range(0, B.shape[1], batch):
                losses.append(mlp.train_step(B[:, j0:j0 + batch], X[:, j0:j0 + batch], lr))
        hist.append(float(np.mean(losses)))
    return hist


def judged_warm_start(mlp: WarmStartMLP, A: CuSparseMatrixCSR, B, N=None):
    """The network's warm start if it beats the zero start, else None: plain block-GMRES judges
    the network and falls back to it.  Without a preconditioner the test is the residual,
    ||B - A X0||_F < ||B||_F.  With the right preconditioner N (an approximate inverse of A) it is
    the estimated error, ||N \\ (B - A X0)||_F < ||N \\ B||_F: the network's misses are mostly
    short-wavelength components that A amplifies in the residual while the preconditioner removes
    them in the first iteration, so the residual alone would discard useful starts."""
    import torch

    from .precond import ldiv_
    from .sparse import mul

    Bc = colmajor(B)
    X0 = mlp.forward(Bc)
    R = Bc.clone()   # a copy with Bc's (column-major) strides; B itself is left untouched
    mul(A, X0, alpha=-1.0, beta=1.0, Y=R)
    if N is None:
        return X0 if float(torch.linalg.norm(R)) < float(torch.linalg.norm(Bc)) else None
    E = empty_colmajor(Bc.shape[0], Bc.shape[1], Bc.device)
    ldiv_(E, N, R)
    e0 = float(torch.linalg.norm(E))
    ldiv_(E, N, Bc)
    return X0 if e0 < float(torch.linalg.norm(E)) else None


def solve(A: CuSparseMatrixCSR, B, N, mlp: WarmStartMLP, Z=None, *, rtol: float = 1e-8,
          itmax: int = 300, judge: str = "error"):
    """Right-preconditioned block-GMRES from the network's warm start, augmented with the learned
    deflation basis Z (if given); the tolerance is rtol ||B||_F whatever the start.

    Plain ILU(0) block-GMRES is the judge and the fallback.  Up front, judged_warm_start keeps
    the warm start only if it beats the zero start (judge "error": the estimated error through N,
    the default; "residual": the residual; "final": always kept).  At the end, its stopping test
    on ||B - A X||_F decides, and if the learned solve does not reach the tolerance within itmax
    the plain solve from the zero start runs instead: the network can cost iterations, never
    accuracy."""
    import torch

    from .krylov import block_gmres

    Bc = colmajor(B)
    nb = float(torch.linalg.norm(Bc))
    if judge == "final":
        X0 = mlp.forward(Bc)
    else:
        X0 = judged_warm_start(mlp, A, Bc, N if judge == "error" else None)
    X, st = block_gmres(A, Bc, X0, N=N, ldiv=True, restart=False, memory=itmax, atol=rtol * nb,
                        rtol=0.0, itmax=itmax, deflation=Z)
    if st.solved or (X0 is None and Z is None):
        return X, st
    Xp, sp_ = block_gmres(A, Bc, N=N, ldiv=True, restart=False, memory=itmax, atol=rtol * nb, rtol=0.0,
                          itmax=itmax)
    sp_.niter += st.niter   # the failed learned attempt counts
    return Xp, sp_


# ---- the sensitivity family: solves the Newton caller makes along a sequence of operating points
class SensitivityFamily:
    """Right-hand sides of the Newton caller's sensitivity solves (benchmarks_nvidia.jl:29-39
    solves Gx X = Gu) along a sequence of nearby operating points of one grid.

    Point t: the state x_t = the solution's, perturbed by N(0, sigma) in every angle and PQ
    magnitude (newton.perturbed_start with seed `seed + t`); Gx(x_t) is assembled on the device
    into A's values, Gu(x_t) into a device block, and the block's right-hand sides are the
    columns of Gu(x_t) for p controls drawn (seeded by t) from a fixed set of controls of interest
    (`controls`, default: up to 512 of the grid's slack / PV controls)."""

    def __init__(self, prob, A: CuSparseMatrixCSR, p: int, *, controls=None, sigma: float = 0.001,
                 seed: int = 0):
        import torch

        from . import newton as NT

        self.prob, self.A, self.p, self.sigma, self.seed = prob, A, int(p), float(sigma), int(seed)
        self.asm = NT.DeviceAssembly(prob, A)
        nc = self.asm.n_ctrl
        if controls is None:
            rng = np.random.default_rng(seed)
            controls = np.sort(rng.choice(nc, size=min(512, nc), replace=False))
        self.controls = np.asarray(controls, dtype=np.int64)
        if self.p > len(self.controls):
            raise ValueError(f"p = {p} exceeds the {len(self.controls)} controls of interest")
        dev = A.nzVal.device
        self.Gu = torch.empty((nc, self.asm.n), dtype=torch.float64, device=dev).t()   # column-major
        self._dev = dev

    def point(self, t: int):
        """Assemble point t: A's values become Gx(x_t); returns B_t (column-major n x p)."""
        import torch

        from . import newton as NT

        x = NT.perturbed_start(self.prob, self.sigma, seed=self.seed + t)
        self.asm.jacobian(torch.as_tensor(x, device=self._dev), self.Gu)
        rng = np.random.default_rng(1_000_003 + 7919 * self.seed + t)
        cols = np.sort(rng.choice(self.controls, size=self.p, replace=False))
        idx = torch.as_tensor(cols, device=self._dev)
        return colmajor(self.Gu.index_select(1, idx))


def family_pairs(fam: SensitivityFamily, N, points, *, rtol: float = 1e-10, itmax: int = 400):
    """Training data the solver generates on the family: for each point t, B_t and its plain
    ILU(0) block-GMRES solution (N refactored at the point).  Returns [(B_t, X_t)] (device,
    column-major) and the median ||x|| / ||b||."""
    import torch

    from .krylov import block_gmres

    pairs, ratios = [], []
    for t in points:
        B = fam.point(t)
        N.refactor(fam.A.nzVal)
        X, st = block_gmres(fam.A, B, N=N, ldiv=True, restart=False, memory=itmax, atol=0.0, rtol=rtol,
                            itmax=itmax)
        if not st.solved:
            continue
        pairs.append((B, X))
        ratios.append((torch.linalg.norm(X, dim=0) / torch.linalg.norm(B, dim=0)).cpu().numpy())
    scale = float(np.median(np.concatenate(ratios))) if ratios else 1.0
    return pairs, scale
