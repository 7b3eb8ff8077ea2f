// Launchers of the small (p x p) kernels in small.cu.
#pragma once

#include "bpf_internal.cuh"
#include "dense.cuh"

namespace bpf {

// Packed upper-triangular block storage of the block Hessenberg R: block (i, j), i <= j, at
// j (j + 1) / 2 + i (src/block_gmres.jl:54,302,369-372).
__host__ __device__ inline size_t rblk_pos(int i, int j) { return (size_t)j * (j + 1) / 2 + i; }

// Doubles per block column of the reflector storage HY: Y_j (2p x (p+1)), T_j (p x (p+1)),
// R_jj^{-1} (p x p), rounded up to an even count (16-byte aligned blocks for bulk copies).
__host__ __device__ inline size_t hy_stride(int p) {
    const size_t s = 3 * (size_t)p * (p + 1) + (size_t)p * p;
    return (s + 1) & ~(size_t)1;
}

// Cholesky of G (p x p) for Cholesky-QR: Rinv = R^{-1}, Racc <- R Racc (pass > 0) or R.
// gscr: 2 p^2 doubles of global scratch.  Flags as documented at cholqr().
bpf_status launch_chol(bpf_ctx *ctx, int n, int p, const double *G, double *Rinv, double *Racc,
                       double *gscr, int pass, SolveState *st, const int *gate, const int *gate2,
                       int *shift_flag, int *reorth_flag, int iter_tag = -1);

// One block-Hessenberg QR update of block-GMRES iteration k (1-based): apply the stored
// reflectors to block column k-1, factor [R_jj; C], update Z and the stopping test.
// HY: hy_stride(p) doubles per block column; scr: 5 p^2 + p global scratch; tau: p.
bpf_status launch_hess(bpf_ctx *ctx, int p, int k, double *Rblk, double *HY, double *tau,
                       double *Z, const double *Cm, SolveState *st, double *hist, double *scr);

// Block back substitution R Y = Z over block rows 0..k-1 (Z is overwritten).
bpf_status launch_backsub(bpf_ctx *ctx, int p, int k, const double *Rblk, const double *HY,
                          double *Z, double *Y);

}  // namespace bpf
