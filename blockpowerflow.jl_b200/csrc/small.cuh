// Launchers of the small (p x p) kernels in small.cu.
#pragma once

#include "bpf_internal.cuh"
#include "dense.cuh"

namespace bpf {

// Cholesky of G (p x p) for Cholesky-QR: Rinv = R^{-1}, Racc <- R Racc (pass > 0) or R.
// Rtmp: p x p global scratch.  Flags as documented at cholqr().
bpf_status launch_chol(bpf_ctx *ctx, int n, int p, const double *G, double *Rinv, double *Racc,
                       double *Rtmp, int pass, SolveState *st, const int *gate, const int *gate2,
                       int *shift_flag, int *reorth_flag);

// One block-Hessenberg QR update of block-GMRES iteration k (1-based): apply the stored
// reflectors to block column k-1, factor [R_jj; C], update Z and the stopping test.
// scr: 3 p x p global scratch; tau: p.
bpf_status launch_hess(bpf_ctx *ctx, int p, int k, double *Rblk, double *HY, double *tau,
                       double *Z, const double *Cm, SolveState *st, double *hist, double *scr);

}  // namespace bpf
