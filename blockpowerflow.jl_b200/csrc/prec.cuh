// Internal types of the preconditioner / triangular-factor machinery.
#pragma once

#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#include "bpf_internal.cuh"

namespace bpf {

// A triangular factor analysed on the host: rows stored level by level.
struct TriHost {
    int n = 0;
    int nlev = 0;
    int max_level_rows = 0;
    bool unit = true;
    std::vector<int> lev_ptr;  // nlev+1, positions into rows
    std::vector<int> rows;     // n, row id at each level-sorted position
    std::vector<int> rp;       // n+1, per level-sorted position
    std::vector<int> ci;       // off-diagonal column ids
    std::vector<int> map;      // position of each off-diagonal entry in the source pattern
    std::vector<int> dmap;     // position of the diagonal in the source pattern (non-unit)
};

// Plain-pointer view passed to kernels.
struct TriKernelArgs {
    int n, nlev, nnz;
    const int *lev_ptr, *rows, *rp, *ci, *map, *dmap;
    double *val;
    float *valf;
    double *dinv;
    float *dinvf;
};

struct TriDev {
    int n = 0, nlev = 0, nnz = 0, max_level_rows = 0;
    bool unit = true;
    std::vector<int> lev_ptr_h;
    int *lev_ptr = nullptr, *rows = nullptr, *rp = nullptr, *ci = nullptr, *map = nullptr,
        *dmap = nullptr;
    double *val = nullptr;
    float *valf = nullptr;
    double *dinv = nullptr;
    float *dinvf = nullptr;
    TriKernelArgs args() const {
        TriKernelArgs a;
        a.n = n;
        a.nlev = nlev;
        a.nnz = nnz;
        a.lev_ptr = lev_ptr;
        a.rows = rows;
        a.rp = rp;
        a.ci = ci;
        a.map = map;
        a.dmap = dmap;
        a.val = val;
        a.valf = valf;
        a.dinv = dinv;
        a.dinvf = dinvf;
        return a;
    }
};

enum PrecKind { PREC_ILU0 = 1, PREC_IC0 = 2, PREC_LU = 3, PREC_BJ = 4 };

TriHost build_tri(int n, const int *rp, const int *ci, const int *diag, int part, bool unit);
// An allocator whose value-less construct leaves the element uninitialised, so resize() of a
// buffer that is written in full right after (tens of millions of update pairs) neither zero-fills
// it nor takes its first-touch page faults on one thread.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void *>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U *p, Args &&...args) {
        ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
    }
};
using PairVec = std::vector<int, NoInitAlloc<int>>;

// false (and empty outputs) when the pair count exceeds INT_MAX
bool build_pairs(int n, const int *rp, const int *ci, const int *diag, bool ic,
                 std::vector<int> &pp, PairVec &pdst, PairVec &psrc);
bpf_status tri_upload(bpf_ctx *ctx, const TriHost &h, TriDev &d);
void tri_free(TriDev &d);
bpf_status tri_scatter(bpf_ctx *ctx, const TriDev &d, const double *fv);

}  // namespace bpf

// The preconditioner object behind the C ABI (NVIDIA_ILU0 / NVIDIA_IC0).
struct bpf_prec {
    bpf_ctx *ctx = nullptr;
    int kind = 0;
    int n = 0, nnz = 0, nrhs = 0;
    int fdtype = BPF_F64;
    // pattern (0-based device copies) and factor values in pattern order
    int *rp = nullptr, *ci = nullptr, *diag = nullptr;
    double *fv = nullptr;
    int *pp = nullptr, *pdst = nullptr, *psrc = nullptr;
    long long npairs = 0;
    bpf::TriDev lower;   // forward solve (L unit for ILU0; L for IC0)
    bpf::TriDev upper;   // backward solve (U for ILU0; L' for IC0)
    // LU on a fill pattern (the RF refactorization): right-looking column steps; step k (scale
    // column k of L by 1 / u_kk, then apply its update pairs) waits for the steps that update
    // row k or column k.  cl_lev_ptr / cl_ent: the L entries of each level's steps.
    int cl_nlev = 0, cl_max_level = 0;
    int *cl_lev_ptr = nullptr, *cl_ent = nullptr;
    // Without stored update pairs (patterns whose pairs exceed 2^31 - 1, or BPF_LU_PAIRLESS=1):
    // each L entry's updates are found by a search in its row; cl_row = the row of each listed
    // entry.  npairs then counts the updates.
    bool pairless = false;
    int *cl_row = nullptr;
    // LU solves in push form (right-looking): per level of each sweep, the factor entries whose
    // source row became final at that level, as (source row, target row, position in fv).
    int ps_nlev[2] = {0, 0}, ps_max_level = 0;
    int *ps_ptr[2] = {nullptr, nullptr}, *ps_src[2] = {nullptr, nullptr},
        *ps_dst[2] = {nullptr, nullptr}, *ps_pos[2] = {nullptr, nullptr};
    // Symmetric reordering (bpf_ilu0_create_ordered): the factors are those of A_hat =
    // A(perm, perm); perm[i] = original row of factor row i; amap[k] = position of A's entry
    // k in A_hat's pattern; zbuf = n x zcols factor-ordered scratch of the solves.
    int ordering = BPF_ORDER_NATURAL;
    int *perm = nullptr, *amap = nullptr;
    std::vector<int> perm_host;
    double *zbuf = nullptr;
    int zcols = 0;
    // Sync-free triangular solves: one ready word per factor row, 2e when the forward sweep of
    // launch e has produced the row and 2e + 1 after the backward sweep (monotone across
    // launches, so nothing is reset between them).
    unsigned *sf_flags = nullptr;
    mutable unsigned sf_epoch = 0;
    // Block-Jacobi (bpf_block_jacobi_create): rows of each block (nblk x 32, -1 padded), block and
    // local index of every row, dense inverses (nblk x 32 x 32); fv holds A's values.
    int bj_nblk = 0, bj_bs = 0;
    int *bj_rows = nullptr, *bj_blk = nullptr, *bj_loc = nullptr;
    double *bj_inv = nullptr;
};

namespace bpf {
bpf_status prec_setup(bpf_ctx *ctx, int kind, int n, const std::vector<int> &rp,
                      const std::vector<int> &ci, const std::vector<int> &diag, bpf_prec **out);
bpf_status csr_pattern_to_host(bpf_ctx *ctx, const bpf_csr_desc *A, std::vector<int> &rp,
                               std::vector<int> &ci, bool need_diag, std::vector<int> *diag);
bpf_status factor_numeric(bpf_ctx *ctx, bpf_prec *P);
bpf_status prec_apply_rowmajor(bpf_ctx *ctx, const bpf_prec *P, int p, const double *X,
                               double *Y, const int *gate = nullptr);
// Reordered preconditioners: make the factor-ordered scratch hold p columns (allocates when it
// grows; prec_apply_rowmajor itself never allocates and rejects p > zcols).
bpf_status prec_reserve_z(bpf_ctx *ctx, bpf_prec *P, int p);
// A's values into the factor storage (a copy, or the scatter through amap when reordered).
bpf_status prec_load_values(bpf_ctx *ctx, bpf_prec *P, const double *vals);
// Block-Jacobi: inverses of the diagonal blocks from fv; Y = P X (row-major, Y may be X).
bpf_status bj_setup(bpf_ctx *ctx, bpf_prec *P);
bpf_status bj_apply_rowmajor(bpf_ctx *ctx, const bpf_prec *P, int p, const double *X, double *Y);
// Y = U^{-1} L^{-1} Y in place (row-major n x p, p <= 256) for an LU factor with push lists.
bpf_status lu_solve_push_rowmajor(bpf_ctx *ctx, const bpf_prec *P, int p, double *Y);
}  // namespace bpf
