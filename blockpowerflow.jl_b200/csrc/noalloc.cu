// bpf_prec_apply_noalloc: ldiv!(Y, P, X) for callers that cannot allocate device memory.
//
// bpf_prec_apply converts the column-major block into the library's row-major layout in a
// workspace buffer that the context grows with cudaMalloc on first use (and again whenever a
// larger block arrives).  Some callers cannot allow that: hosts whose device memory is owned by
// an external pool or allocator (a framework's caching allocator, a fixed arena carved out at
// start-up, where a cudaMalloc behind the pool's back can fail or fragment it), and real-time or
// latency-bound loops that forbid allocation after set-up (a cudaMalloc synchronizes the device
// and takes an unbounded time).  This entry point runs the same conversion and triangular-solve
// kernels with its scratch in a file-scope __device__ array instead, so after the preconditioner
// has been built it performs no allocation at all.
//
// Limits and sharing rules:
//  * The scratch holds kNoAllocScratchDoubles = 2^20 doubles (8 MiB).  A call solves its block
//    in slices of at most 256 right-hand sides, so it needs n * min(p, 256) <= 2^20 doubles;
//    larger requests are rejected with BPF_ERR_NOT_SUPPORTED.  Every GPU that loads the
//    library carries these 8 MiB until the process exits.
//  * Every call on a device shares the one array and leaves the last call's contents in it.
//    Nothing needs to start at zero (each slice is overwritten by the layout conversion before
//    it is read), but two calls whose work overlaps on the GPU (different streams or
//    contexts without ordering between them) race on the array.
//  * The array's device address is looked up with cudaGetSymbolAddress, with that device
//    current, on the first call made on a device after a library context was created there
//    (creating a context forgets the device's address, so a context made after a device reset
//    never uses a stale one).  That first call does the set-up; the later ones only read it.
//  * A reordered preconditioner solves through its own factor-ordered scratch, sized at creation
//    for `nrhs` columns; this entry point never grows it, so such a preconditioner takes at most
//    min(nrhs, 256) columns per slice here (BPF_ERR_NOT_SUPPORTED beyond).
#include <algorithm>
#include <mutex>

#include "bpf_internal.cuh"
#include "prec.cuh"

namespace bpf {

constexpr size_t kNoAllocScratchDoubles = size_t(1) << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

static double *g_noalloc_ptr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

// A context was created on `dev`: look the address up again on the next call there.
void noalloc_forget_device(int dev) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    g_noalloc_ptr[dev] = nullptr;
}

// Device address of the scratch on the current device (looked up once per device and context
// generation).
static bpf_status noalloc_scratch(bpf_ctx *ctx, double **out) {
    int dev = -1;
    BPF_CUDA(ctx, cudaGetDevice(&dev));
    if (dev != ctx->device)
        return set_error(ctx, BPF_ERR_INVALID_VALUE,
                         "prec_apply_noalloc: device %d is current, the preconditioner lives on %d",
                         dev, ctx->device);
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "prec_apply_noalloc: device index %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_error(ctx, e, "cudaGetSymbolAddress", __FILE__, __LINE__);
        g_noalloc_ptr[dev] = (double *)p;
    }
    *out = g_noalloc_ptr[dev];
    return BPF_SUCCESS;
}

}  // namespace bpf

using namespace bpf;

extern "C" bpf_status bpf_prec_apply_noalloc(bpf_prec *P, int p, const double *X, int ldx,
                                             double *Y, int ldy) {
    if (!P) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = P->ctx;
    const int n = P->n;
    if (p < 0 || (p > 0 && n > 0 && (!X || !Y)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "prec_apply_noalloc: invalid argument");
    if (ldx < std::max(1, n) || ldy < std::max(1, n))
        return set_error(ctx, BPF_ERR_DIMENSION, "prec_apply_noalloc: leading dimension < n");
    if (n == 0 || p == 0) return BPF_SUCCESS;
    const int chunk = 256;
    const size_t need = (size_t)n * (size_t)std::min(p, chunk);
    if (need > kNoAllocScratchDoubles)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "prec_apply_noalloc: n * min(p, 256) = %zu doubles exceeds the %zu-double "
                         "static scratch; use bpf_prec_apply",
                         need, kNoAllocScratchDoubles);
    if (P->perm && std::min(p, chunk) > P->zcols)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "prec_apply_noalloc: this reordered preconditioner was created for %d right-hand "
                         "sides and bpf_prec_apply_noalloc never grows its scratch; pass at most %d columns "
                         "per call or create it with nrhs >= %d",
                         P->zcols, P->zcols, std::min(p, chunk));
    double *buf = nullptr;
    BPF_TRY(noalloc_scratch(ctx, &buf));
    for (int c0 = 0; c0 < p; c0 += chunk) {
        const int pc = std::min(chunk, p - c0);
        BPF_TRY(colmajor_to_rowmajor(ctx, n, pc, X + (size_t)c0 * ldx, ldx, buf));
        BPF_TRY(prec_apply_rowmajor(ctx, P, pc, buf, buf));
        BPF_TRY(rowmajor_to_colmajor(ctx, n, pc, buf, Y + (size_t)c0 * ldy, ldy));
    }
    return BPF_SUCCESS;
}
