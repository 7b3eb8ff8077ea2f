// bpf_prec_apply_noalloc: ldiv!(Y, P, X) for callers that cannot allocate device memory.
//
// bpf_prec_apply converts the column-major block into the library's row-major layout in a
// workspace buffer that the context grows with cudaMalloc on first use (and again whenever a
// larger block arrives).  Some callers cannot allow that: code running inside a stream capture
// that must not see a cudaMalloc, hosts whose device memory is owned by an external pool or
// allocator (a framework's caching allocator, a fixed arena carved out at start-up), or
// real-time loops that forbid allocation after set-up.  This entry point runs the same
// conversion and triangular-solve kernels with its scratch in a file-scope __device__ array
// instead, so after the preconditioner has been built it performs no allocation at all.
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
//  * The array's device address is looked up once per device with cudaGetSymbolAddress, with
//    that device current, on the first call made on it; make that first call before any stream
//    capture begins.
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

// Device address of the scratch on the current device (looked up once per device).
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
