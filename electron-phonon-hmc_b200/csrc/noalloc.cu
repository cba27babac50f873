// Log det + inverse that allocates nothing: the LU's workspace lives in a
// file-scope device array instead of buffers from cudaMalloc.
//
// For callers whose device memory belongs to someone else -- a framework's
// caching allocator or a pool sized once at start-up -- or who must not
// allocate after initialisation: for them a cudaMalloc inside the library
// either fails or takes memory the owner has already accounted for.  They pass
// the matrix (device memory they own) and get it back inverted, with log|det|,
// the sign and the pivots; the library touches no allocator.
//
// Limits and sharing:
//  * n <= kNoAllocMaxN (256): the workspace is the inverse buffer (n*n doubles),
//    U's diagonal (n+2 doubles), the pivots and their composed permutation
//    (2n ints), status flags and the LU kernel's panel flags, about
//    0.5 MB, held by every GPU that loads the library until the process exits;
//  * all calls share that one array and it keeps the last call's contents;
//    calls that overlap on the GPU (different streams or threads, or another
//    device context sharing the GPU) race on it and must be serialised by the
//    caller;
//  * every call looks up the array's device address on the current device
//    (cudaGetSymbolAddress, a host-side lookup), so no address outlives a
//    device reset or belongs to another device;
//  * the matrix must be memory of the current device;
//  * the call synchronizes the stream before it returns: log|det|, the sign
//    and the pivots are read back to the host.
#include "ephmc_internal.cuh"

namespace {

constexpr unsigned kNoAllocMaxN = 256;
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffX = 0;
constexpr size_t kOffDiag = kOffX + align256(sizeof(double) * kNoAllocMaxN * kNoAllocMaxN);
constexpr size_t kOffIpiv = kOffDiag + align256(sizeof(double) * (kNoAllocMaxN + 2));
constexpr size_t kOffInfo = kOffIpiv + align256(sizeof(int) * 2 * kNoAllocMaxN);  // pivots + permutation
constexpr size_t kOffSync = kOffInfo + align256(sizeof(int) * 2);
constexpr size_t kNoAllocBytes = kOffSync + align256(sizeof(unsigned) * ephmc::lu_sync_words(kNoAllocMaxN));

// Host code must not take this symbol's address directly (that is a host-side
// stand-in); the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// the array's device address on the current device, looked up anew by every
// call (a cached address would be stale after a device reset)
int scratch_for_current_device(unsigned char **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return ephmc::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    *out = static_cast<unsigned char *>(p);
    return EPHMC_OK;
}

}  // namespace

extern "C" {

EPHMC_API int ephmc_logdet_inverse_noalloc(double *M, unsigned n, double *logdet, int *sign, int *ipiv,
                                           void *stream) {
    ephmc::clear_status();
    if (!M || n == 0) {
        ephmc::set_status(EPHMC_ERR_ARG, "ephmc_logdet_inverse_noalloc: null matrix or n == 0");
        return EPHMC_ERR_ARG;
    }
    if (n > kNoAllocMaxN) {
        ephmc::set_status(EPHMC_ERR_ARG,
                          "ephmc_logdet_inverse_noalloc: n exceeds the 256 x 256 limit of the static workspace");
        return EPHMC_ERR_ARG;
    }
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, M) != cudaSuccess ||
        (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        ephmc::set_status(EPHMC_ERR_ARG, "ephmc_logdet_inverse_noalloc: M must be device memory");
        return EPHMC_ERR_ARG;
    }
    int dev = 0;
    EPHMC_CUDA(cudaGetDevice(&dev));
    if (a.type == cudaMemoryTypeDevice && a.device != dev) {
        // the workspace of the current device would be combined with another GPU's matrix
        ephmc::set_status(EPHMC_ERR_ARG, "ephmc_logdet_inverse_noalloc: M is memory of another device than the "
                                         "current one");
        return EPHMC_ERR_ARG;
    }
    unsigned char *base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc != EPHMC_OK) return rc;
    ephmc::LUWork w;
    w.V = (int)n;
    w.X = reinterpret_cast<double *>(base + kOffX);
    w.diag = reinterpret_cast<double *>(base + kOffDiag);
    w.ipiv = reinterpret_cast<int *>(base + kOffIpiv);
    w.info = reinterpret_cast<int *>(base + kOffInfo);  // zeroed by the factorisation itself
    w.sync = reinterpret_cast<unsigned *>(base + kOffSync);  // zero-initialised with the module
    w.sync_words = ephmc::lu_sync_words(kNoAllocMaxN);
    int sg = 1;
    double ld = 0;
    // synchronizes the stream: the results come back to the host
    rc = ephmc::lu_logdet_inverse(M, w, &ld, &sg, ipiv, static_cast<cudaStream_t>(stream));
    if (rc != EPHMC_OK) {
        ephmc::set_status(rc, rc == EPHMC_ERR_SINGULAR ? "zero pivot" : nullptr);
        return rc;  // *logdet and *sign are left as they were
    }
    if (logdet) *logdet = ld;
    if (sign) *sign = sg;
    return EPHMC_OK;
}

}  // extern "C"
