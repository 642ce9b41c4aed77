// trlx_g_dot_noalloc: the Gram-Schmidt projection of trlx_g_dot for callers
// that must not allocate device memory.
//
// Who needs it: code that runs under an application-wide device-memory
// budget or a caching allocator that owns all GPU memory (where a library's
// own cudaMalloc can fail or fragment the pool), and code called from inside
// a user operator or another library's hot loop, where cudaMalloc/cudaFree
// may synchronize the device and stall or deadlock the caller.  This entry
// point takes its reduction scratch from a fixed array compiled into the
// library instead of allocating it.
//
// The scratch is one file-scope __device__ array of kScratchDoubles doubles
// (592 KiB + a 256-byte header holding the grid ticket).  Every GPU that
// loads this library holds that array until the process exits.  It supports
// m1 + m2 <= TRLX_G_DOT_NOALLOC_MAX_COLS (512) columns; larger requests are
// rejected with -7.  All calls share the array and it keeps the last call's
// contents: the ticket is cleared at the start of every call, and the
// partial sums are always written before they are read.  Two calls whose
// kernels overlap on the GPU (different streams, or different host threads
// on the same device) race on the array and give wrong results; serialise
// them, e.g. on one stream.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in).  The first call on each device, with that
// device current, looks the address up with cudaGetSymbolAddress and caches
// it.  With CUDA's lazy module loading (the default) that lookup is also
// what loads the library's module, and with it the array, onto the device:
// the first call may itself allocate device memory and synchronize.  Make it
// once per device as a warm-up, outside any memory budget, hot loop or
// stream capture; later calls allocate nothing.
#include <cstdio>
#include <mutex>

#include "../../../include/trlx.h"
#include "gdot.h"

namespace {

constexpr int kMaxBlocks = 148;
constexpr int kMaxCols = TRLX_G_DOT_NOALLOC_MAX_COLS;
constexpr size_t kHeaderDoubles = 32;  // 256 bytes: grid ticket
constexpr size_t kScratchDoubles = kHeaderDoubles + (size_t)kMaxBlocks * kMaxCols;

static __device__ __align__(256) double g_gdot_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_gdot_scratch on the current device (set-up on first
// use per device).  Returns nullptr and prints the CUDA error on failure.
double *scratch_address(int *err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *err = -1001;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_gdot_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "trlx_g_dot_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                         cudaGetErrorString(e));
            *err = -1001;
            return nullptr;
        }
        g_scratch_addr[dev] = p;
    }
    return static_cast<double *>(g_scratch_addr[dev]);
}

}  // namespace

extern "C" int trlx_g_dot_noalloc(int nrow, const double *v1, int ld1, int m1, const double *v2, int ld2, int m2,
                                  const double *rr, double *wrk, void *stream) {
    const int m = m1 + m2;
    if (m1 < 0 || m2 < 0 || nrow < 0) return -1;
    if (m <= 0) return 0;
    if (ld1 < nrow || ld2 < nrow) {
        std::fprintf(stderr, "trlx_g_dot_noalloc: incorrect array sizes\n");
        return -201;
    }
    if (m > kMaxCols) {
        std::fprintf(stderr, "trlx_g_dot_noalloc: %d columns exceed the fixed scratch limit of %d\n", m, kMaxCols);
        return -7;
    }
    if (!rr || !wrk || (m1 > 0 && !v1) || (m2 > 0 && !v2)) return -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // No local rows (a rank that owns none): the partial products are zero.
    if (nrow == 0) return cudaMemsetAsync(wrk, 0, sizeof(double) * m, st) == cudaSuccess ? 0 : -1001;
    int err = 0;
    double *base = scratch_address(&err);
    if (!base) return err;
    unsigned *ticket = reinterpret_cast<unsigned *>(base);
    double *part = base + kHeaderDoubles;
    if (cudaMemsetAsync(ticket, 0, sizeof(unsigned), st) != cudaSuccess) return -1001;
    long chunk = 0;
    const int nb = trlb::gdot_grid(nrow, kMaxBlocks, &chunk);
    return trlb::launch_gdot<double>(nrow, v1, ld1, m1, v2, ld2, m2, rr, wrk, part, ticket, nb, chunk, st);
}
