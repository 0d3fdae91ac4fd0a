// Allocation-free NW alignment entry point.
//
// Some callers cannot call cudaMalloc at the moment they need an alignment:
// hosts whose device memory is handed out entirely by a framework's pool
// allocator (a cudaMalloc beside the pool fails or fragments it), or
// latency-critical paths that forbid driver allocations.  indialign_nw_align
// allocates its trace scratch on first use; this variant runs the same kernel
// (k_nw_explicit) with its scratch in a fixed file-scope device array
// instead, so it allocates nothing.
//
// The array holds the NW trace, the stripe boundary row, the reversed
// alignment and the kernel's work counters for one problem of at most
// kNoAllocMaxLen x kNoAllocMaxLen (about 1.1 MB, held on every GPU that loads
// this library until the process exits).  All calls share it: two calls whose
// kernels overlap on the GPU race on it.  The kernel zeroes the boundary row
// itself and writes every trace word it later reads, so no state carries over
// from the previous call; the counters are never read.  The first call on a
// device looks up the array's device address (cudaGetSymbolAddress) with
// that device current.  The call returns after `stream` synchronizes.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/indialign_b200.h"
#include "kernels.h"

namespace ia {

constexpr int kNoAllocMaxLen = 2048;
constexpr size_t kNATraceWords = nw_trace_words_for(kNoAllocMaxLen, kNoAllocMaxLen);
constexpr size_t kNABhOff = ((kNATraceWords * 4 + 255) / 256) * 256;
constexpr size_t kNAAlOff = kNABhOff + (((kNoAllocMaxLen + 1) * 8 + 255) / 256) * 256;
constexpr size_t kNACtrOff = kNAAlOff + ((kNoAllocMaxLen * 4 + 255) / 256) * 256;
constexpr size_t kNABytes = kNACtrOff + 256;

static __device__ __align__(256) unsigned char g_nw_scratch[kNABytes];

static std::mutex g_na_mu;
static unsigned char *g_na_ptr[64];  // device address of g_nw_scratch per device

}  // namespace ia

extern "C" int indialign_nw_align_noalloc(const double *d_smat, int np, int nn, double gap,
                                          int *d_ap, int *d_an, int *d_na, void *stream) {
    ia::set_last_error_text("");
    if (!d_smat || !d_ap || !d_an || !d_na) {
        ia::set_last_error_text("nw_align_noalloc: null pointer");
        return INDIALIGN_E_INPUT;
    }
    if (np < 1 || nn < 1 || np > ia::kNoAllocMaxLen || nn > ia::kNoAllocMaxLen) {
        ia::set_last_error_text("nw_align_noalloc: np and nn must be in 1..2048 (fixed scratch size)");
        return INDIALIGN_E_INPUT;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return INDIALIGN_E_NODEVICE;
    unsigned char *base = nullptr;
    {
        // set-up, once per device, with that device current: the array's name
        // is a host-side stand-in, the kernel needs its device address
        std::lock_guard<std::mutex> lk(ia::g_na_mu);
        if (!ia::g_na_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, ia::g_nw_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                ia::set_last_error_text("nw_align_noalloc: cudaGetSymbolAddress of the scratch array failed");
                return INDIALIGN_E_CUDA;
            }
            ia::g_na_ptr[dev] = static_cast<unsigned char *>(p);
        }
        base = ia::g_na_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ia::launch_nw_explicit(d_smat, np, nn, gap, reinterpret_cast<uint32_t *>(base),
                           reinterpret_cast<double *>(base + ia::kNABhOff),
                           reinterpret_cast<uint32_t *>(base + ia::kNAAlOff), d_ap, d_an, d_na,
                           reinterpret_cast<unsigned long long *>(base + ia::kNACtrOff), st);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ia::set_last_error_text(cudaGetErrorString(e));
        return INDIALIGN_E_CUDA;
    }
    return INDIALIGN_OK;
}
