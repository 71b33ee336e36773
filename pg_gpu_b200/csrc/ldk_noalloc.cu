// ldk_parse_noalloc: the binned parse for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc (or any allocator) around a
// parse: a host runtime bound over a foreign-function layer (a JNI, cgo or N-API plugin)
// that owns no device allocator and only receives the input and output buffers from its
// host, or an application whose memory manager forbids allocations outside its own pool.
// For them this entry point takes its scratch from a file-scope device array of
// LDK_NOALLOC_SCRATCH_BYTES instead of a caller workspace.
//
// * The array is part of this library's device image: every GPU that loads it holds
//   the array until the process exits.
// * Host code cannot use the array's name as a device address.  The first call on each
//   device resolves the address (cudaGetSymbolAddress, with that device current) and
//   caches it together with the device's current context; a call that finds another
//   context current (the old one was destroyed, e.g. by cudaDeviceReset, and a new one
//   created) resolves it again.
// * All calls share the one array, which keeps the last call's contents.  Everything
//   that must start at zero (the status word, the row counter, the fixed-point bin
//   accumulators, the outputs) is cleared by each call on its stream; calls that overlap
//   on the GPU (different streams, or host threads without ordering) race on the array
//   and must not be issued.
// * A parse whose scratch need exceeds the array fails with LDK_ERR_UNSUPPORTED and a
//   message giving both sizes; nothing is allocated to make it fit.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "ldk_internal.h"

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[LDK_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};

// The calling thread's current driver context (null if none or the query is unavailable).
CUcontext current_context() {
    static PFN_cuCtxGetCurrent_v4000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
    });
    CUcontext ctx = nullptr;
    if (fn && fn(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    return ctx;
}

}  // namespace

extern "C" int ldk_parse_noalloc(const ldk_parse_t* d, const ldk_parse_out_t* out, void* stream) {
    using ldk::set_error;
    const size_t need = ldk_parse_workspace_size(d);
    if (need == 0) return ldk::parse_impl(d, out, nullptr, 0, stream, true);  // reports the invalid argument
    if (need > (size_t)LDK_NOALLOC_SCRATCH_BYTES) {
        set_error("ldk_parse_noalloc: this parse needs %zu bytes of scratch but the static array holds %zu; "
                  "use ldk_parse with a caller workspace",
                  need, (size_t)LDK_NOALLOC_SCRATCH_BYTES);
        return LDK_ERR_UNSUPPORTED;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_error("ldk_parse_noalloc: no usable CUDA device");
        return LDK_ERR_CUDA;
    }
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        // cudaGetSymbolAddress makes the device's primary context current if none is, so the
        // context is read after it
        if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != current_context()) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                set_error("ldk_parse_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return LDK_ERR_CUDA;
            }
            g_scratch_addr[dev] = p;
            g_scratch_ctx[dev] = current_context();
        }
        scratch = g_scratch_addr[dev];
    }
    return ldk::parse_impl(d, out, scratch, (size_t)LDK_NOALLOC_SCRATCH_BYTES, stream, true);
}
