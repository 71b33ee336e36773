// ldk_parse_noalloc: the binned parse for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc (or any allocator) around a
// parse: code that runs while a CUDA graph is being captured on its stream, or a host
// runtime bound over a foreign-function layer (a JNI, cgo or N-API plugin) that owns
// no device allocator and only receives the input and output buffers from its host.
// For them this entry point takes its scratch from a file-scope device array of
// LDK_NOALLOC_SCRATCH_BYTES instead of a caller workspace.
//
// * The array is part of this library's device image: every GPU that loads it holds
//   the array until the process exits.
// * The first call on each device resolves the array's device address
//   (cudaGetSymbolAddress, with that device current) and caches it; make that first
//   call before any stream capture begins.
// * All calls share the one array, which keeps the last call's contents.  Everything
//   that must start at zero (the status word, the row counter, the outputs) is cleared
//   by each call on its stream; calls that overlap on the GPU (different streams, or
//   host threads without ordering) race on the array and must not be issued.
// * A parse whose scratch need exceeds the array fails with LDK_ERR_UNSUPPORTED and a
//   message giving both sizes; nothing is allocated to make it fit.
#include <mutex>

#include "ldk_internal.h"

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[LDK_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

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
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                set_error("ldk_parse_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return LDK_ERR_CUDA;
            }
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    return ldk::parse_impl(d, out, scratch, (size_t)LDK_NOALLOC_SCRATCH_BYTES, stream, true);
}
