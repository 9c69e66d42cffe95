// Allocation-free variant of the canonical-key radix sort.
//
// Some callers cannot allocate device memory at the point where they need the
// pairs put in canonical order: an engine that hands this library a fixed,
// preallocated arena and owns every other byte of HBM, a host thread that runs
// under a memory budget enforced by another framework's caching allocator, or a
// loop that must not take the latency of an allocation between two launches.
// tj_sort_keys_noalloc serves them.  The caller passes only the input and the
// output arrays; the sort's scratch (the ping-pong key buffer, the digit
// histograms, the scan workspace) is a file-scope device array of fixed size,
// so no call reaches cudaMalloc, cudaMallocAsync, cudaFree or any allocating
// library routine.
//
// Limits and sharing:
//  * at most kNoAllocMaxKeys keys per call; larger inputs are rejected;
//  * every GPU that loads this library keeps the array (about 9 MiB) until the
//    process exits;
//  * all calls on a device share the one array, so calls that overlap on the GPU
//    (different streams, or different host threads) race on it and corrupt each
//    other -- serialise them;
//  * the array keeps the last call's contents.  Every scratch word a call reads was
//    written earlier in the same call (each pass rewrites the whole histogram and
//    scan table), so nothing has to be cleared between calls;
//  * the first call in a CUDA context looks up the array's device address with
//    cudaGetSymbolAddress (with that context current) and caches it per context, so a
//    new context (after cudaDeviceReset, or a driver-API context) resolves its own
//    address; make the first non-empty call in a context before any stream capture;
//  * keys_in and keys_out must be the same array or not overlap at all.
#include <mutex>

#include "../../include/tensorjoin.h"
#include "tj_internal.h"

namespace tj {
namespace {

constexpr long long kNoAllocMaxKeys = 1ll << 20;   // 1,048,576 keys
constexpr size_t kTmpBytes = (size_t)kNoAllocMaxKeys * sizeof(uint64_t);
constexpr size_t kScratchBytes = kTmpBytes + ((size_t)1 << 20);   // + 1 MiB for histograms and scan workspace

// In host code this name is a host-side stand-in, not a device address: only the
// address returned by cudaGetSymbolAddress may be handed to a kernel.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

CUcontext current_context() {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        TJ_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) fail(TJ_ERR_CUDA, "cuCtxGetCurrent not available");
        fn = (CtxGetCurrentFn)p;
    }
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS) fail(TJ_ERR_CUDA, "cuCtxGetCurrent failed");
    return c;   // null when no runtime call has made a context current on this thread yet
}

void* symbol_address() {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        fail(TJ_ERR_CUDA, std::string("cudaGetSymbolAddress of the sort scratch failed: ") + cudaGetErrorString(e));
    }
    return p;
}

// The scratch array's device address, per CUDA context (a symbol's address belongs to the context
// the module was loaded in).
std::mutex g_mu;
struct Entry {
    CUcontext ctx;
    void* addr;
};
Entry g_addr[64] = {};
int g_n = 0;

void* scratch_for_current_context() {
    std::lock_guard<std::mutex> lk(g_mu);
    CUcontext ctx = current_context();
    if (!ctx) {   // the symbol lookup initialises the device's primary context and makes it current
        void* p = symbol_address();
        ctx = current_context();
        if (!ctx) fail(TJ_ERR_CUDA, "no current CUDA context");
        if (g_n == 64) g_n = 0;
        g_addr[g_n++] = Entry{ctx, p};
        return p;
    }
    for (int i = 0; i < g_n; ++i)
        if (g_addr[i].ctx == ctx) return g_addr[i].addr;
    void* p = symbol_address();
    if (g_n == 64) g_n = 0;   // a process that made 64 contexts: start the cache over
    g_addr[g_n++] = Entry{ctx, p};
    return p;
}

}  // namespace
}  // namespace tj

using namespace tj;

extern "C" int tj_sort_keys_noalloc(const uint64_t* keys_in, uint64_t* keys_out, int64_t n, int32_t key_bits,
                                    void* stream) {
    try {
        if (n < 0) fail(TJ_ERR_INVALID, "n must be >= 0");
        if (n > kNoAllocMaxKeys)
            fail(TJ_ERR_INVALID, "n = " + std::to_string(n) + " exceeds the allocation-free sort's maximum of " +
                                     std::to_string(kNoAllocMaxKeys) + " keys");
        if (key_bits < 1 || key_bits > 64) fail(TJ_ERR_INVALID, "key_bits must be in [1, 64]");
        if (n > 0 && (!keys_in || !keys_out)) fail(TJ_ERR_INVALID, "null key pointer");
        if (n == 0) return TJ_OK;
        const uintptr_t a0 = (uintptr_t)keys_in, b0 = (uintptr_t)keys_out, len = (uintptr_t)n * sizeof(uint64_t);
        if (a0 != b0 && a0 < b0 + len && b0 < a0 + len)
            fail(TJ_ERR_INVALID, "keys_in and keys_out overlap without being the same array");
        cudaStream_t st = (cudaStream_t)stream;
        unsigned char* base = (unsigned char*)scratch_for_current_context();
        static_assert(kScratchBytes >= kTmpBytes, "scratch layout");
        const size_t ws_elems = radix_workspace_elems((size_t)n);
        if (ws_elems * sizeof(uint32_t) > kScratchBytes - kTmpBytes) fail(TJ_ERR_INVALID, "scratch layout too small");
        uint64_t* tmp = (uint64_t*)base;
        uint32_t* ws = (uint32_t*)(base + kTmpBytes);
        if (keys_out != keys_in)
            TJ_CUDA(cudaMemcpyAsync(keys_out, keys_in, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
        radix_sort(keys_out, nullptr, tmp, nullptr, (size_t)n, key_bits, ws, st);
        TJ_CUDA(cudaGetLastError());
        return TJ_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (...) {
        set_last_error("unknown error");
        return TJ_ERR_INVALID;
    }
}
