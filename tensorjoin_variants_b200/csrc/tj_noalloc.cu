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
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that first
//    call before any stream capture on that device.
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

std::mutex g_mu;
void* g_addr[64] = {};

void* scratch_for_current_device() {
    int dev = 0;
    TJ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(TJ_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            fail(TJ_ERR_CUDA, std::string("cudaGetSymbolAddress of the sort scratch failed: ") +
                                  cudaGetErrorString(e));
        }
        g_addr[dev] = p;
    }
    return g_addr[dev];
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
        cudaStream_t st = (cudaStream_t)stream;
        unsigned char* base = (unsigned char*)scratch_for_current_device();
        if (n == 0) return TJ_OK;
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
