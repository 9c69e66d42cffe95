// Device memory for joins.
//
// Three tiers, chosen so that a steady stream of joins maps no new device memory:
//  * a workspace per (host thread, device) for every temporary of one join: one cudaMalloc'd
//    block used as a stack (blocks freed in reverse order are reclaimed at once, stream order
//    keeps reuse safe because a join issues all its work on one stream).  When a join needs more
//    than the workspace holds, the excess comes from the pool and, once the join has finished,
//    the workspace is re-made at 1.25x the join's need;
//  * a small per-device cache of result buffers: a freed result hands its key buffer back with an
//    event recorded on its stream, and a later join of similar size takes it (waiting on that
//    event on the device, not on the host);
//  * the stream-ordered pool (cudaMallocFromPoolAsync, release threshold max) behind both.
// Allocating large blocks from the pool inside every join cost milliseconds to seconds of host
// time on this hardware whenever the pool re-mapped memory, with the GPU idle meanwhile.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/tensorjoin.h"
#include "tj_internal.h"

namespace tj {

namespace {

constexpr int kMaxDev = 64;

std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxDev] = {};

int current_device() {
    int dev = 0;
    TJ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDev) fail(TJ_ERR_INVALID, "device ordinal out of range");
    return dev;
}

// TJ_TRACE_ALLOC=<ms> in the environment logs, to stderr, every pool allocation whose host call
// took longer than <ms> milliseconds, with the pool's reserved / used bytes afterwards.
double trace_alloc_ms() {
    static const double v = [] {
        const char* e = getenv("TJ_TRACE_ALLOC");
        return e ? atof(e) : -1.0;
    }();
    return v;
}

void* pool_alloc(size_t bytes, cudaStream_t st) {
    void* p = nullptr;
    cudaMemPool_t pool = pool_for_current();
    const double lim = trace_alloc_ms();
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
    if (lim >= 0.0) {
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > lim) {
            uint64_t res = 0, used = 0;
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &res);
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
            fprintf(stderr, "[tj alloc] %zu bytes took %.2f ms (pool reserved %llu MiB, used %llu MiB)\n", bytes, ms,
                    (unsigned long long)(res >> 20), (unsigned long long)(used >> 20));
        }
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(TJ_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    return p;
}

// ---------------------------------------------------------------- per-thread workspace
struct Workspace {
    char* base = nullptr;
    size_t cap = 0;
    size_t top = 0;                               // bytes in use at the top of the stack
    size_t need = 0;                              // the join's high-water mark (workspace + overflow)
    size_t over_live = 0;                         // bytes of live overflow (pool) blocks
    bool active = false;
    int suspended = 0;
    std::vector<std::pair<size_t, bool>> live;    // offsets of live blocks, bottom to top; freed flag
    std::unordered_map<void*, size_t> over;       // overflow blocks -> bytes
};
thread_local Workspace g_ws[kMaxDev];

// ---------------------------------------------------------------- result-buffer cache
struct Cached {
    void* p;
    size_t cap;
    cudaEvent_t ev;   // recorded on the releasing stream when the buffer was given back
};
constexpr size_t kCacheEntries = 4;
constexpr size_t kCacheBytes = (size_t)32 << 30;
std::mutex g_cache_mu;
std::vector<Cached> g_cache[kMaxDev];

}  // namespace

cudaMemPool_t pool_for_current() {
    const int dev = current_device();
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        TJ_CUDA(cudaMemPoolCreate(&g_pools[dev], &props));
        uint64_t thr = ~0ull;
        TJ_CUDA(cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &thr));
    }
    return g_pools[dev];
}

void* dalloc(size_t bytes, cudaStream_t st) {
    Workspace& W = g_ws[current_device()];
    if (W.active && !W.suspended) {
        const size_t sz = (bytes + 255) & ~(size_t)255;
        if (W.top + sz <= W.cap) {
            const size_t o = W.top;
            W.top += sz;
            W.live.push_back({o, false});
            W.need = std::max(W.need, W.top + W.over_live);
            return W.base + o;
        }
        void* p = pool_alloc(sz, st);
        W.over[p] = sz;
        W.over_live += sz;
        W.need = std::max(W.need, W.top + W.over_live);
        return p;
    }
    return pool_alloc(bytes, st);
}

void dfree(void* p, cudaStream_t st) {
    if (!p) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
        cudaGetLastError();
        cudaFreeAsync(p, st);
        return;
    }
    Workspace& W = g_ws[dev];
    char* c = (char*)p;
    if (W.base && c >= W.base && c < W.base + W.cap) {
        const size_t o = (size_t)(c - W.base);
        for (size_t i = W.live.size(); i-- > 0;)
            if (W.live[i].first == o && !W.live[i].second) { W.live[i].second = true; break; }
        while (!W.live.empty() && W.live.back().second) {
            W.top = W.live.back().first;
            W.live.pop_back();
        }
        return;
    }
    auto it = W.over.find(p);
    if (it != W.over.end()) {
        W.over_live -= it->second;
        W.over.erase(it);
    }
    cudaFreeAsync(p, st);
}

WorkspaceScope::WorkspaceScope(cudaStream_t s) : st(s), dev(current_device()) {
    Workspace& W = g_ws[dev];
    if (W.active) fail(TJ_ERR_INVALID, "nested join workspace");
    W.active = true;
    W.suspended = 0;
    W.top = 0;
    W.need = 0;
    W.over_live = 0;
    W.live.clear();
    W.over.clear();
}

WorkspaceScope::~WorkspaceScope() {
    Workspace& W = g_ws[dev];
    W.active = false;
    // a join that failed part-way may still have kernels in flight on workspace memory
    if (std::uncaught_exceptions() > 0 || !W.live.empty()) cudaStreamSynchronize(st);
    W.live.clear();
    W.over.clear();
    W.top = 0;
    W.over_live = 0;
    if (W.need > W.cap) try {
        cudaStreamSynchronize(st);
        if (W.base) cudaFree(W.base);
        W.base = nullptr;
        W.cap = 0;
        const size_t gran = (size_t)64 << 20;
        const size_t cap = ((W.need + W.need / 4 + gran - 1) / gran) * gran;
        void* p = nullptr;
        if (cudaMalloc(&p, cap) != cudaSuccess) {
            // the overflow blocks went back to the pool: hand that idle memory to the driver and try
            // again (only then: a trimmed pool maps its memory anew, which took hundreds of ms)
            cudaGetLastError();
            cudaMemPoolTrimTo(pool_for_current(), 0);
            if (cudaMalloc(&p, cap) != cudaSuccess) p = nullptr;
        }
        if (p) {
            W.base = (char*)p;
            W.cap = cap;
        }
        cudaGetLastError();   // a failed growth leaves the next join on the pool
        if (trace_alloc_ms() >= 0.0)
            fprintf(stderr, "[tj workspace] re-made at %zu MiB for a need of %zu MiB%s\n", cap >> 20, W.need >> 20,
                    p ? "" : " (failed: the next join allocates from the pool)");
    } catch (...) {
        cudaGetLastError();
    }
    W.need = 0;
}

WorkspaceSuspend::WorkspaceSuspend() : dev(current_device()) { g_ws[dev].suspended++; }
WorkspaceSuspend::~WorkspaceSuspend() { g_ws[dev].suspended--; }

size_t workspace_bytes() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
        cudaGetLastError();
        return 0;
    }
    return g_ws[dev].cap;
}

void* result_alloc(size_t bytes, cudaStream_t st, size_t* cap_out) {
    *cap_out = 0;
    if (bytes == 0) return nullptr;
    const int dev = current_device();
    {
        std::unique_lock<std::mutex> lk(g_cache_mu);
        auto& C = g_cache[dev];
        size_t best = C.size();
        for (size_t i = 0; i < C.size(); ++i)
            if (C[i].cap >= bytes && C[i].cap <= 2 * bytes + ((size_t)16 << 20) &&
                (best == C.size() || C[i].cap < C[best].cap))
                best = i;
        if (best < C.size()) {
            const Cached e = C[best];
            C.erase(C.begin() + (long)best);
            lk.unlock();
            TJ_CUDA(cudaStreamWaitEvent(st, e.ev, 0));
            cudaEventDestroy(e.ev);
            *cap_out = e.cap;
            return e.p;
        }
    }
    const size_t gran = (size_t)2 << 20;
    const size_t cap = ((bytes + gran - 1) / gran) * gran;
    WorkspaceSuspend off;   // result buffers outlive the join: never from the workspace
    void* p = pool_alloc(cap, st);
    *cap_out = cap;
    return p;
}

void result_release(void* p, size_t cap, cudaStream_t st) {
    if (!p) return;
    cudaPointerAttributes pa;
    int dev = -1;
    if (cudaPointerGetAttributes(&pa, p) == cudaSuccess) dev = pa.device;
    cudaGetLastError();
    cudaEvent_t ev = nullptr;
    if (dev < 0 || dev >= kMaxDev || cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(ev, st) != cudaSuccess) {
        cudaGetLastError();
        if (ev) cudaEventDestroy(ev);
        cudaFreeAsync(p, st);
        return;
    }
    std::vector<Cached> drop;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        auto& C = g_cache[dev];
        C.push_back({p, cap, ev});
        size_t total = 0;
        for (const auto& e : C) total += e.cap;
        while (C.size() > kCacheEntries || (C.size() > 1 && total > kCacheBytes)) {
            total -= C.front().cap;
            drop.push_back(C.front());
            C.erase(C.begin());
        }
    }
    for (const auto& e : drop) {   // free after the last use recorded in its event
        cudaStreamWaitEvent(st, e.ev, 0);
        cudaFreeAsync(e.p, st);
        cudaEventDestroy(e.ev);
    }
}

void release_cached(cudaStream_t st) {
    const int dev = current_device();
    std::vector<Cached> drop;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        drop.swap(g_cache[dev]);
    }
    for (const auto& e : drop) {
        TJ_CUDA(cudaEventSynchronize(e.ev));
        cudaFreeAsync(e.p, st);
        cudaEventDestroy(e.ev);
    }
    Workspace& W = g_ws[dev];
    if (!W.active && W.base) {
        TJ_CUDA(cudaFree(W.base));
        W.base = nullptr;
        W.cap = 0;
    }
}

}  // namespace tj
