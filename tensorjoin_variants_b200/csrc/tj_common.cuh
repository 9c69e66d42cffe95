// Shared device/host helpers for the B200 certified exact epsilon-join.
// sm_100a only: tcgen05 (UMMA + TMEM), TMA bulk tensor copies, mbarriers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#define TJ_DEV __device__ __forceinline__

namespace tj {

// ---------------------------------------------------------------- constants
constexpr int kWarp = 32;
constexpr int kTileR = 128;     // R-side tile rows (UMMA M)
constexpr int kTileS = 256;     // S-side tile rows (UMMA N)
constexpr int kBK = 64;         // 16-bit elements per k-block = one 128-byte swizzle row (widest)
constexpr uint64_t kSentinel = ~0ull;

// Device status word bits (written with atomicOr, read by the host once per join).
enum : unsigned {
    kStatusWaitTimeout = 1u << 0,   // a bounded mbarrier wait gave up
    kStatusBadInput = 1u << 1,      // NaN / Inf / out-of-range magnitude in an input row
    kStatusTmemAlloc = 1u << 2,     // TMEM allocation returned an unexpected address
    kStatusFp16Range = 1u << 3,     // |x| too large for an FP16 operand
    kStatusGuard = 1u << 4,         // a guard region after an output buffer was overwritten
};

// Counters block shared by the screen, refine and emit stages (device memory, u64 each).  The first
// kCountersPerAttempt words restart with every screen attempt (capacity retries rerun the screen).
struct Counters {
    unsigned long long acc_reserved;   // slots reserved in the accept buffer (incl. sentinel padding)
    unsigned long long acc_valid;      // accepted pairs written (screen + refine)
    unsigned long long band_reserved;  // slots reserved in the band buffer
    unsigned long long band_valid;     // band pairs written
    unsigned long long screen_accept;  // accepted directly by the certified screen
    unsigned long long refine_accept;  // accepted by FP64 refinement
    unsigned long long rare_checks;    // pairs that reached the per-pair FP64 certificate
    unsigned long long items;          // tile pairs screened
    unsigned long long band_fp64;      // band pairs that reached the FP64 terminal
    unsigned long long xl_items;       // int8 four-product screen: items that took the low-limb products
    unsigned long long status;         // kStatus* bits
    unsigned long long pairs_screened; // distance evaluations of the candidate list
    unsigned long long screen_ops;     // algorithmic screen operations of the candidate list
    unsigned long long class_items[4]; // candidate tile pairs per class
    unsigned long long screen_reserved;  // acc_reserved after the screen, before the refinement appends
    unsigned long long chunk_next;       // work queue of the one-SM screen: chunks taken beyond the first wave
    unsigned long long pad[1];
};
constexpr int kCountersPerAttempt = 10;

// Per-join parameters (batched mode has one per join; a single join uses one entry).
struct JoinParams {
    double T;            // threshold on squared distance
    double Tm;           // certified-in bound:  D <= Tm  =>  fp64 oracle value <= T
    double Tp;           // certified-out bound: D >  Tp  =>  fp64 oracle value >  T
    double gn;           // relative error bound of the FP64 norms
    double gmma;         // tensor-core accumulation premise coefficient
    double cabs;         // absolute underflow allowance of the accumulation
    unsigned long long key_off;   // offset added to i * n_cols + j (batched: prefix of |R||S|)
    long long n_rows;    // |R| (self: N)
    long long n_cols;    // |S| (self: N)
    int self_join;       // 1: R == S, emit each unordered pair once (i < j)
    int d;               // dimensions
    int pad[2];
};

// ---------------------------------------------------------------- small helpers
TJ_DEV unsigned lane_id() { unsigned r; asm volatile("mov.u32 %0, %%laneid;" : "=r"(r)); return r; }
TJ_DEV unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

TJ_DEV float f32_up(double x) { float r; asm("cvt.rp.f32.f64 %0, %1;" : "=f"(r) : "d"(x)); return r; }
TJ_DEV float f32_dn(double x) { float r; asm("cvt.rm.f32.f64 %0, %1;" : "=f"(r) : "d"(x)); return r; }

// v0 = fma(-2, p0, c0), v1 = fma(-2, p1, c1) as one packed FP32x2 FMA (sm_100), each lane rounded
// exactly as the scalar fmaf.
TJ_DEV void fma_m2_x2(float p0, float p1, float c0, float c1, float& v0, float& v1) {
    asm("{\n\t.reg .b64 a, c, m, r;\n\t"
        "mov.b64 a, {%2, %3};\n\t"
        "mov.b64 c, {%4, %5};\n\t"
        "mov.b64 m, {%6, %6};\n\t"
        "fma.rn.f32x2 r, a, m, c;\n\t"
        "mov.b64 {%0, %1}, r;\n\t}"
        : "=f"(v0), "=f"(v1) : "f"(p0), "f"(p1), "f"(c0), "f"(c1), "f"(-2.0f));
}
// Position of the j-th (0-based) set bit of w (w has more than j set bits): a binary search on the
// popcounts of the low halves.
TJ_DEV int nth_set_bit(uint32_t w, unsigned j) {
    int pos = 0;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const unsigned c = __popc(w & ((1u << s) - 1u));
        if (j >= c) {
            j -= c;
            w >>= s;
            pos += s;
        }
    }
    return pos;
}
// min of three floats in one instruction (sm_100); a NaN operand is ignored, as by fminf.
TJ_DEV float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

TJ_DEV float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// exclusive warp prefix sum of v (all 32 lanes participate)
TJ_DEV unsigned warp_excl_scan(unsigned v, unsigned& total) {
    unsigned x = v;
    const unsigned lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// ---------------------------------------------------------------- mbarrier (bounded waits)
TJ_DEV void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
TJ_DEV void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
TJ_DEV void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

TJ_DEV void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
TJ_DEV void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}
// `count` arrivals at once
TJ_DEV void mbar_arrive_cnt(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
TJ_DEV bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
TJ_DEV unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after `limit_ns` of wall time, sets the timeout bit and returns false.
// Every wait in every kernel of this library goes through here, so no kernel can spin forever.
// Limits of a millisecond or more first spin 256 times without reading the clock; shorter limits
// (set through tj_set_wait_limit, for tests of the timeout path) start the clock at once.
constexpr unsigned long long kWaitLimitNs = 4000000000ull;   // 4 s
constexpr unsigned long long kDrainLimitNs = 1000000000ull;  // waits for a CTA's own copies in flight
TJ_DEV bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long* status,
                      unsigned long long limit_ns = kWaitLimitNs) {
    const int spins = limit_ns >= 1000000ull ? 256 : 1;
    for (int it = 0; it < spins; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(64);
        if (global_ns() - t0 > limit_ns) break;
    }
    atomicOr(status, (unsigned long long)kStatusWaitTimeout);
    return false;
}

// ---------------------------------------------------------------- TMA
TJ_DEV void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        :: "r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y) : "memory");
}
// Contiguous global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16),
// completing on an mbarrier transaction count.
TJ_DEV void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        :: "r"(smem_u32(dst)), "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// 16-byte global -> shared copy issued by one thread (both addresses 16-byte aligned), bypassing L1;
// copies are grouped by commit and waited for by group count.
TJ_DEV void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_u32(dst)), "l"((uint64_t)src) : "memory");
}
TJ_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int kPending>
TJ_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(kPending) : "memory"); }
TJ_DEV void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" :: "l"((uint64_t)map) : "memory");
}

// ---------------------------------------------------------------- tcgen05 (UMMA + TMEM)
TJ_DEV void tmem_alloc(unsigned* dst_smem, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
TJ_DEV void tmem_dealloc(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
TJ_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
TJ_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (FP16 or BF16 inputs, FP32 accumulate)
TJ_DEV void umma_f16(unsigned d_tmem, uint64_t adesc, uint64_t bdesc, unsigned idesc, unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}
// D[tmem] (+)= A * B^T, kind::i8 (signed 8-bit inputs, exact INT32 accumulate)
TJ_DEV void umma_i8(unsigned d_tmem, uint64_t adesc, uint64_t bdesc, unsigned idesc, unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}
// Arrive on an mbarrier once all previously issued tcgen05.mma of this thread have completed.
TJ_DEV void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

// ---------------------------------------------------------------- CTA pairs (cta_group::2)
TJ_DEV unsigned cluster_ctarank() { unsigned r; asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r)); return r; }
// all threads of both CTAs of the cluster (release / acquire at cluster scope)
TJ_DEV void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// shared::cluster address of the same shared variable in CTA `rank` of the cluster
TJ_DEV unsigned mapa_shared(const void* p, unsigned rank) {
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}
// arrive on an mbarrier of (possibly) another CTA of the cluster, releasing at cluster scope
TJ_DEV void mbar_arrive_cluster(unsigned bar_cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" :: "r"(bar_cluster_addr) : "memory");
}
TJ_DEV bool mbar_try_wait_cluster(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait with cluster-scope acquire (a barrier that the other CTA of the pair arrives on)
TJ_DEV bool mbar_wait_cluster(uint64_t* bar, unsigned parity, unsigned long long* status,
                              unsigned long long limit_ns = kWaitLimitNs) {
    const int spins = limit_ns >= 1000000ull ? 256 : 1;
    for (int it = 0; it < spins; ++it)
        if (mbar_try_wait_cluster(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try_wait_cluster(bar, parity)) return true;
        __nanosleep(64);
        if (global_ns() - t0 > limit_ns) break;
    }
    atomicOr(status, (unsigned long long)kStatusWaitTimeout);
    return false;
}
// TMA tile load into this CTA's shared memory whose completion is counted on an mbarrier of
// either CTA of the pair (cta_group::2); no multicast.
TJ_DEV void tma_load_2d_pair(void* dst, const CUtensorMap* map, unsigned bar_cluster_addr, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];"
        :: "r"(smem_u32(dst)), "l"((uint64_t)map), "r"(bar_cluster_addr), "r"(x), "r"(y) : "memory");
}
TJ_DEV void tmem_alloc_pair(unsigned* dst_smem, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
TJ_DEV void tmem_dealloc_pair(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
// D (both CTAs' TMEM) (+)= A (M = 256: 128 rows from each CTA) * B^T (N columns, half from each CTA)
TJ_DEV void umma_f16_pair(unsigned d_tmem, uint64_t adesc, uint64_t bdesc, unsigned idesc, unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}
// arrive once, on completion of this thread's prior pair MMAs, on the mbarrier at this offset in
// every CTA of `cta_mask`
TJ_DEV void umma_commit_pair_mc(uint64_t* bar, uint16_t cta_mask) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
                 :: "r"(smem_u32(bar)), "h"(cta_mask) : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns; thread t receives lane (base_lane + t).
TJ_DEV void tmem_ld32(unsigned taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr) : "memory");
}
TJ_DEV void tmem_ld8(unsigned taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr) : "memory");
}
TJ_DEV void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
TJ_DEV void tmem_ld16(unsigned taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr) : "memory");
}
// Wait for the outstanding TMEM loads, with the registers of one of them as operands: their uses
// cannot be scheduled above the wait (a load whose registers are still in flight may be issued
// before other work, and waited for after it).
TJ_DEV void tmem_wait16(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :: "memory");
}

// UMMA shared-memory descriptor: K-major operand in the 128-byte swizzle canonical layout
// (8-row x 128-byte atoms, atoms stacked every 1024 bytes), as written by a TMA box of
// 128-byte rows with CU_TENSOR_MAP_SWIZZLE_128B.  Base must be 1024-byte aligned;
// stepping K inside the atom adds the byte offset to the start address field.
TJ_DEV uint64_t desc_sw128(const void* smem_base, unsigned byte_off) {
    const unsigned a = smem_u32(smem_base) + byte_off;
    uint64_t d = 0;
    d |= (uint64_t)((a >> 4) & 0x3FFFu);          // start address >> 4
    d |= (uint64_t)1u << 16;                        // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;              // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1u << 46;                        // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                        // layout: SWIZZLE_128B
    return d;
}

// The same descriptor for a K-major operand whose rows are `row_bytes` = 32, 64 or 128 bytes
// (16, 32 or 64 16-bit elements), written by a TMA box of that width with the matching
// CU_TENSOR_MAP_SWIZZLE_32B / 64B / 128B mode: atoms of 8 rows, stride byte offset 8 * row_bytes,
// layout code 6 / 4 / 2.  The constant upper half is computed once on the host (desc_hi).
__host__ __device__ constexpr uint32_t desc_hi_for_rows(unsigned row_bytes) {
    return ((8u * row_bytes) >> 4) | (1u << 14) |
           ((row_bytes == 32u ? 6u : row_bytes == 64u ? 4u : 2u) << 29);
}
TJ_DEV uint64_t desc_kmajor(const void* smem_base, unsigned byte_off, uint32_t desc_hi) {
    const unsigned a = smem_u32(smem_base) + byte_off;
    return ((uint64_t)desc_hi << 32) | (uint64_t)(1u << 16) | (uint64_t)((a >> 4) & 0x3FFFu);
}

// UMMA instruction descriptor (kind::f16 / kind::i8, dense, K-major A and B).
// a/b format: f16 = 0, bf16 = 1 (kind::f16); u8 = 0, s8 = 1 (kind::i8).  c format: f32 = 1, s32 = 2.
__host__ __device__ constexpr unsigned make_idesc(unsigned c_fmt, unsigned ab_fmt, unsigned M, unsigned N) {
    return (c_fmt << 4) | (ab_fmt << 7) | (ab_fmt << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

}  // namespace tj
