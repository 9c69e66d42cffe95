// Device exclusive scan and LSD radix sort, written for this library.
//
// Radix sort: 8-bit digits, least significant first, only the low `bits` bits
// of each key are considered (bit width trimmed to the key range, as the
// output stage trims it to ceil(log2(max key + 2))).  Each pass is
//   1. per-block digit histogram (digit-major [256][blocks]),
//   2. device-wide exclusive scan of that table,
//   3. stable scatter: every warp ranks its keys round by round (the lanes sharing a
//      digit found by eight ballots), warps are combined in order through shared counters,
//      the tile is regrouped by digit in shared memory and written out in runs.
// Stability across passes makes the whole sort correct for any bit width.
//
// It replaces the CUB SortKeys call of the reference's output stage
// (tensorjoin_20260908_output_audit/src/output.cu:26-31).
#include "tj_internal.h"

namespace tj {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of kScanTile u32 values; writes block totals.
__global__ void __launch_bounds__(kScanThreads) scan_tiles(const uint32_t* in, uint32_t* out, size_t n,
                                                           uint32_t* sums) {
    __shared__ uint32_t warp_tot[32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        local += v[k];
    }
    unsigned tot;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned pre = warp_excl_scan(local, tot);
    if (lane == 0) warp_tot[warp] = tot;
    __syncthreads();
    if (warp == 0) {
        unsigned wt = warp_tot[lane], all;
        unsigned wp = warp_excl_scan(wt, all);
        warp_tot[lane] = wp;
        if (lane == 0 && sums) sums[blockIdx.x] = all;
    }
    __syncthreads();
    uint32_t run = pre + warp_tot[warp];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

__global__ void add_block_offsets(uint32_t* out, size_t n, const uint32_t* offs) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / kScanTile];
}

__global__ void write_total(const uint32_t* in_last, const uint32_t* out_last, uint32_t* total) {
    *total = *in_last + *out_last;
}

}  // namespace

size_t scan_workspace_elems(size_t n) {
    size_t total = 0;
    while (n > 1) {
        n = (n + kScanTile - 1) / kScanTile;
        total += n + 1;
    }
    return total + 1;
}

// out[i] = sum_{k<i} in[k]; optional *total = sum of all (device pointer).
// `ws` needs scan_workspace_elems(n) u32 elements.  `in` and `out` may alias.
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total, uint32_t* ws,
                        cudaStream_t st) {
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
        return;
    }
    const size_t nb = (n + kScanTile - 1) / kScanTile;
    // keep a copy of the last input element when aliasing in/out, for the total
    uint32_t* last_copy = ws;  // 1 element
    uint32_t* sums = ws + 1;
    if (total) cudaMemcpyAsync(last_copy, in + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    launch(scan_tiles, (unsigned)nb, kScanThreads, 0, st, in, out, n, nb > 1 ? sums : nullptr);
    if (nb > 1) {
        exclusive_scan_u32(sums, sums, nb, nullptr, sums + nb, st);
        launch(add_block_offsets, (unsigned)((n + 255) / 256), 256, 0, st, out, n, sums);
    }
    if (total) launch(write_total, 1, 1, 0, st, last_copy, out + (n - 1), total);
}

// ------------------------------------------------------------------ radix sort
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsRounds = 16;                         // keys per thread
constexpr int kRsTile = kRsThreads * kRsRounds;       // 4096 keys per block

TJ_DEV unsigned digit_of(uint64_t k, int shift) { return (unsigned)(k >> shift) & 0xFFu; }

// Lanes of the warp (among `valid`) whose 8-bit digit equals this lane's, from eight ballots: a
// peer agrees with the lane on every bit.  Every lane of the warp calls it.  Ballots and logic ops
// run at full rate, where a match instruction over 32 arbitrary values does not.
TJ_DEV unsigned digit_peers(unsigned dg, unsigned valid) {
    unsigned peers = valid;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const unsigned m = __ballot_sync(0xffffffffu, (dg >> b) & 1u);
        peers &= ((dg >> b) & 1u) ? m : ~m;
    }
    return peers;
}
// The same with each step as one three-input logic op (the single-sweep scatter).
TJ_DEV unsigned digit_peers_lop3(unsigned dg, unsigned valid) {
    unsigned peers = valid;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const unsigned bit = (dg >> b) & 1u;
        const unsigned m = __ballot_sync(0xffffffffu, bit);
        const unsigned ext = 0u - bit;   // all ones where the lane's bit is set
        // peers &= ~(m ^ ext): the lanes whose bit b equals this lane's, in one three-input logic op
        asm("lop3.b32 %0, %1, %2, %3, 0x90;" : "=r"(peers) : "r"(peers), "r"(m), "r"(ext));
    }
    return peers;
}

// Byte kByte of a key (a compile-time digit position: a constant shift and mask).
template <int kByte>
TJ_DEV unsigned key_byte(uint64_t k) {
    const uint32_t w = kByte < 4 ? (uint32_t)k : (uint32_t)(k >> 32);
    return (w >> (8 * (kByte & 3))) & 0xFFu;
}

__global__ void __launch_bounds__(kRsThreads) rs_hist(const uint64_t* keys, size_t n, int shift, uint32_t* hist,
                                                     unsigned nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kRsTile;
    unsigned dg[kRsRounds];   // all loads in flight before the shared-memory counting
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
        const size_t i = base + (size_t)r * kRsThreads + threadIdx.x;
        dg[r] = i < n ? digit_of(keys[i], shift) : 256u;
    }
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r)
        if (dg[r] < 256u) atomicAdd(&h[dg[r]], 1u);
    __syncthreads();
    hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// The scatter runs 512 threads over the same 4096-key tile (8 keys per thread): twice the warps
// of the histogram kernel, to hide the latency of its load, rank and regroup phases.
constexpr int kScThreads = 512;
constexpr int kScWarps = kScThreads / 32;
constexpr int kScRounds = kRsTile / kScThreads;       // 8 keys per thread

// Block-wide exclusive scan of one value per thread over kWarps warps (every thread calls it).
template <int kWarps>
TJ_DEV uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tot) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned tot;
    const unsigned pre = warp_excl_scan(v, tot);
    if (lane == 0) warp_tot[warp] = tot;
    __syncthreads();
    uint32_t off = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) off += (w < (int)warp) ? warp_tot[w] : 0u;
    return off + pre;
}

// Stable scatter of one 4096-key tile.  Keys are ranked per warp (round by round with
// ballots), the block's keys are regrouped by digit in shared memory, and then written
// out in that order, so consecutive threads store consecutive addresses of one digit's run
// (about 16 keys = 128 B per digit and tile for 8-bit digits) instead of scattered 8-byte words.
template <bool kVals>
__global__ void __launch_bounds__(kScThreads, kVals ? 2 : 3) rs_scatter(const uint64_t* keys_in, const uint32_t* vals_in,
                                                        uint64_t* keys_out, uint32_t* vals_out, size_t n, int shift,
                                                        const uint32_t* offs, unsigned nblocks) {
    extern __shared__ __align__(16) unsigned char rs_dyn[];
    uint64_t* sk = (uint64_t*)rs_dyn;                      // [kRsTile] keys grouped by digit
    uint32_t* sv = (uint32_t*)(rs_dyn + kRsTile * 8);      // [kRsTile] values (kVals)
    __shared__ uint32_t wcnt[kScWarps][256];   // per warp and digit: count, then tile-local start
    __shared__ uint32_t gdelta[256];   // global start minus tile-local start of each digit's run (mod 2^32)
    __shared__ uint32_t wtot[kScWarps];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kScWarps * 256; i += kScThreads) (&wcnt[0][0])[i] = 0;
    const uint32_t gbase = threadIdx.x < 256 ? offs[(size_t)threadIdx.x * nblocks + blockIdx.x] : 0u;
    __syncthreads();

    // warp w owns the contiguous run [w*256, (w+1)*256) of this block's tile; round r, lane l -> r*32 + l
    const size_t tbase = (size_t)blockIdx.x * kRsTile;
    const size_t wbase = tbase + (size_t)warp * (kScRounds * 32);
    uint64_t k[kScRounds];
    uint32_t v[kScRounds];
    uint32_t rank[kScRounds];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kScRounds; ++r) {
        const size_t i = wbase + (size_t)r * 32 + lane;
        k[r] = i < n ? keys_in[i] : 0ull;
    }
#pragma unroll
    for (int r = 0; r < kScRounds; ++r) {
        const bool ok = wbase + (size_t)r * 32 + lane < n;
        const unsigned valid = __ballot_sync(0xffffffffu, ok);
        const unsigned dg = digit_of(k[r], shift);
        const unsigned peers = digit_peers(dg, valid);
        const unsigned prev = ok ? wcnt[warp][dg] : 0u;
        rank[r] = ok ? prev + __popc(peers & lt) : 0xFFFFFFFFu;
        __syncwarp();
        if (ok && (peers & lt) == 0) wcnt[warp][dg] = prev + __popc(peers);
        __syncwarp();
    }
    if (kVals) {   // values load while the block meets at the barrier (fewer live registers above)
#pragma unroll
        for (int r = 0; r < kScRounds; ++r) {
            const size_t i = wbase + (size_t)r * 32 + lane;
            v[r] = i < n ? vals_in[i] : 0u;
        }
    }
    __syncthreads();
    {   // per digit (threads 0..255): total over warps, tile-local start by a block scan, then each
        // warp's start of that digit's run (one shared read per key in the regroup below)
        const unsigned dg = threadIdx.x;
        uint32_t run = 0;
        if (dg < 256) {
#pragma unroll
            for (int w = 0; w < kScWarps; ++w) run += wcnt[w][dg];
        }
        const uint32_t ls = block_excl_scan<kScWarps>(run, wtot);
        if (dg < 256) {
            uint32_t at = ls;
#pragma unroll
            for (int w = 0; w < kScWarps; ++w) {
                const uint32_t t = wcnt[w][dg];
                wcnt[w][dg] = at;
                at += t;
            }
            gdelta[dg] = gbase - ls;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kScRounds; ++r) {
        if (rank[r] != 0xFFFFFFFFu) {
            const unsigned p = wcnt[warp][digit_of(k[r], shift)] + rank[r];
            sk[p] = k[r];
            if (kVals) sv[p] = v[r];
        }
    }
    __syncthreads();
    const unsigned cnt = (unsigned)min((size_t)kRsTile, n - tbase);
    for (unsigned p = threadIdx.x; p < cnt; p += kScThreads) {
        const uint64_t key = sk[p];
        const size_t pos = (size_t)(uint32_t)(gdelta[digit_of(key, shift)] + p);
        keys_out[pos] = key;
        if (kVals) vals_out[pos] = sv[p];
    }
}

// Whole sort of a small array (n <= kSmallSort) in one CTA: per pass a histogram of all keys and
// its scan give each digit's start, then the 4096-key chunks are ranked in order exactly as in
// rs_scatter (16 warps, ballot ranking) and written to their final positions; the running digit
// starts carry stability across chunks.  Keys ping-pong through global memory (L2-resident at this
// size); __syncthreads orders each pass's writes before the next pass's reads within the block.
// One launch replaces the four to five launches per pass of the multi-block path.
constexpr unsigned kSmallSort = 16384;

template <bool kVals>
__global__ void __launch_bounds__(kScThreads) rs_small(uint64_t* keys, uint32_t* vals, uint64_t* ktmp,
                                                      uint32_t* vtmp, unsigned n, int passes) {
    __shared__ uint32_t wcnt[kScWarps][256];
    __shared__ uint32_t base[256];     // this pass: next output position of each digit
    __shared__ uint32_t wtot[kScWarps];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, t = threadIdx.x;
    const unsigned lt = (1u << lane) - 1u;
    uint64_t *kin = keys, *kout = ktmp;
    uint32_t *vin = vals, *vout = vtmp;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = 8 * pass;
        if (t < 256) base[t] = 0;
        __syncthreads();
        for (unsigned i = t; i < n; i += kScThreads) atomicAdd(&base[digit_of(kin[i], shift)], 1u);
        __syncthreads();
        const uint32_t cnt = t < 256 ? base[t] : 0u;
        const uint32_t ex = block_excl_scan<kScWarps>(cnt, wtot);
        __syncthreads();                       // every thread has read base[] for its count
        if (t < 256) base[t] = ex;
        for (unsigned c0 = 0; c0 < n; c0 += kRsTile) {
            for (int i = t; i < kScWarps * 256; i += kScThreads) (&wcnt[0][0])[i] = 0;
            __syncthreads();
            const unsigned wbase = c0 + warp * (kScRounds * 32);
            uint64_t k[kScRounds];
            uint32_t rank[kScRounds];
#pragma unroll
            for (int r = 0; r < kScRounds; ++r) {
                const unsigned i = wbase + r * 32 + lane;
                k[r] = i < n ? kin[i] : 0ull;
            }
#pragma unroll
            for (int r = 0; r < kScRounds; ++r) {
                const bool ok = wbase + r * 32 + lane < n;
                const unsigned valid = __ballot_sync(0xffffffffu, ok);
                const unsigned dg = digit_of(k[r], shift);
                const unsigned peers = digit_peers(dg, valid);
                const unsigned prev = ok ? wcnt[warp][dg] : 0u;
                rank[r] = ok ? prev + __popc(peers & lt) : 0xFFFFFFFFu;
                __syncwarp();
                if (ok && (peers & lt) == 0) wcnt[warp][dg] = prev + __popc(peers);
                __syncwarp();
            }
            __syncthreads();
            if (t < 256) {   // each warp's start of digit t in this chunk; advance the digit's start
                uint32_t at = base[t];
#pragma unroll
                for (int w = 0; w < kScWarps; ++w) {
                    const uint32_t c = wcnt[w][t];
                    wcnt[w][t] = at;
                    at += c;
                }
                base[t] = at;
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < kScRounds; ++r) {
                if (rank[r] != 0xFFFFFFFFu) {
                    const unsigned i = wbase + r * 32 + lane;
                    const unsigned pos = wcnt[warp][digit_of(k[r], shift)] + rank[r];
                    kout[pos] = k[r];
                    if (kVals) vout[pos] = vin[i];
                }
            }
            __syncthreads();   // wcnt is reused by the next chunk
        }
        uint64_t* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
        __syncthreads();       // this pass's writes are read by the next pass
    }
    if (kin != keys) {         // odd number of passes: the result is in the temporaries
        for (unsigned i = t; i < n; i += kScThreads) {
            keys[i] = kin[i];
            if (kVals) vals[i] = vin[i];
        }
    }
}

// ------------------------------------------------------------------ single-sweep passes
// For large arrays the digit histograms of all passes come from one read of the keys (os_hist), and
// each pass is then one kernel (os_scatter): a tile takes the next tile number from a counter,
// ranks its keys as rs_scatter does, publishes its per-digit counts, and walks back over the tiles
// before it until it meets one that has published its inclusive prefix (a chained scan across the
// tiles, each step adding a predecessor's counts).  Tile numbers follow the order in which blocks
// start, so every tile a block waits on belongs to a block that is already running and publishes its
// counts without waiting on anything; the walk is bounded all the same and sets the timeout bit if it
// gives up.  Per pass the keys are read once and written once.
constexpr uint64_t kOsAgg = 1ull << 62;   // status word: the tile's own count of the digit
constexpr uint64_t kOsPre = 1ull << 63;   // status word: count of the digit over tiles 0..t
constexpr uint64_t kOsVal = kOsAgg - 1;
constexpr int kOsMaxPasses = 8;
constexpr int kOsHistThreads = 512;
constexpr int kOsHistKeys = 4;            // keys per thread whose loads are issued together

// All digit histograms from one read.  Per pass, each run of lanes that share a digit (keys arrive
// in array order, so the high digits of nearly sorted keys form long runs) adds its length once, from
// the run's first lane: a shuffle finds the run starts, a ballot of the starts gives each run's end.
template <int kPasses>
__global__ void __launch_bounds__(kOsHistThreads) os_hist(const uint64_t* keys, size_t n, uint32_t* ghist) {
    __shared__ uint32_t h[kPasses][256];
    for (int i = threadIdx.x; i < kPasses * 256; i += kOsHistThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31;
    const size_t step = (size_t)gridDim.x * kOsHistThreads * kOsHistKeys;
    // whole warps walk the array (indices past n count nothing), kOsHistKeys keys per thread, each
    // warp's 32 keys of one load contiguous
    for (size_t b = (size_t)blockIdx.x * kOsHistThreads * kOsHistKeys; b < n; b += step) {
        uint64_t k[kOsHistKeys];
#pragma unroll
        for (int u = 0; u < kOsHistKeys; ++u) {
            const size_t i = b + (size_t)u * kOsHistThreads + threadIdx.x;
            k[u] = i < n ? keys[i] : 0ull;
        }
#pragma unroll
        for (int u = 0; u < kOsHistKeys; ++u) {
            const size_t i = b + (size_t)u * kOsHistThreads + threadIdx.x;
            const unsigned live = __ballot_sync(0xffffffffu, i < n);   // a prefix of the warp's lanes
            const uint64_t prev = __shfl_up_sync(0xffffffffu, k[u], 1);
#pragma unroll
            for (int p = 0; p < kPasses; ++p) {
                const unsigned dg = (unsigned)(k[u] >> (8 * p)) & 0xFFu;
                const bool start = (lane == 0 || dg != ((unsigned)(prev >> (8 * p)) & 0xFFu)) && ((live >> lane) & 1u);
                const unsigned starts = __ballot_sync(0xffffffffu, start) | ~live;   // the dead tail ends a run
                if (start) {
                    const unsigned after = starts & ~((2u << lane) - 1u);   // run starts above this lane
                    const unsigned end = after ? (unsigned)__ffs(after) - 1u : 32u;
                    atomicAdd(&h[p][dg], end - lane);
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kPasses * 256; i += kOsHistThreads) {
        const uint32_t c = (&h[0][0])[i];
        if (c) atomicAdd(&ghist[i], c);
    }
}

// Per pass: the exclusive prefix of the 256 digit counts (one block of 256 threads per pass).
__global__ void __launch_bounds__(256) os_starts(const uint32_t* ghist, uint32_t* gstart) {
    __shared__ uint32_t wtot[8];
    const uint32_t v = ghist[blockIdx.x * 256 + threadIdx.x];
    gstart[blockIdx.x * 256 + threadIdx.x] = block_excl_scan<8>(v, wtot);
}

TJ_DEV uint64_t ld_status(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
TJ_DEV void st_status(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

// kRounds keys per thread: 8 (4096-key tiles) with values, 16 (8192-key tiles, two blocks per SM)
// for keys alone, which halves the tiles and with them the fixed per-tile cost (the barriers, the
// digit scan and the look-back round trip) against the same traffic.
template <bool kVals, int kRounds, int kByte>
__global__ void __launch_bounds__(kScThreads, 2) os_scatter(const uint64_t* keys_in, const uint32_t* vals_in,
                                                            uint64_t* keys_out, uint32_t* vals_out, size_t n,
                                                            const uint32_t* gstart, uint64_t* tstat, uint32_t* tile_ctr,
                                                            unsigned long long* status) {
    constexpr int kTile = kRounds * kScThreads;
    extern __shared__ __align__(16) unsigned char rs_dyn[];
    uint64_t* sk = (uint64_t*)rs_dyn;                      // [kTile] keys grouped by digit
    uint32_t* sv = (uint32_t*)(rs_dyn + kTile * 8);        // [kTile] values (kVals)
    __shared__ uint32_t wcnt[kScWarps][256];   // per warp and digit: count, then tile-local start
    __shared__ uint32_t gdelta[256];   // global start minus tile-local start of each digit's run (mod 2^32)
    __shared__ uint32_t wtot[kScWarps];
    __shared__ uint32_t tile_sh;
    __shared__ int gave_up;   // a look-back ran out of time: this tile writes nothing
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        tile_sh = atomicAdd(tile_ctr, 1u);
        gave_up = 0;
    }
    for (int i = threadIdx.x; i < kScWarps * 256; i += kScThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const unsigned t = tile_sh;
    const size_t tbase = (size_t)t * kTile;
    const size_t wbase = tbase + (size_t)warp * (kRounds * 32);
    uint64_t k[kRounds];
    uint32_t v[kRounds];
    uint32_t rank[kRounds];
    const unsigned lt = (1u << lane) - 1u;
    // keys of this warp's run that exist (n < 2^32, so 32-bit offsets)
    const unsigned rem = wbase >= n ? 0u : (unsigned)min(n - wbase, (size_t)(kRounds * 32));
#pragma unroll
    for (int r = 0; r < kRounds; ++r) k[r] = (unsigned)(r * 32) + lane < rem ? keys_in[wbase + r * 32 + lane] : 0ull;
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const bool ok = (unsigned)(r * 32) + lane < rem;
        const unsigned valid = __ballot_sync(0xffffffffu, ok);
        const unsigned dg = key_byte<kByte>(k[r]);
        const unsigned peers = digit_peers_lop3(dg, valid);
        const unsigned prev = ok ? wcnt[warp][dg] : 0u;
        rank[r] = ok ? prev + __popc(peers & lt) : 0xFFFFFFFFu;
        __syncwarp();
        if (ok && (peers & lt) == 0) wcnt[warp][dg] = prev + __popc(peers);
        __syncwarp();
    }
    if (kVals) {
#pragma unroll
        for (int r = 0; r < kRounds; ++r) v[r] = (unsigned)(r * 32) + lane < rem ? vals_in[wbase + r * 32 + lane] : 0u;
    }
    __syncthreads();
    {   // per digit (threads 0..255): the tile's count, published at once; its tile-local start, each
        // warp's start, and the digit's global start from the chained scan over the tiles before this one
        const unsigned dg = threadIdx.x;
        uint64_t* mine = tstat + (size_t)t * 256 + (dg & 255);
        uint32_t run = 0;
        if (dg < 256) {
#pragma unroll
            for (int w = 0; w < kScWarps; ++w) run += wcnt[w][dg];
            st_status(mine, (uint64_t)run | (t == 0 ? kOsPre : kOsAgg));
        }
        const uint32_t ls = block_excl_scan<kScWarps>(run, wtot);
        if (dg < 256) {
            uint32_t at = ls;
#pragma unroll
            for (int w = 0; w < kScWarps; ++w) {
                const uint32_t c = wcnt[w][dg];
                wcnt[w][dg] = at;
                at += c;
            }
            uint64_t excl = 0;
            if (t > 0) {
                long long j = (long long)t - 1;
                unsigned spins = 0;
                unsigned long long t0 = 0;
                while (true) {
                    const uint64_t w = ld_status(tstat + (size_t)j * 256 + dg);
                    if (w & (kOsPre | kOsAgg)) {
                        excl += w & kOsVal;
                        if ((w & kOsPre) || j == 0) break;   // tile 0 always publishes a prefix
                        --j;
                        continue;
                    }
                    if (++spins == 64) t0 = global_ns();
                    if (spins > 64) {
                        __nanosleep(32);
                        if (global_ns() - t0 > kWaitLimitNs) {
                            atomicOr(status, (unsigned long long)kStatusWaitTimeout);
                            gave_up = 1;
                            break;
                        }
                    }
                }
                st_status(mine, (excl + run) | kOsPre);
            }
            gdelta[dg] = gstart[dg] + (uint32_t)excl - ls;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        if (rank[r] != 0xFFFFFFFFu) {
            const unsigned p = wcnt[warp][key_byte<kByte>(k[r])] + rank[r];
            sk[p] = k[r];
            if (kVals) sv[p] = v[r];
        }
    }
    __syncthreads();
    if (gave_up) return;
    const unsigned cnt = (unsigned)min((size_t)kTile, n - tbase);
    bool outside = false;
    for (unsigned p = threadIdx.x; p < cnt; p += kScThreads) {
        const uint64_t key = sk[p];
        const uint32_t pos = gdelta[key_byte<kByte>(key)] + p;
        if (pos >= (uint32_t)n) {   // cannot happen with consistent counts; checked so that nothing lands outside
            outside = true;
            continue;
        }
        keys_out[pos] = key;
        if (kVals) vals_out[pos] = sv[p];
    }
    if (outside) atomicOr(status, (unsigned long long)kStatusGuard);
}

// One single-sweep pass over digit `byte` (the kernel is compiled per digit position).
template <bool kVals, int kRounds, int kByte>
void os_scatter_launch(unsigned nb, size_t dyn, cudaStream_t st, const uint64_t* kin, const uint32_t* vin,
                       uint64_t* kout, uint32_t* vout, size_t n, const uint32_t* gstart, uint64_t* tstat,
                       uint32_t* ctr, unsigned long long* status) {
    auto* f = os_scatter<kVals, kRounds, kByte>;
    TJ_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    TJ_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    launch(f, nb, kScThreads, dyn, st, kin, vin, kout, vout, n, gstart, tstat, ctr, status);
}
template <bool kVals, int kRounds>
void os_scatter_pass(int byte, unsigned nb, size_t dyn, cudaStream_t st, const uint64_t* kin, const uint32_t* vin,
                     uint64_t* kout, uint32_t* vout, size_t n, const uint32_t* gstart, uint64_t* tstat, uint32_t* ctr,
                     unsigned long long* status) {
    switch (byte) {
#define TJ_OSS(B) \
    case B: os_scatter_launch<kVals, kRounds, B>(nb, dyn, st, kin, vin, kout, vout, n, gstart, tstat, ctr, status); break;
        TJ_OSS(0) TJ_OSS(1) TJ_OSS(2) TJ_OSS(3) TJ_OSS(4) TJ_OSS(5) TJ_OSS(6) TJ_OSS(7)
#undef TJ_OSS
        default: fail(-1, "radix_sort: digit position out of range");
    }
}

}  // namespace

size_t radix_workspace_elems(size_t n) {
    const size_t nb = (n + kRsTile - 1) / kRsTile;
    const size_t h = 256 * nb;
    // the multi-pass layout (two digit tables and a scan) or the single-sweep one (a 64-bit status
    // word per tile and digit, the histograms and starts of all passes, the tile counter), whichever
    // is larger, plus alignment slack
    return std::max(2 * h + scan_workspace_elems(h), 2 * h + 2 * kOsMaxPasses * 256 + 64) + 16;
}

// Sorts (keys, vals) ascending by the low `bits` bits of keys, ping-ponging through
// keys_tmp/vals_tmp.  vals may be null.  ws: radix_workspace_elems(n) u32.  With a status word
// (device), arrays of more than kOneSweepMin keys take the single-sweep passes, whose bounded
// look-back sets kStatusWaitTimeout there if it ever gives up.  With `in_tmp`, a result that ends in
// the temporaries after an odd number of passes stays there and *in_tmp is set (the caller swaps its
// buffers); without it the result is copied back into keys/vals.
constexpr size_t kOneSweepMin = (size_t)1 << 20;

void radix_sort(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, size_t n, int bits,
                uint32_t* ws, cudaStream_t st, unsigned long long* status, bool* in_tmp) {
    if (in_tmp) *in_tmp = false;
    if (n <= 1 || bits <= 0) return;
    if (n >= (1ull << 32)) fail(-1, "radix_sort: more than 2^32 - 1 keys");
    if (status && n > kOneSweepMin) {
        const int passes = (bits + 7) / 8;
        // keys alone: 8192-key tiles; with values: 4096-key tiles
        constexpr int kRoundsK = 16, kRoundsV = 8;
        const size_t tile = (size_t)kScThreads * (vals ? kRoundsV : kRoundsK);
        const size_t dyn_k = tile * 8, dyn_kv = tile * 12;
        const unsigned nb = (unsigned)((n + tile - 1) / tile);
        uint64_t* tstat = (uint64_t*)(((uintptr_t)ws + 15) & ~(uintptr_t)15);   // [nb][256]
        uint32_t* ghist = (uint32_t*)(tstat + (size_t)nb * 256);                // [passes][256]
        uint32_t* gstart = ghist + kOsMaxPasses * 256;                           // [passes][256]
        uint32_t* ctr = gstart + kOsMaxPasses * 256;                              // [passes]
        TJ_CUDA(cudaMemsetAsync(ghist, 0, (size_t)passes * 256 * sizeof(uint32_t), st));
        TJ_CUDA(cudaMemsetAsync(ctr, 0, (size_t)passes * sizeof(uint32_t), st));
        const unsigned hb = (unsigned)std::min<size_t>((size_t)num_sms() * 4,
                                                       (n + kOsHistThreads * kOsHistKeys - 1) /
                                                           (kOsHistThreads * kOsHistKeys));
        switch (passes) {
#define TJ_OSH(P) \
    case P: launch(os_hist<P>, hb, kOsHistThreads, 0, st, (const uint64_t*)keys, n, ghist); break;
            TJ_OSH(1) TJ_OSH(2) TJ_OSH(3) TJ_OSH(4) TJ_OSH(5) TJ_OSH(6) TJ_OSH(7) TJ_OSH(8)
#undef TJ_OSH
            default: fail(-1, "radix_sort: more than 64 key bits");
        }
        launch(os_starts, (unsigned)passes, 256, 0, st, (const uint32_t*)ghist, gstart);
        uint64_t *kin = keys, *kout = keys_tmp;
        uint32_t *vin = vals, *vout = vals_tmp;
        for (int p = 0; p < passes; ++p) {
            TJ_CUDA(cudaMemsetAsync(tstat, 0, (size_t)nb * 256 * sizeof(uint64_t), st));
            if (vals)
                os_scatter_pass<true, kRoundsV>(p, nb, dyn_kv, st, kin, vin, kout, vout, n, gstart + p * 256, tstat,
                                                ctr + p, status);
            else
                os_scatter_pass<false, kRoundsK>(p, nb, dyn_k, st, kin, nullptr, kout, nullptr, n, gstart + p * 256,
                                                 tstat, ctr + p, status);
            std::swap(kin, kout);
            std::swap(vin, vout);
        }
        if (kin != keys) {
            if (in_tmp) {
                *in_tmp = true;
            } else {
                TJ_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
                if (vals) TJ_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
            }
        }
        return;
    }
    if (n <= kSmallSort) {
        const int passes = (bits + 7) / 8;
        if (vals)
            launch(rs_small<true>, 1, kScThreads, 0, st, keys, vals, keys_tmp, vals_tmp, (unsigned)n, passes);
        else
            launch(rs_small<false>, 1, kScThreads, 0, st, keys, (uint32_t*)nullptr, keys_tmp, (uint32_t*)nullptr,
                   (unsigned)n, passes);
        return;
    }
    const size_t dyn_k = (size_t)kRsTile * 8, dyn_kv = (size_t)kRsTile * 12;
    TJ_CUDA(cudaFuncSetAttribute(rs_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_k));
    TJ_CUDA(cudaFuncSetAttribute(rs_scatter<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    if (vals) {
        TJ_CUDA(cudaFuncSetAttribute(rs_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_kv));
        TJ_CUDA(cudaFuncSetAttribute(rs_scatter<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    }
    const unsigned nb = (unsigned)((n + kRsTile - 1) / kRsTile);
    const size_t h = 256 * (size_t)nb;
    uint32_t* hist = ws;
    uint32_t* offs = ws + h;
    uint32_t* sws = ws + 2 * h;
    const int passes = (bits + 7) / 8;
    uint64_t *kin = keys, *kout = keys_tmp;
    uint32_t *vin = vals, *vout = vals_tmp;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        launch(rs_hist, nb, kRsThreads, 0, st, kin, n, shift, hist, nb);
        exclusive_scan_u32(hist, offs, h, nullptr, sws, st);
        if (vals)
            launch(rs_scatter<true>, nb, kScThreads, dyn_kv, st, kin, vin, kout, vout, n, shift, offs, nb);
        else
            launch(rs_scatter<false>, nb, kScThreads, dyn_k, st, kin, nullptr, kout, nullptr, n, shift, offs, nb);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    if (kin != keys) {
        cudaMemcpyAsync(keys, kin, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
        if (vals) cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    }
}

int radix_passes(int bits) { return (bits + 7) / 8; }

bool radix_result_in_tmp(size_t n, int bits) { return n > kOneSweepMin && radix_passes(bits) % 2 == 1; }

}  // namespace tj
